"""Sigma evaluation over several GPUs: one process per GPU, each rank evaluates an interleaved shard of every
topology's work units into its own packed Sigma slab, then one all-reduce (sum) of the slab combines the
ranks.  This replaces the reference's MPI scatter of flat indices followed by an all-reduce of each
topology's Sigma (python/triqs_xca/block_sparse_solver.py:629-640); the shards need no other exchange.

``evaluator`` is anything with the device-evaluator methods used below (``DiagramEvaluator``);
``allreduce`` sums the Sigma slab over the ranks in place (``torch.distributed.all_reduce`` on the slab's
tensor under NCCL, or under gloo in the CPU tests).
"""

from . import diag


def sigma_terms(max_order):
    """(order, topology, factor) of eval_pseudo_particle_self_energy (block_sparse_solver.py:597-640):
    Sigma = sum_order sum_topology (-1)^order * parity * (-1)^(order+1) * compute_self_energy."""
    out = []
    for order in range(1, max_order + 1):
        for sign, topo in diag.all_connected_pairings(order):
            out.append((order, topo, float((-1) ** order * sign * (-1) ** (order + 1))))
    return out


def self_energy_sharded(evaluator, G_dev, S_dev, terms, rank, world, allreduce=None):
    """S = sum over terms of factor * Sigma(topology), this rank's shard of the work, summed over ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} out of range for world size {world}")
    evaluator.zero_device(S_dev, evaluator.slab)
    for _, topo, fac in terms:
        evaluator.compute_self_energy_device_shard(G_dev, topo, fac, S_dev, rank, world)
    if world > 1:
        if allreduce is None:
            raise ValueError("world size > 1 needs an all-reduce")
        evaluator.synchronize()
        allreduce()
