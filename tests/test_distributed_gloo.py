"""The multi-rank Sigma step (xca_b200.distributed) on CPU: world size 2 over gloo.

Each rank runs self_energy_sharded with an oracle-backed evaluator whose shard is the flat indices
f with f % world == rank (the device evaluator deals work units round-robin instead; that partition
is checked on the GPU in test_gpu_sigma.py).  After the one all-reduce every rank holds the full
Sigma, which must equal the single-process sum up to the order of the summation.
"""

import os
import socket

import numpy as np
import pytest
import torch

from oracle import oracle as O
from xca_b200 import distributed, models


class OracleShardEvaluator:
    """compute_self_energy_device_shard on CPU tensors through the oracle."""

    def __init__(self, model, dlr):
        self.ev = O.Evaluator(dlr, model.beta, model.hyb_poles, model.hyb_coeffs, model.dims, model.labels,
                              model.F_index, model.F_blocks, model.Fd_index, model.Fd_blocks)
        self.slab = int(sum(dlr.r * d * d for d in model.dims))
        self.G = None

    def zero_device(self, S, n):
        S[:n] = 0.0

    def compute_self_energy_device_shard(self, G, topo, fac, S, shard, n_shards):
        t = np.array(topo, np.int32)
        nmax = self.ev.num_self_energy_backbones(t)
        fix = np.arange(shard, nmax, n_shards)
        if len(fix) == 0:
            return
        part = self.ev.compute_self_energy(self.G, t, f_ix=fix)
        S += fac * torch.from_numpy(np.concatenate([p.real.ravel() for p in part]))

    def synchronize(self):
        pass


def _model():
    d = O.Dlr(40.0, 1e-10)
    m = models.two_fermion(d.rf, d.it, 2.0, 40.0, 1e-10, U=3.0, mu=0.7, hyb_pole=-1.5)
    return m, d


def _worker(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m, d = _model()
        ev = OracleShardEvaluator(m, d)
        ev.G = m.G0
        S = torch.zeros(ev.slab, dtype=torch.float64)
        distributed.self_energy_sharded(ev, None, S, distributed.sigma_terms(3), rank, world, lambda: dist.all_reduce(S))
        np.save(f"{out_path}.{rank}.npy", S.numpy())
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_sigma_equals_single_process(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    out = str(tmp_path / "sigma")
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    m, d = _model()
    ref = O.sigma_total(O.Evaluator(d, m.beta, m.hyb_poles, m.hyb_coeffs, m.dims, m.labels, m.F_index, m.F_blocks,
                                    m.Fd_index, m.Fd_blocks), m.G0, 3)
    ref = np.concatenate([s.real.ravel() for s in ref])
    assert np.max(np.abs(ref)) > 0
    for rank in range(world):
        got = np.load(f"{out}.{rank}.npy")
        assert np.max(np.abs(got - ref)) <= 1e-14 * np.max(np.abs(ref))


def test_sharded_step_argument_checks():
    m, d = _model()
    ev = OracleShardEvaluator(m, d)
    ev.G = m.G0
    S = torch.zeros(ev.slab, dtype=torch.float64)
    with pytest.raises(ValueError):
        distributed.self_energy_sharded(ev, None, S, distributed.sigma_terms(1), 2, 2)
    with pytest.raises(ValueError):
        distributed.self_energy_sharded(ev, None, S, distributed.sigma_terms(1), 0, 2)  # no all-reduce
    distributed.self_energy_sharded(ev, None, S, distributed.sigma_terms(2), 0, 1)
    ref = np.concatenate([s.real.ravel() for s in O.sigma_total(ev.ev, m.G0, 2)])
    assert np.max(np.abs(S.numpy() - ref)) <= 1e-14 * np.max(np.abs(ref))
