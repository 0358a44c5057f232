"""Job-batched Sigma (``DiagramEvaluator.compute_self_energy_device_batch``): the panel work of many
(evaluator, topology) jobs in one launch.  Each job's Sigma must equal the oracle's golden values to the
fast mode's tolerance (1e-12 relative per tau node, items summed with atomics in a varying order), the
evaluators sharing a device and a padded DLR rank; the d shell's wide chains follow the batch on their own
evaluator's stream.  Mixed padded ranks, the ordered mode and two G's of one evaluator are refused."""

import os

import numpy as np
import pytest

from oracle import oracle as O
from xca_b200 import models

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_FAST_PER_NODE = 1e-12


def _evaluator(name, builder):
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    path = os.path.join(GOLDEN, f"sigma_{name}_ordered.npz")
    if not os.path.exists(path):
        pytest.skip(f"golden file {path} not generated")
    fx = np.load(path)
    beta, lam, eps = float(fx["beta"]), float(fx["lam"]), float(fx["eps"])
    m = builder(fx["rf"], fx["it"], beta, lam, eps)
    Fq = BlockOpSymQuartet(m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks, m.dims)
    ev = DiagramEvaluator.from_arrays(beta, lam, eps, fx["rf"], fx["it"], m.hyb_poles, m.hyb_coeffs, Fq)
    return fx, ev


def _per_node_rel(ev, a, b):
    r = ev.r
    num, den, off = np.zeros(r), np.zeros(r), 0
    for d in ev.dims:
        sz = r * d * d
        num = np.maximum(num, np.max(np.abs(a[off:off + sz] - b[off:off + sz]).reshape(r, -1), axis=1))
        den = np.maximum(den, np.max(np.abs(b[off:off + sz]).reshape(r, -1), axis=1))
        off += sz
    return float(np.max(num / np.maximum(den, 1e-300)))


def _on_device(ev, fx, slot):
    buf_g = ev.device_buffer(slot, ev.slab)
    ev.to_device(buf_g, fx["G"])
    return buf_g


def test_batch_of_two_evaluators_matches_golden():
    from xca_b200.block_sparse import DiagramEvaluator
    fk, ek = _evaluator("kanamori_2orb", models.kanamori_2orb)
    fo, eo = _evaluator("t2g_oca", models.t2g_3orb)
    ft, _ = _evaluator("t2g_tca", models.t2g_3orb)
    assert ek.padded_rank == eo.padded_rank == 48
    assert np.array_equal(fo["G"], ft["G"])
    gk, go = _on_device(ek, fk, 30), _on_device(eo, fo, 30)
    jobs, gold = [], []
    # one output slab per job (scale 1), and one slab for the signed total of the Kanamori orders 1-3
    for k in range(int(fk["n_topologies"])):
        jobs.append((ek, gk, fk[f"topo_{k}"], 1.0, ek.device_buffer(40 + k, ek.slab)))
        gold.append((ek, fk[f"sigma_{k}"]))
    for k in range(int(fo["n_topologies"])):
        jobs.append((eo, go, fo[f"topo_{k}"], 1.0, eo.device_buffer(40 + k, eo.slab)))
        gold.append((eo, fo[f"sigma_{k}"]))
    jobs.append((eo, go, ft["topo_0"], 1.0, eo.device_buffer(50, eo.slab)))
    gold.append((eo, ft["sigma_0"]))
    total = ek.device_buffer(60, ek.slab)
    ek.zero_device(total, ek.slab)
    facs = [(-1) ** o * s * (-1) ** (o + 1) for o in (1, 2, 3) for s, _ in O.connected_pairings(o)]
    gold_total = sum(f * fk[f"sigma_{k}"] for k, f in enumerate(facs))
    for k, f in enumerate(facs):
        jobs.append((ek, gk, fk[f"topo_{k}"], float(f), total))
    for j in jobs[:len(gold)]:
        j[0].zero_device(j[4], j[0].slab)
    # the t2g evaluator leads: its stream carries the launch, the Kanamori stream is ordered after it
    order = [len(jobs) - len(facs) - 1] + [i for i in range(len(jobs)) if i != len(jobs) - len(facs) - 1]
    DiagramEvaluator.compute_self_energy_device_batch([jobs[i] for i in order])
    worst = 0.0
    for (ev, g), j in zip(gold, jobs):
        got = ev.to_host(j[4], ev.slab)
        assert np.max(np.abs(g)) > 0
        worst = max(worst, _per_node_rel(ev, got, g))
    rel_total = _per_node_rel(ek, ek.to_host(total, ek.slab), gold_total)
    print(f"batched jobs vs golden: worst per-node {worst:.2e}; Kanamori signed total {rel_total:.2e}")
    assert worst <= TOL_FAST_PER_NODE and rel_total <= TOL_FAST_PER_NODE


def test_batch_refusals():
    from xca_b200.block_sparse import DiagramEvaluator
    fk, ek = _evaluator("kanamori_2orb", models.kanamori_2orb)
    fd, ed = _evaluator("dshell_subsets", models.dshell_5orb)
    assert ed.padded_rank == 32 and ek.padded_rank == 48
    gk, gd = _on_device(ek, fk, 30), _on_device(ed, fd, 30)
    sk, sd = ek.device_buffer(31, ek.slab), ed.device_buffer(31, ed.slab)
    topo = [[0, 1]]
    with pytest.raises(ValueError):
        DiagramEvaluator.compute_self_energy_device_batch([(ek, gk, topo, 1.0, sk), (ed, gd, topo, 1.0, sd)])
    with pytest.raises(ValueError):
        DiagramEvaluator.compute_self_energy_device_batch([(ek, gk, topo, 1.0, sk), (ek, sk, topo, 1.0, gk)])
    ek.precision_mode = "fp64_ordered"
    with pytest.raises(NotImplementedError):
        DiagramEvaluator.compute_self_energy_device_batch([(ek, gk, topo, 1.0, sk)])


def test_batch_wide_chains_dshell():
    # the d shell's 100 x 100 blocks run on the wide kernel after the batched panel launch; NCA and OCA
    # batched against one ordered evaluation per topology on the same evaluator
    from xca_b200.block_sparse import DiagramEvaluator
    fd, ed = _evaluator("dshell_subsets", models.dshell_5orb)
    gd = _on_device(ed, fd, 30)
    topos = [[[0, 1]], [[0, 2], [1, 3]]]
    outs = [ed.device_buffer(40 + k, ed.slab) for k in range(len(topos))]
    for o in outs:
        ed.zero_device(o, ed.slab)
    DiagramEvaluator.compute_self_energy_device_batch([(ed, gd, t, 1.0, o) for t, o in zip(topos, outs)])
    got = [ed.to_host(o, ed.slab) for o in outs]
    ed.precision_mode = "fp64_ordered"
    for t, g in zip(topos, got):
        ref = ed.device_buffer(50, ed.slab)
        ed.zero_device(ref, ed.slab)
        ed.compute_self_energy_device(gd, t, 1.0, ref)
        rel = _per_node_rel(ed, g, ed.to_host(ref, ed.slab))
        print(f"d shell {t}: batched vs ordered per-node {rel:.2e}")
        assert rel <= TOL_FAST_PER_NODE
