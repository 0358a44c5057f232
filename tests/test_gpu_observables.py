"""GPU parity of the observables on converged or seeded propagators against the oracle:
convolve_ppsc (c++/triqs_xca/block_sparse.cpp:832-850), expectation_value (:797-818) and
compute_one_time_correlator (c++/triqs_xca/block_sparse_backbone.cpp:843-866).

Tolerances: every result is a short chain of the oracle's own operations in its order, so device and
oracle agree to round-off; 1e-13 relative to the largest entry (the correlator sums items with atomics)."""

import numpy as np
import pytest

from oracle import oracle as O
from xca_b200 import models
from xca_b200.atom_diag import FockSpace

pytestmark = pytest.mark.gpu


def _kanamori():
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    beta, lam, eps = 4.0, 40.0, 1e-8
    d = O.Dlr(lam, eps)
    m = models.kanamori_2orb(d.rf, d.it, beta, lam, eps)
    Fq = BlockOpSymQuartet(m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks, m.dims)
    ev = DiagramEvaluator.from_arrays(beta, lam, eps, d.rf, d.it, m.hyb_poles, m.hyb_coeffs, Fq)
    ora = O.Evaluator(d, beta, m.hyb_poles, m.hyb_coeffs, m.dims, m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks)
    return d, m, ev, ora


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(np.asarray(b))), 1e-300))


def test_convolve_ppsc_vs_oracle():
    d, m, ev, ora = _kanamori()
    G1, G2 = models.seeded_G(m, 4), models.seeded_G(m, 5)
    got = ev.convolve_ppsc(G1, G2)
    ref = O.convolve_ppsc(d, m.beta, G1, G2)
    worst = max(_rel(a, b) for a, b in zip(got, ref))
    print(f"convolve_ppsc: {worst:.2e}")
    assert worst <= 1e-13


def test_convolve_ppsc_free_function_matches_method():
    from xca_b200.block_sparse import convolve_ppsc
    from xca_b200.pycppdlr import MeshDLRImTime
    beta, lam, eps = 4.0, 40.0, 1e-8
    mesh = MeshDLRImTime(beta=beta, statistic="Fermion", w_max=lam / beta, eps=eps)
    m = models.kanamori_2orb(mesh.dlr_rf, mesh.dlr_it.it, beta, lam, eps)
    G1, G2 = models.seeded_G(m, 4), models.seeded_G(m, 5)
    d = O.Dlr(lam, eps, rf=mesh.dlr_rf, it=mesh.dlr_it.it)
    got = convolve_ppsc(G1, G2, mesh)
    ref = O.convolve_ppsc(d, beta, G1, G2)
    assert max(_rel(a, b) for a, b in zip(got, ref)) <= 1e-13


def test_expectation_value_vs_oracle():
    d, m, ev, ora = _kanamori()
    fs = FockSpace(m.n)
    G = models.seeded_G(m, 6)
    for op in (fs.n_op(0), fs.n_op(0) @ fs.n_op(2), sum(fs.n_op(k) for k in range(m.n))):
        idx, blks = m.ad.get_op_mat(op)
        got = ev.expectation_value(op, m.ad, G)
        ref = O.expectation_value(d, G, idx, blks)
        print(f"expectation value {got.real:+.15e} vs {ref.real:+.15e}")
        assert abs(got - ref) <= 1e-13 * max(abs(ref), 1.0)


@pytest.mark.parametrize("topo", [[[0, 1]], [[0, 2], [1, 3]], [[0, 3], [1, 4], [2, 5]]])
def test_one_time_correlator_vs_oracle(topo):
    d, m, ev, ora = _kanamori()
    fs = FockSpace(m.n)
    G = models.seeded_G(m, 7)
    ops_tau = [fs.n_op(0), fs.n_op(1)]
    ops_0 = [fs.n_op(0), fs.n_op(2), fs.n_op(3)]
    f_ix = None if len(topo) < 3 else np.arange(0, ev.get_num_single_ptcle_gf_backbones(topo), 5)
    got = ev.compute_one_time_correlator(G, ops_tau, ops_0, m.ad, topo, f_ix=f_ix)
    ref = ora.compute_one_time_correlator(G, [m.ad.get_op_mat(o) for o in ops_tau], [m.ad.get_op_mat(o) for o in ops_0],
                                          np.array(topo, np.int32), f_ix=f_ix)
    rel = _rel(got, ref)
    print(f"one-time correlator {topo}: {rel:.2e}")
    assert got.shape == (ev.r, 2, 3)
    assert np.max(np.abs(ref)) > 0
    assert rel <= 1e-13


def test_one_time_correlator_with_field_operators_is_single_particle_gf():
    # ops_tau = c_o, ops_0 = c^dag_o reproduces compute_single_ptcle_gf term for term
    d, m, ev, ora = _kanamori()
    fs = FockSpace(m.n)
    G = models.seeded_G(m, 8)
    topo = [[0, 2], [1, 3]]
    got = ev.compute_one_time_correlator(G, [fs.c(o) for o in range(m.n)], [fs.cdag(o) for o in range(m.n)], m.ad, topo)
    ref = ev.compute_single_ptcle_gf(G, topo)
    assert _rel(got, ref) <= 1e-14
