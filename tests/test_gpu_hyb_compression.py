"""Sigma and solves with a compressed hybridization (a few fitted poles in place of one per DLR frequency,
fit_hybridization(compression=True), python/triqs_xca/block_sparse_solver.py:146-185).

The evaluator takes any pole set, so the device is held to the oracle on the same compressed poles (bit for
bit in the ordered mode); against the uncompressed representation the results differ by the fit error."""

import time

import numpy as np
import pytest

from oracle import oracle as O
from xca_b200 import hyb_fit, models

pytestmark = pytest.mark.gpu


def _t2g_compressed():
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    beta, lam, eps = 50.0, 500.0, 1e-10
    d = O.Dlr(lam, eps)
    m = models.t2g_3orb(d.rf, d.it, beta, lam, eps)
    delta = (models.kernel(d.it[:, None], d.rf[None, :]) @ m.hyb_coeffs.reshape(d.r, -1)).reshape(d.r, 6, 6)
    poles, coeffs, err = hyb_fit.compress_hybridization(d.rf, d.it, beta, delta, 1e-9)
    Fq = BlockOpSymQuartet(m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks, m.dims)
    ev = DiagramEvaluator.from_arrays(beta, lam, eps, d.rf, d.it, poles, coeffs, Fq)
    ora = O.Evaluator(d, beta, poles, coeffs, m.dims, m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks)
    return d, m, ev, ora, poles


def test_t2g_compressed_sigma_ordered_vs_oracle():
    d, m, ev, ora, poles = _t2g_compressed()
    assert len(poles) == 8
    ev.precision_mode = "fp64_ordered"
    G = models.seeded_G(m, 0)
    oca = np.array([[0, 2], [1, 3]], np.int32)
    got = ev.compute_self_energy(G, oca)
    ref = ora.compute_self_energy_ordered(G, oca)
    assert all(np.array_equal(a, b) for a, b in zip(got, ref))
    tca = np.array([[0, 3], [1, 4], [2, 5]], np.int32)
    fix = np.sort(np.random.default_rng(5).choice(ev.get_num_self_energy_backbones(tca), 400, replace=False))
    got = ev.compute_self_energy(G, tca, f_ix=fix)
    ref = ora.compute_self_energy_list_ordered(G, tca, fix)
    assert all(np.array_equal(a, b) for a, b in zip(got, ref))
    assert max(np.max(np.abs(x)) for x in ref) > 0


def test_kanamori_tca_compressed_vs_dlr_poles():
    # the benchmark model's TCA Sigma with the DLR poles and with a compressed Bethe hybridization
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    beta, lam, eps = 20.0, 200.0, 1e-12
    d = O.Dlr(lam, eps)
    m = models.kanamori_2orb(d.rf, d.it, beta, lam, eps)
    dv = models.bethe_delta(beta, d.it)
    delta = np.zeros((d.r, 4, 4))
    for i in range(4):
        delta[:, i, i] = dv
    poles, coeffs, err = hyb_fit.compress_hybridization(d.rf, d.it, beta, delta, 1e-10)
    Fq = BlockOpSymQuartet(m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks, m.dims)
    G = models.seeded_G(m, 0)
    out, times = {}, {}
    for name, (p, c) in (("dlr", (m.hyb_poles, m.hyb_coeffs)), ("compressed", (poles, coeffs))):
        ev = DiagramEvaluator.from_arrays(beta, lam, eps, d.rf, d.it, p, c, Fq)
        bg, bs = ev.device_buffer(30, ev.slab), ev.device_buffer(31, ev.slab)
        ev.to_device(bg, ev.pack(G).real)
        tot = np.zeros(ev.slab)
        for rep in range(2):
            ev.zero_device(bs, ev.slab)
            ev.synchronize()
            t0 = time.perf_counter()
            for order in (1, 2, 3):
                for sign, topo in O.connected_pairings(order):
                    ev.compute_self_energy_device(bg, topo, float((-1) ** order * sign * (-1) ** (order + 1)), bs)
            ev.synchronize()
            times[name] = time.perf_counter() - t0
        out[name] = ev.to_host(bs, ev.slab)
    rel = np.max(np.abs(out["compressed"] - out["dlr"])) / np.max(np.abs(out["dlr"]))
    print(f"Kanamori orders 1-3: {len(m.hyb_poles)} DLR poles {times['dlr'] * 1e3:.1f} ms, {len(poles)} fitted poles "
          f"{times['compressed'] * 1e3:.1f} ms (fit error {err:.1e}); Sigma differs by {rel:.1e} of its maximum")
    assert len(poles) < len(m.hyb_poles) // 2
    assert times["compressed"] < times["dlr"]


def test_anderson_oca_solve_with_compression():
    from xca_b200.block_sparse_solver import BlockSparseSolver
    from xca_b200.pycppdlr import MeshDLRImTime
    beta, lam, eps = 10.0, 100.0, 1e-10
    mesh = MeshDLRImTime(beta=beta, statistic="Fermion", w_max=lam / beta, eps=eps)
    m = models.anderson(mesh.dlr_rf, mesh.dlr_it.it, beta, lam, eps)
    res = {}
    for comp in (False, True):
        S = BlockSparseSolver(m.ad, beta, lam / beta, eps, precision="fp64_ordered")
        delta = np.zeros((S.r, 2, 2), np.complex128)
        dv = models.bethe_delta(beta, S.it)
        delta[:, 0, 0] = dv
        delta[:, 1, 1] = dv
        S.Delta_tau = delta
        S.solve(max_order=2, tol=1e-9, maxiter=60, hyb_comp=comp, hyb_tol=1e-10)
        res[comp] = S
    S = res[True]
    assert S.hyb_compression and len(S.hyb_poles) < S.r // 2
    d = O.Dlr(lam, eps, rf=S.rf, it=S.it)
    ev = O.Evaluator(d, beta, S.hyb_poles, S.hyb_coeffs, m.dims, m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks)
    G, Sig, eta, g, n_iter, diff = O.solve(d, ev, beta, m.G0, 2, 1e-9, 60, spgf_max_order=2, ordered=True)
    assert S.n_ppsc_iter == n_iter
    assert max(float(np.max(np.abs(a - b))) for a, b in zip(S.G, G)) <= 1e-13
    dG = max(float(np.max(np.abs(a - b))) for a, b in zip(S.G, res[False].G))
    print(f"Anderson OCA: {len(S.hyb_poles)} fitted poles vs {S.r} DLR poles, converged G differ by {dG:.1e}")
    assert dG < 1e-7
