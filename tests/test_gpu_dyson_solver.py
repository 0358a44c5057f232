"""GPU parity of the Dyson solve, the trace / normalisation and the self-consistent loop against the oracle.

Tolerances: the Dyson system matrix I + M is well conditioned for these pseudo-particle problems, so
device and oracle agree to round-off; we require 1e-12 relative to the block's largest entry.  The
trace and the normalisation: 1e-13 relative.  The self-consistent solve compounds the round-off of the
Sigma accumulation (items are summed in another order on the device) over the iterations: G, Sigma
and eta must agree to 1e-10 (the convergence tolerance of the solve is 1e-10 as well).
"""

import numpy as np
import pytest

from oracle import oracle as O
from xca_b200 import models

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("eta", [0.0, 0.7])
def test_dyson_block_vs_oracle(eta):
    # Sigma = the NCA self-energy of G0 (what the solve loop feeds the Dyson solver), Kanamori, Lambda = 200
    from xca_b200.dlr_dyson_ppsc import DysonItPPSC
    from xca_b200.pycppdlr import ImTimeOps, build_dlr_rf
    beta, lam, eps = 20.0, 200.0, 1e-12
    itops = ImTimeOps(lam, build_dlr_rf(lam, eps))
    d = O.Dlr(lam, eps, rf=itops.get_rfnodes(), it=itops.get_itnodes())
    m = models.kanamori_2orb(d.rf, d.it, beta, lam, eps)
    ora = O.Evaluator(d, beta, m.hyb_poles, m.hyb_coeffs, m.dims, m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks)
    Sig = [-s for s in ora.compute_self_energy(m.G0, np.array([[0, 1]], np.int32))]
    for b, g0 in enumerate(m.G0):
        dev = DysonItPPSC(beta, itops, g0).solve(Sig[b], eta)
        ref = d.dyson_solve(beta, g0, Sig[b], eta)
        assert _rel(dev, ref) < 1e-12, b
        herm = DysonItPPSC(beta, itops, g0).solve(Sig[b], eta, hermitize=True)
        assert _rel(herm, 0.5 * (ref + np.transpose(ref, (0, 2, 1)))) < 1e-12, b


def test_dyson_backward_error_strong_sigma():
    # a strong, arbitrary Sigma (0.3 x a seeded propagator) makes I + M ill-conditioned, so device and oracle
    # solutions may differ by cond * 1e-16; the device solution must still solve the oracle's system:
    # ||(I + M) g - g0|| <= 1e-13 (||I + M|| ||g|| + ||g0||) (max norms)
    from xca_b200.dlr_dyson_ppsc import DysonItPPSC
    from xca_b200.pycppdlr import ImTimeOps, build_dlr_rf
    beta, lam, eps = 20.0, 200.0, 1e-12
    itops = ImTimeOps(lam, build_dlr_rf(lam, eps))
    d = O.Dlr(lam, eps, rf=itops.get_rfnodes(), it=itops.get_itnodes())
    m = models.kanamori_2orb(d.rf, d.it, beta, lam, eps)
    G = models.seeded_G(m, 3)
    for b, g0 in enumerate(m.G0):
        sig, eta = 0.3 * G[b], 0.7
        g = DysonItPPSC(beta, itops, g0).solve(sig, eta)
        r, n = g0.shape[:2]
        ggs = -(d.convolve(beta, d.vals2coefs(g0), d.vals2coefs(sig), time_order=True) + eta * g0)
        A = np.eye(r * n) + d.convmat(beta, d.vals2coefs(ggs), time_order=True)
        res = A @ g.reshape(r * n, n) - g0.reshape(r * n, n)
        bound = np.max(np.abs(A).sum(axis=1)) * np.max(np.abs(g)) + np.max(np.abs(g0))
        assert np.max(np.abs(res)) <= 1e-13 * bound, b


@pytest.mark.parametrize("kind", ["kanamori", "anderson"])
def test_dyson_lu_paths_bit_identical(kind):
    # the three factorisations of the Dyson system -- one CTA with the matrix in shared memory (N <= 160),
    # one CTA in global memory, the multi-CTA blocked LU -- perform the same operations in the same order:
    # the solutions agree bit for bit, and with the oracle's solve to 1e-12 (Kanamori N = 168; Anderson N = r, 1 x 1 blocks)
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    beta, lam, eps = (20.0, 200.0, 1e-12) if kind == "kanamori" else (10.0, 100.0, 1e-10)
    d = O.Dlr(lam, eps)
    m = (models.kanamori_2orb if kind == "kanamori" else models.anderson)(d.rf, d.it, beta, lam, eps)
    Fq = BlockOpSymQuartet(m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks, m.dims)
    ev = DiagramEvaluator.from_arrays(beta, lam, eps, d.rf, d.it, m.hyb_poles, m.hyb_coeffs, Fq)
    ev.dyson_setup(m.G0)
    G = models.seeded_G(m, 2)
    sig = [0.05 * g for g in G]
    bs, bg = ev.device_buffer(30, ev.slab), ev.device_buffer(31, ev.slab)
    ev.to_device(bs, ev.pack(sig).real)
    outs = {}
    n_max = d.r * int(max(m.dims))
    for name, thr in (("one_cta", 1 << 30), ("blocked", 0)):
        ev.set_tuning(dyson_blocked_min_n=thr)
        ev.dyson_solve_device(bs, 0.4, bg, hermitize=False)
        outs[name] = ev.to_host(bg, ev.slab)
    assert np.array_equal(outs["one_cta"], outs["blocked"]), n_max
    ref = np.concatenate([d.dyson_solve(beta, g0, s, 0.4).real.ravel() for g0, s in zip(m.G0, sig)])
    assert _rel(outs["blocked"], ref) < 1e-12
    print(f"{kind}: N = {n_max}, LU paths identical, |dev - oracle| / max = {_rel(outs['blocked'], ref):.2e}")


def test_dyson_zero_sigma_returns_g0():
    from xca_b200.dlr_dyson_ppsc import DysonItPPSC
    from xca_b200.pycppdlr import ImTimeOps, build_dlr_rf
    beta, lam, eps = 10.0, 100.0, 1e-10
    itops = ImTimeOps(lam, build_dlr_rf(lam, eps))
    m = models.anderson(itops.get_rfnodes(), itops.get_itnodes(), beta, lam, eps)
    for g0 in m.G0:
        g = DysonItPPSC(beta, itops, g0).solve(np.zeros_like(g0), 0.0)
        assert _rel(g, g0) < 1e-13


def _evaluator(beta, lam, eps, model_fn):
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    d = O.Dlr(lam, eps)
    m = model_fn(d.rf, d.it, beta, lam, eps)
    Fq = BlockOpSymQuartet(m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks, m.dims)
    ev = DiagramEvaluator.from_arrays(beta, lam, eps, d.rf, d.it, m.hyb_poles, m.hyb_coeffs, Fq)
    return d, m, ev


def test_trace_and_normalize_vs_oracle():
    beta, lam, eps = 20.0, 200.0, 1e-12
    d, m, ev = _evaluator(beta, lam, eps, models.kanamori_2orb)
    G = [1.7 * g for g in m.G0]
    tr = ev.trace(G)
    ref = O.trace_beta(d, G)
    assert abs(tr - ref) <= 1e-13 * abs(ref)
    buf = ev.device_buffer(20, ev.slab)
    ev.to_device(buf, ev.pack(G).real)
    assert abs(ev.trace_device(buf) - ref) <= 1e-13 * abs(ref)
    Z, de = ev.normalize_device(buf)
    Gn = [x.astype(np.complex128) for x in ev.unpack(ev.to_host(buf, ev.slab))]
    Gr, eta = O.normalize(d, beta, G, 0.0)
    assert abs(Z + ref.real) <= 1e-13 * abs(ref)
    assert abs(de - eta) <= 1e-14 * max(abs(eta), 1.0)
    for a, b in zip(Gn, Gr):
        assert _rel(a, b) < 1e-13


def test_device_mixing_and_max_abs_diff():
    beta, lam, eps = 4.0, 40.0, 1e-8
    d, m, ev = _evaluator(beta, lam, eps, models.kanamori_2orb)
    A = models.seeded_G(m, 1)
    Bm = models.seeded_G(m, 2)
    a = ev.device_buffer(21, ev.slab)
    b = ev.device_buffer(22, ev.slab)
    ev.to_device(a, ev.pack(A).real)
    ev.to_device(b, ev.pack(Bm).real)
    ref = max(np.max(np.abs(x - y)) for x, y in zip(A, Bm))
    assert ev.max_abs_diff_device(a, b) == ref
    ev.axpby_device(0.3, a, 0.7, b)
    got = ev.unpack(ev.to_host(b, ev.slab))
    for g, x, y in zip(got, A, Bm):
        assert np.array_equal(g, (0.3 * x + 0.7 * y).real)


@pytest.mark.parametrize("max_order", [1, 2])
def test_anderson_self_consistent_solve_vs_oracle(max_order):
    # the single-orbital Anderson impurity (U = 2, mu = 1, beta = 10, Lambda = 100, eps = 1e-10, Bethe t = 1)
    from xca_b200.block_sparse_solver import BlockSparseSolver
    from xca_b200.pycppdlr import MeshDLRImTime
    beta, lam, eps = 10.0, 100.0, 1e-10
    mesh = MeshDLRImTime(beta=beta, statistic="Fermion", w_max=lam / beta, eps=eps)
    m = models.anderson(mesh.dlr_rf, mesh.dlr_it.it, beta, lam, eps)
    S = BlockSparseSolver(m.ad, beta, lam / beta, eps)
    delta = np.zeros((S.r, 2, 2), np.complex128)
    dv = models.bethe_delta(beta, S.it)
    delta[:, 0, 0] = dv
    delta[:, 1, 1] = dv
    S.Delta_tau = delta
    S.solve(max_order=max_order, tol=1e-10, maxiter=60, mix=1.0, hyb_comp=False)

    d = O.Dlr(lam, eps, rf=S.rf, it=S.it)
    ev = O.Evaluator(d, beta, S.hyb_poles, S.hyb_coeffs, m.dims, m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks)
    G, Sig, eta, g, n_iter, diff = O.solve(d, ev, beta, m.G0, max_order, 1e-10, 60, mix=1.0, spgf_max_order=max_order)
    assert diff < 1e-10 and S.diff_G < 1e-10
    assert abs(S.n_ppsc_iter - n_iter) <= 1
    assert abs(S.eta - eta) < 1e-10
    for a, b in zip(S.G, G):
        assert np.max(np.abs(a - b)) < 1e-10
    for a, b in zip(S.Sigma, Sig):
        assert np.max(np.abs(a - b)) < 1e-10 * max(1.0, np.max(np.abs(b)))
    # single-particle G(tau) of the converged propagator, orders 1..max_order
    assert np.max(np.abs(S.G_tau - g)) < 1e-10
    assert np.max(np.abs(g)) > 0.1


def test_t2g_nca_solve_vs_oracle():
    # three-orbital t2g Kanamori, NCA self-consistent solve and single-particle G(tau) (16 blocks up to 9 x 9)
    from xca_b200.block_sparse_solver import BlockSparseSolver
    from xca_b200.pycppdlr import MeshDLRImTime
    beta, lam, eps = 50.0, 500.0, 1e-10
    mesh = MeshDLRImTime(beta=beta, statistic="Fermion", w_max=lam / beta, eps=eps)
    m = models.t2g_3orb(mesh.dlr_rf, mesh.dlr_it.it, beta, lam, eps)
    S = BlockSparseSolver(m.ad, beta, lam / beta, eps)
    rf, it = S.rf, S.it
    S.Delta_tau = np.asarray(models.kernel(it[:, None], rf[None, :]) @ m.hyb_coeffs.reshape(len(rf), -1)).reshape(S.Delta_tau.shape)
    S.solve(max_order=1, tol=1e-8, maxiter=40, mix=1.0, hyb_comp=False)
    d = O.Dlr(lam, eps, rf=rf, it=it)
    ev = O.Evaluator(d, beta, S.hyb_poles, S.hyb_coeffs, m.dims, m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks)
    G, Sig, eta, g, n_iter, diff = O.solve(d, ev, beta, m.G0, 1, 1e-8, 40, mix=1.0, spgf_max_order=1)
    # the item sums run in another (and run-to-run varying) order on the device (1e-16), and this model's
    # Sigma amplifies input differences by up to ~1e7 (items with poles near +-Lambda), so two converged
    # iterations agree to a few times the convergence tolerance of the solve (1e-8), not to round-off:
    # the bound is 10 x tol
    assert diff < 1e-8 and S.diff_G < 1e-8
    assert abs(S.eta - eta) < 1e-8
    for a, b in zip(S.G, G):
        assert np.max(np.abs(a - b)) < 1e-7
    assert np.max(np.abs(S.G_tau - g)) < 1e-7


def test_dyson_concurrent_contexts_of_different_sizes():
    # two contexts in two threads solve Dyson systems of different sizes at the same time, both with the
    # matrix in shared memory: every launch must find the kernel's shared-memory limit above its own size
    # (the limit is the kernel's, not the context's), and each result must equal its solve alone
    import threading
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    cases = []
    for builder, beta, lam, eps in ((models.anderson, 10.0, 100.0, 1e-10), (models.kanamori_2orb, 4.0, 40.0, 1e-8)):
        d = O.Dlr(lam, eps)
        m = builder(d.rf, d.it, beta, lam, eps)
        Fq = BlockOpSymQuartet(m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks, m.dims)
        ev = DiagramEvaluator.from_arrays(beta, lam, eps, d.rf, d.it, m.hyb_poles, m.hyb_coeffs, Fq)
        ev.dyson_setup(m.G0)
        bs, bg = ev.device_buffer(30, ev.slab), ev.device_buffer(31, ev.slab)
        ev.to_device(bs, ev.pack([0.05 * g for g in models.seeded_G(m, 4)]).real)
        ev.dyson_solve_device(bs, 0.3, bg)
        cases.append((ev, bs, bg, ev.to_host(bg, ev.slab), d.r * int(max(m.dims))))
    assert cases[0][4] != cases[1][4] and max(c[4] for c in cases) <= 160
    errors = []

    def work(ev, bs, bg, ref, _n):
        try:
            for _ in range(300):
                ev.dyson_solve_device(bs, 0.3, bg)
            assert np.array_equal(ev.to_host(bg, ev.slab), ref)
        except BaseException as e:  # reported to the main thread
            errors.append(e)

    threads = [threading.Thread(target=work, args=c) for c in cases]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors


def test_dyson_solve_with_op_vs_oracle():
    # solve_with_op(sig, eta, op) (dlr_dyson_ppsc.hpp:188-216): the source term gains G0(t) op; per Kanamori block
    # against the oracle's restatement (1e-12), and with op = 0 equal to solve() bit for bit
    from xca_b200.dlr_dyson_ppsc import DysonItPPSC
    from xca_b200.pycppdlr import ImTimeOps, build_dlr_rf
    beta, lam, eps = 20.0, 200.0, 1e-12
    itops = ImTimeOps(lam, build_dlr_rf(lam, eps))
    d = O.Dlr(lam, eps, rf=itops.get_rfnodes(), it=itops.get_itnodes())
    m = models.kanamori_2orb(d.rf, d.it, beta, lam, eps)
    ora = O.Evaluator(d, beta, m.hyb_poles, m.hyb_coeffs, m.dims, m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks)
    Sig = [-s for s in ora.compute_self_energy(m.G0, np.array([[0, 1]], np.int32))]
    rng = np.random.default_rng(5)
    for b, g0 in enumerate(m.G0):
        n = g0.shape[1]
        a = rng.normal(0.0, 0.3, (n, n))
        op = a + a.T
        solver = DysonItPPSC(beta, itops, g0)
        dev = solver.solve_with_op(Sig[b], 0.4, op)
        ref = d.dyson_solve(beta, g0, Sig[b], 0.4, op=op)
        assert _rel(dev, ref) < 1e-12, b
        assert np.array_equal(solver.solve_with_op(Sig[b], 0.4, np.zeros((n, n))), solver.solve(Sig[b], 0.4)), b
