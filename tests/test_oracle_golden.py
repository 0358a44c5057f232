"""Pins the CPU oracle against the reference's own known answers.

Every expectation here is a closed form or stored output written in the reference's tests:

* DLR rank r = 36 at (Lambda = 200, eps = 1e-10)   test/c++/test_block_sparse_backbone_eval.cpp:47-50
* backbone flat-index decode and vertex flags      test/c++/test_block_sparse_backbone_eval.cpp:41-134
* one-fermion Sigma, NCA/OCA/3rd order              test/c++/test_block_sparse_backbone_eval.cpp:142-268
* one-fermion single-particle G                     test/c++/test_block_sparse_backbone_gf_eval.cpp:35-133
* two-fermion Sigma and single-particle G           test/c++/test_block_sparse_two_fermions.cpp:34-150
* Volterra conv(-1, -1) = tau                       test/python/volterra_integral.py:12-34
* reflect / interpolation / full convolution        test/python/pycppdlr.py:59-141
* Fock-space matrices and H blocks                  test/c++/test_atom_diag_utils.cpp:96-239
* topologies and parities of diag.py                tests/golden/topologies.json (from the reference's diag.py)

The reference tests assert at the DLR accuracy eps on cppdlr's own node set.  This build's node set
is a restatement (the exact cppdlr placement is not pinned beyond the rank), so the Sigma / spgf
checks use 5 * eps.
"""

import json
import os

import numpy as np
import pytest

from oracle import dlr_ref
from oracle import oracle as O
from xca_b200 import diag, models
from xca_b200.atom_diag import AtomDiag, FockSpace, get_operators

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _dlr(lam, eps):
    return O.Dlr(lam, eps)


def _ev(model, dlr):
    return O.Evaluator(dlr, model.beta, model.hyb_poles, model.hyb_coeffs, model.dims, model.labels,
                       model.F_index, model.F_blocks, model.Fd_index, model.Fd_blocks)


def test_dlr_rank_pin():
    assert len(dlr_ref.build_dlr_rf(200.0, 1e-10)) == 36


def test_dlr_nodes_sorted_and_symmetric():
    rf = dlr_ref.build_dlr_rf(200.0, 1e-10)
    it = dlr_ref.build_dlr_it(200.0, rf)
    assert np.all(np.diff(rf) > 0)
    assert np.all(np.diff(dlr_ref.rel2abs(it)) > 0)
    assert np.all(np.abs(rf) <= 200.0)


def test_topologies_match_reference_diag():
    ref = json.load(open(os.path.join(GOLDEN, "topologies.json")))
    for order in range(1, 5):
        mine = [[s, [list(p) for p in t]] for s, t in diag.all_connected_pairings(order)]
        assert mine == ref[str(order)]["connected"]
        mine_all = [[s, [list(p) for p in t]] for s, t in diag.all_pairings(order)]
        assert mine_all == ref[str(order)]["all"]
    assert [len(ref[str(k)]["connected"]) for k in range(1, 5)] == [1, 1, 4, 27]


def test_oracle_topologies_match_reference_diag():
    ref = json.load(open(os.path.join(GOLDEN, "topologies.json")))
    for order in range(1, 5):
        mine = [[s, [list(p) for p in t]] for s, t in O.connected_pairings(order)]
        assert mine == ref[str(order)]["connected"]


def test_volterra_constant():
    # conv(G, G) with G = -1 is tau: the collected reference case (beta = 1, w_max = 1, eps = 1e-12)
    # asserts err < 1e-2 eps (volterra_integral.py:12-34); the sweep of its __main__ block is held to eps.
    for w_max, eps, fac in [(1.0, 1e-12, 1e-2), (10.0, 1e-10, 1.0), (100.0, 1e-8, 1.0), (1000.0, 1e-6, 1.0)]:
        beta = 1.0
        d = _dlr(w_max * beta, eps)
        G = -np.ones((d.r, 1, 1), complex)
        gc = d.vals2coefs(G)
        h = d.convolve(beta, gc, gc, time_order=True)
        err = np.max(np.abs(h[:, 0, 0] - d.tau(beta)))
        assert err < fac * eps, (w_max, eps, err)


def _free_g(H, beta, tau):
    E, U = np.linalg.eigh(H)
    g = models.kernel(tau[:, None] / beta, beta * E[None, :])  # signed kernel: G = K
    return np.einsum("lE,aE,bE->lab", g, U, U.conj())


def test_pycppdlr_reflect_interp_convolve():
    beta, lam, eps = 13.0, 200.0, 1e-8
    d = _dlr(lam, eps)
    tau = d.tau(beta)
    H = np.array([[1.0]])
    g = _free_g(H, beta, tau).astype(complex)
    assert np.max(np.abs(d.reflect(g) - _free_g(-H, beta, tau))) < 1e-6
    gc = d.vals2coefs(g)
    tf = np.linspace(0, beta, 100)
    gf = _free_g(H, beta, tf)
    interp = np.array([d.coefs2eval(gc, t / beta) for t in tf])
    # the reference asserts < eps on cppdlr's nodes; the restated node set interpolates within 2 eps
    assert np.max(np.abs(gf - interp)) < 2 * eps
    e1, e2 = 3.0, 3.3
    g1 = _free_g(np.array([[e1]]), beta, tau).astype(complex)
    g2 = _free_g(np.array([[e2]]), beta, tau).astype(complex)
    gg = d.convolve(beta, d.vals2coefs(g1), d.vals2coefs(g2), time_order=False)
    ana = (g1 - g2) / (e1 - e2)
    assert np.max(np.abs(gg - ana)) < eps


def test_convmat_matches_convolve():
    beta = 3.0
    d = _dlr(40.0, 1e-10)
    rng = np.random.default_rng(5)
    for to in (True, False):
        # f as coefficients, g as values of a DLR expansion (random values would be ill-conditioned)
        f = rng.normal(size=(d.r, 3, 3)) + 1j * rng.normal(size=(d.r, 3, 3))
        gc = rng.normal(size=(d.r, 3, 2)) + 1j * rng.normal(size=(d.r, 3, 2))
        g = d.coefs2vals(gc)
        h = d.convolve(beta, f, d.vals2coefs(g), time_order=to)
        M = d.convmat(beta, f, time_order=to)
        h2 = (M @ g.reshape(d.r * 3, 2)).reshape(d.r, 3, 2)
        assert np.max(np.abs(h - h2)) < 1e-10 * np.max(np.abs(h))


def test_backbone_indexing():
    # test_block_sparse_backbone_eval.cpp:41-134 through the oracle's item decode: the flat index
    # f_ix = o_ix + n^(m-1) (p_ix + p^(m-1) fb_ix) of fb = (1, 1, 0), poles (3, 19), orbitals (3, 2)
    rf = dlr_ref.build_dlr_rf(200.0, 1e-10)
    r, n = len(rf), 4
    assert r == 36
    fb_ix, p_ix, o_ix = 1 + 2 * 1, 3 + r * 19, 3 + n * 2
    f_ix = o_ix + p_ix * n * n + fb_ix * n * n * r * r
    assert f_ix % (n * n) == o_ix and (f_ix // (n * n)) % (r * r) == p_ix and f_ix // (n * n * r * r) == fb_ix
    assert rf[3] < 0 < rf[19]


def test_one_fermion_sigma_and_spgf():
    for beta, pole in ((2.0, 0.0), (1.0, 0.8)):
        lam, eps = 20.0 * beta, 1e-10
        d = _dlr(lam, eps)
        m = models.one_fermion(d.rf, d.it, beta, lam, eps, hyb_pole=pole)
        ev = _ev(m, d)
        t = dlr_ref.rel2abs(d.it)
        G0a = -np.exp(-t * np.log(2))
        assert np.max(np.abs(m.G0[0][:, 0, 0] - G0a)) < eps
        nca = ev.compute_self_energy(m.G0, [[0, 1]])
        oca = ev.compute_self_energy(m.G0, [[0, 2], [1, 3]])
        tca = ev.compute_self_energy(m.G0, [[0, 3], [1, 4], [2, 5]])
        g1 = ev.compute_single_ptcle_gf(m.G0, [[0, 1]])
        g2 = ev.compute_single_ptcle_gf(m.G0, [[0, 2], [1, 3]])
        g3 = ev.compute_single_ptcle_gf(m.G0, [[0, 3], [1, 4], [2, 5]])
        tol = 5 * eps
        if pole == 0.0:
            for b in range(2):
                assert np.max(np.abs(nca[b][:, 0, 0] + G0a / 2)) < tol
            ana = (beta * t) ** 4 * np.exp(-t * np.log(2)) / 192.0
            assert np.max(np.abs(tca[0][:, 0, 0] - ana)) < tol
            g3a = (beta / 2) ** 4 * (1 - t) ** 2 * t ** 2 / 2
        else:
            om, tom = pole, t * pole
            n0 = np.exp(-t * np.log(2)) * np.exp(tom) / (np.exp(beta * om) + 1)
            n1 = np.exp(-t * np.log(2)) * np.exp(-tom) / (np.exp(-beta * om) + 1)
            assert np.max(np.abs(nca[0][:, 0, 0] - n0)) < tol
            assert np.max(np.abs(nca[1][:, 0, 0] - n1)) < tol
            den = 2 * om * (om * (np.exp(beta * om) + 1)) ** 3
            a0 = (tom ** 2 * np.exp(tom) - 4 * tom * np.exp(tom) - 2 * tom + 6 * np.exp(tom) - 6) * np.exp(beta * om)
            a1 = (tom ** 2 + 4 * tom + 2 * (tom - 3) * np.exp(tom) + 6) * np.exp(om * (2 * beta - t))
            a0 *= np.exp(-t * np.log(2)) / den
            a1 *= np.exp(-t * np.log(2)) / den
            assert np.max(np.abs(tca[0][:, 0, 0] - a0)) < tol
            assert np.max(np.abs(tca[1][:, 0, 0] - a1)) < tol
            g3a = (t + (np.exp(-om * t) - 1.0) / om) * (t - beta + (np.exp(om * (beta - t)) - 1.0) / om) / (
                2 * om * om * (1 + np.exp(-beta * om)) * (np.exp(beta * om) + 1))
        for b in range(2):
            assert np.max(np.abs(oca[b])) < tol
        assert np.max(np.abs(g1[:, 0, 0] - 0.5)) < tol
        assert np.max(np.abs(g2)) < tol
        assert np.max(np.abs(g3[:, 0, 0] - g3a)) < tol


def test_two_fermion_const_hyb():
    beta, lam, eps = 2.0, 40.0, 1e-12
    d = _dlr(lam, eps)
    m = models.two_fermion(d.rf, d.it, beta, lam, eps, U=0.0, mu=0.0, hyb_pole=0.0)
    ev = _ev(m, d)
    t = dlr_ref.rel2abs(d.it)
    ln4 = 2 * np.log(2)
    G0a = -np.exp(-t * ln4)
    tol = 5 * eps * 10
    for b in range(len(m.dims)):
        assert np.max(np.abs(m.G0[b][:, 0, 0] - G0a)) < tol
    nca = ev.compute_self_energy(m.G0, [[0, 1]])
    oca = ev.compute_self_energy(m.G0, [[0, 2], [1, 3]])
    tca = ev.compute_self_energy(m.G0, [[0, 3], [1, 4], [2, 5]])
    oca_a = -0.25 * np.exp(-t * ln4) * t * t * beta * beta
    tca_a = 1.0 / 96 * np.exp(-t * ln4) * t ** 4 * beta ** 4
    for b in range(len(m.dims)):
        assert np.max(np.abs(nca[b][:, 0, 0] + G0a)) < tol
        assert np.max(np.abs(oca[b][:, 0, 0] - oca_a)) < tol
        assert np.max(np.abs(tca[b][:, 0, 0] - tca_a)) < tol
    assert np.max(np.abs(tca[1][:, 1, 1] - tca_a)) < tol
    g1 = ev.compute_single_ptcle_gf(m.G0, [[0, 1]])
    g2 = ev.compute_single_ptcle_gf(m.G0, [[0, 2], [1, 3]])
    g3 = ev.compute_single_ptcle_gf(m.G0, [[0, 3], [1, 4], [2, 5]])
    g1a = np.zeros((d.r, 2, 2))
    g1a[:, 0, 0] = g1a[:, 1, 1] = 0.5
    assert np.max(np.abs(g1 - g1a)) < tol
    g2a = 0.25 * (beta * beta * t - beta * beta * t * t)
    assert np.max(np.abs(g2[:, 0, 0] - g2a)) < tol
    assert np.max(np.abs(g2[:, 1, 1] - g2a)) < tol
    g3a = 0.5 * beta ** 4 * t * t * (-t + 0.5 * (1 + t * t)) / 16.0
    assert np.max(np.abs(g3[:, 0, 0] - 2 * g3a)) < tol
    assert np.max(np.abs(g3[:, 1, 1] - 2 * g3a)) < tol


def test_dyson_zero_sigma_returns_g0():
    # block_sparse_api_one_fermion.py:186-188: Dyson with zero self-energy reproduces G0
    beta, lam, eps = 10.0, 100.0, 1e-10
    d = _dlr(lam, eps)
    m = models.anderson(d.rf, d.it, beta, lam, eps)
    for g0 in m.G0:
        g = d.dyson_solve(beta, g0, np.zeros_like(g0), 0.0)
        assert np.max(np.abs(g - g0)) < 1e-12


def test_dyson_first_order_expansion():
    # G = G0 + G0 * Sigma * G0 + O(Sigma^2) for a small Sigma
    beta, lam, eps = 5.0, 50.0, 1e-12
    d = _dlr(lam, eps)
    m = models.kanamori_2orb(d.rf, d.it, beta, lam, eps)
    rng = np.random.default_rng(3)
    for g0 in m.G0:
        nb = g0.shape[1]
        s = 1e-6 * (rng.normal(size=g0.shape))
        g = d.dyson_solve(beta, g0, s, 0.0)
        gs = d.convolve(beta, d.vals2coefs(g0), d.vals2coefs(s), time_order=True)
        lin = g0 + d.convolve(beta, d.vals2coefs(gs), d.vals2coefs(g0), time_order=True)
        assert np.max(np.abs(g - lin)) < 1e-9, nb  # second order: O(beta^2 |Sigma|^2)


def test_atom_diag_fock_matrices():
    # test_atom_diag_utils.cpp:96-168: two-orbital model, fops (do 0, do 1, up 0, up 1)
    fs = FockSpace(4)
    c = [fs.c(k) for k in range(4)]
    cd = [x.T for x in c]
    n_ = [cd[k] @ c[k] for k in range(4)]
    do, up = (0, 1), (2, 3)
    H = sum(1.0 * n_[up[i]] @ n_[do[i]] + 0.25 * (n_[up[i]] + n_[do[i]]) + 0.1 * (cd[up[i]] @ c[do[i]] + cd[do[i]] @ c[up[i]])
            for i in range(2))
    exp = np.zeros((16, 16))
    for (i, j), v in {(1, 1): .25, (1, 4): .1, (2, 2): .25, (2, 8): .1, (3, 3): .5, (3, 6): -.1, (3, 9): .1, (4, 1): .1,
                      (4, 4): .25, (5, 5): 1.5, (6, 3): -.1, (6, 6): .5, (6, 12): -.1, (7, 7): 1.75, (7, 13): -.1,
                      (8, 2): .1, (8, 8): .25, (9, 3): .1, (9, 9): .5, (9, 12): .1, (10, 10): 1.5, (11, 11): 1.75,
                      (11, 14): -.1, (12, 6): -.1, (12, 9): .1, (12, 12): .5, (13, 7): -.1, (13, 13): 1.75,
                      (14, 11): -.1, (14, 14): 1.75, (15, 15): 3.0}.items():
        exp[i, j] = v
    assert np.max(np.abs(H - exp)) < 1e-13
    ad = AtomDiag(H, 4)
    blocks = [[[0.0]], [[.25, .1], [.1, .25]], [[.25, .1], [.1, .25]],
              [[.5, -.1, .1, 0], [-.1, .5, 0, -.1], [.1, 0, .5, .1], [0, -.1, .1, .5]],
              [[1.5]], [[1.5]], [[1.75, -.1], [-.1, 1.75]], [[1.75, -.1], [-.1, 1.75]], [[3.0]]]
    assert ad.n_subspaces == 9
    for hb, eb in zip(ad.H_blocks, blocks):
        assert np.max(np.abs(hb - np.array(eb))) < 1e-13
    labels, *_ = get_operators(ad)
    assert list(labels) == [0, 1, 0, 1]


def test_oracle_item_list_is_stable():
    # the item list (find_path_self_energy) of a 2-orbital Kanamori TCA topology is reproducible
    beta, lam, eps = 20.0, 40.0, 1e-8
    d = _dlr(lam, eps)
    m = models.kanamori_2orb(d.rf, d.it, beta, lam, eps)
    ev = _ev(m, d)
    G = models.seeded_G(m, 0)
    a = ev.item_list(G, [[0, 2], [1, 4], [3, 5]], 0, 2000)
    b = ev.item_list(G, [[0, 2], [1, 4], [3, 5]], 0, 2000)
    assert a.shape[0] > 0 and np.array_equal(a, b)


def test_get_op_mat_matches_field_operator_blocks():
    # the block form of c_k from AtomDiag.get_op_mat is the F slab of k's symmetry set
    from xca_b200 import models
    from xca_b200.atom_diag import FockSpace
    d = O.Dlr(40.0, 1e-8)
    m = models.kanamori_2orb(d.rf, d.it, 4.0, 40.0, 1e-8)
    fs = FockSpace(m.n)
    sinds = {}
    for o in range(m.n):
        sinds[o] = sum(1 for o2 in range(o) if m.labels[o2] == m.labels[o])
    for o in range(m.n):
        idx, blks = m.ad.get_op_mat(fs.c(o))
        s = m.labels[o]
        assert np.array_equal(idx, m.F_index[s])
        for b in range(len(idx)):
            if idx[b] >= 0:
                assert np.array_equal(blks[b], m.F_blocks[s][b][sinds[o]])
    # a density is block diagonal
    idx, _ = m.ad.get_op_mat(fs.n_op(1))
    assert all(i in (-1, b) for b, i in enumerate(idx))
