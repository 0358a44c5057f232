"""Conditioning of the reference's Sigma evaluation (CPU, oracle only): how much a relative perturbation of
the input propagator G moves Sigma, per order, per input and per pole representation of the hybridization,
and where the amplification comes from.

* The K(0)^-e prefactors are not the source: Backbone::set_pole_inds (c++/triqs_xca/backbone.cpp:86-150) picks
  case 4(a) or 4(b) so that every divisor is K(0, x) at x >= 0, whose magnitude lies in [1/2, 1], so a
  prefactor is at most 2^e.
* The source is the edge: with one pole per DLR frequency the lines carry K(t, +-beta w_l) with |beta w_l| up
  to Lambda, so G_b K(t, +-beta w_l) has exponents beyond the DLR basis and its coefficients
  K^-1 (G_b K) (the edge's vals2coefs, block_sparse_backbone.cpp:175-177) are up to 1e5-1e6 times larger
  than its values (cond K ~ 1 / eps).  A compressed hybridization (a few poles inside the band) removes it.

The thresholds below bracket the measured factors (two-orbital Kanamori, Lambda = 200, eps = 1e-12): they
pin that third-order Sigma amplifies a 1e-14 input change by more than 1e8 with the DLR poles, and by less
than 1e2 (atomic G0) with the compressed poles."""

import numpy as np
import pytest

from oracle import oracle as O
from xca_b200 import hyb_fit, models

BETA, LAM, EPS = 20.0, 200.0, 1e-12


@pytest.fixture(scope="module")
def setup():
    d = O.Dlr(LAM, EPS)
    m = models.kanamori_2orb(d.rf, d.it, BETA, LAM, EPS)
    dv = models.bethe_delta(BETA, d.it)
    delta = np.zeros((d.r, 4, 4))
    for i in range(4):
        delta[:, i, i] = dv
    cp, cc, _ = hyb_fit.compress_hybridization(d.rf, d.it, BETA, delta, 1e-10)
    return d, m, (m.hyb_poles, m.hyb_coeffs), (cp, cc)


def _amplification(d, m, poles, G, topo, nfix=120, rel=1e-14):
    p, c = poles
    ev = O.Evaluator(d, BETA, p, c, m.dims, m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks)
    t = np.array(topo, np.int32)
    nmax = ev.num_self_energy_backbones(t)
    fix = np.sort(np.random.default_rng(1).choice(nmax, min(nmax, nfix), replace=False))
    rng = np.random.default_rng(3)
    Gp = [g * (1 + rel * rng.uniform(-1, 1, g.shape)) for g in G]
    s1 = ev.compute_self_energy(G, t, f_ix=fix)
    s2 = ev.compute_self_energy(Gp, t, f_ix=fix)
    return max(np.max(np.abs(x - y)) for x, y in zip(s1, s2)) / max(np.max(np.abs(x)) for x in s1) / rel


def test_prefactor_divisors_bounded(setup):
    d, m, _, _ = setup
    # the divisor of a line is K(0, x) with x = -beta w (forward, w <= 0 / backward, w >= 0 in case 4(a)) or
    # x = +beta w (case 4(b)): x >= 0 in every case, and |K(0, x)| = 1 / (1 + exp(-x)) in [1/2, 1]
    for w in BETA * np.asarray(m.hyb_poles):
        for fwd in (True, False):
            case_a = (w <= 0) if fwd else (w >= 0)
            x = -w if case_a == fwd else w
            x = abs(x) if w == 0 else x
            assert x >= 0
            k0 = abs(float(models.kernel(0.0, x)))
            assert 0.5 <= k0 <= 1.0


def test_edge_coefficients_grow_with_the_pole(setup):
    d, m, _, _ = setup
    K = models.kernel(d.it[:, None], d.rf[None, :])
    g = models.seeded_G(m, 0)[4][:, 0, 0].real
    ratio = {}
    for l in (0, d.r // 2, d.r - 1):
        gk = g * models.kernel(d.it, d.rf[l])
        ratio[l] = np.max(np.abs(np.linalg.solve(K, gk))) / np.max(np.abs(gk))
    assert ratio[0] > 1e4 * ratio[d.r // 2] and ratio[d.r - 1] > 1e4 * ratio[d.r // 2]


@pytest.mark.parametrize("order_topo", [[[0, 2], [1, 3]], [[0, 3], [1, 4], [2, 5]]])
def test_amplification_dlr_vs_compressed_poles(setup, order_topo):
    d, m, dlr, comp = setup
    G = models.seeded_G(m, 0)
    a_dlr_seed = _amplification(d, m, dlr, G, order_topo)
    a_dlr_g0 = _amplification(d, m, dlr, m.G0, order_topo)
    a_cmp_seed = _amplification(d, m, comp, G, order_topo)
    a_cmp_g0 = _amplification(d, m, comp, m.G0, order_topo)
    print(f"{order_topo}: DLR poles seeded G {a_dlr_seed:.1e}, G0 {a_dlr_g0:.1e}; "
          f"{len(comp[0])} fitted poles seeded G {a_cmp_seed:.1e}, G0 {a_cmp_g0:.1e}")
    assert a_dlr_seed > 1e8 and a_dlr_g0 > 1e5
    assert a_cmp_g0 < 1e2 and a_cmp_seed < 1e6
    assert a_cmp_seed < 1e-3 * a_dlr_seed
