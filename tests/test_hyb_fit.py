"""Hybridization pole compression (the compression=True branch of fit_hybridization,
python/triqs_xca/block_sparse_solver.py:146-185, adapol in the reference): host-side, no GPU.

adapol is not available here, so parity is against the functions' own definitions: the three-orbital
t2g hybridization is built from 8 bath poles and must come back as those 8 poles with the fit error below
the tolerance; the Bethe hybridization needs far fewer poles than the DLR rank."""

import numpy as np
import pytest

from oracle import dlr_ref
from xca_b200 import hyb_fit, models


def _basis(lam, eps):
    rf = dlr_ref.build_dlr_rf(lam, eps)
    return rf, dlr_ref.build_dlr_it(lam, rf)


def test_t2g_recovers_its_bath_poles():
    beta, lam, eps = 50.0, 500.0, 1e-10
    rf, it = _basis(lam, eps)
    m = models.t2g_3orb(rf, it, beta, lam, eps)
    delta = (models.kernel(it[:, None], rf[None, :]) @ m.hyb_coeffs.reshape(len(rf), -1)).reshape(len(it), 6, 6)
    poles, coeffs, err = hyb_fit.compress_hybridization(rf, it, beta, delta, 1e-9)
    assert err < 1e-9
    assert len(poles) == 8
    assert np.max(np.abs(np.sort(poles) - np.sort(m.extra["bath_w"]))) < 1e-5  # two bath poles lie 7e-3 apart
    rec = np.einsum("tk,kab->tab", models.kernel(it[:, None], beta * poles[None, :]), coeffs)
    assert np.max(np.abs(rec - delta)) < 1e-9 * 36


@pytest.mark.parametrize("tol", [1e-6, 1e-8])
def test_bethe_compression(tol):
    beta, lam, eps = 20.0, 200.0, 1e-12
    rf, it = _basis(lam, eps)
    dv = models.bethe_delta(beta, it)
    delta = np.zeros((len(it), 2, 2))
    delta[:, 0, 0] = dv
    delta[:, 1, 1] = dv
    poles, coeffs, err = hyb_fit.compress_hybridization(rf, it, beta, delta, tol)
    assert err < tol
    assert len(poles) < len(rf) // 2
    # the fit stays inside the band: |w| <= half-bandwidth 2
    assert np.max(np.abs(poles)) < 2.0 + 1e-6
    # off-diagonal residues stay zero (spin-diagonal input)
    assert np.max(np.abs(coeffs[:, 0, 1])) < 1e-12


def test_fit_cache_returns_the_same_fit():
    # served solves that share a bath share its fit: the cached call returns exactly the uncached result,
    # as fresh arrays, and a changed input (another tolerance, another Delta) is fitted anew
    beta, lam, eps = 10.0, 100.0, 1e-10
    rf, it = _basis(lam, eps)
    dv = models.bethe_delta(beta, it)
    delta = np.zeros((len(it), 2, 2))
    delta[:, 0, 0] = dv
    delta[:, 1, 1] = dv
    ref = hyb_fit.compress_hybridization(rf, it, beta, delta, 1e-9)
    a = hyb_fit.compress_hybridization_cached(rf, it, beta, delta, 1e-9)
    b = hyb_fit.compress_hybridization_cached(rf, it, beta, delta, 1e-9)
    for x in (a, b):
        assert np.array_equal(x[0], ref[0]) and np.array_equal(x[1], ref[1]) and x[2] == ref[2]
    a[0][0] += 1.0  # the caller's copy, not the cache's
    assert np.array_equal(hyb_fit.compress_hybridization_cached(rf, it, beta, delta, 1e-9)[0], ref[0])
    c = hyb_fit.compress_hybridization_cached(rf, it, beta, 0.5 * delta, 1e-9)
    assert not np.array_equal(c[1], ref[1])
