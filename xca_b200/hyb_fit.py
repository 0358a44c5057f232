"""Hybridization pole compression: a matrix-valued Delta(tau) on the DLR nodes represented by a few real poles,
Delta(tau) = sum_k K(tau / beta, beta w_k) W_k, in place of one pole per DLR frequency.

This is the ``compression=True`` branch of ``BlockSparseSolver.fit_hybridization``
(``python/triqs_xca/block_sparse_solver.py:146-185``), which calls the third-party adapol package (0.2.x,
``deps/CMakeLists.txt:60-66``; an older copy is vendored in ``python/triqs_xca/adapol_depr/``).  Restated here
from the published method it implements: the AAA rational approximation (Nakatsukasa, Sete, Trefethen, SIAM
J. Sci. Comput. 40, A1494 (2018)) of the matrix-valued function on the imaginary frequency axis with support
points in conjugate pairs (so the poles come out real), least-squares residues in imaginary time, removal of
negligible poles and a gradient refinement of the pole positions; the number of AAA terms grows until the
imaginary-time error is below the tolerance (``adapol_depr/fit_utils_xca.py:190-240``).  Host-side set-up,
run once per solve like the reference's.
"""

import hashlib
import threading
from collections import OrderedDict

import numpy as np
import scipy.linalg
import scipy.optimize

from .models import kernel


def _matsubara_points(lam, n_points=160):
    """Positive fermionic Matsubara frequencies nu_n = (2n + 1) pi (dimensionless, units of 1 / beta), n on a
    logarithmic grid up to about the cutoff Lambda."""
    nmax = max(int(lam), 8)
    n = np.unique(np.round(np.logspace(0, np.log10(nmax), n_points)).astype(int) - 1)
    return (2 * n + 1) * np.pi


def delta_iw(rf, coeffs, nu):
    """Delta(i nu) = sum_l c_l / (i nu - om_l) of a DLR expansion (the Matsubara image of the signed kernel)."""
    return np.einsum("nl,lab->nab", 1.0 / (1j * nu[:, None] - rf[None, :]), coeffs)


def aaa_matrix_real(F, nu, tol=1e-14, mmax=60):
    """AAA on matrix-valued samples F (n, a, b) at z = i nu (nu > 0), the points taken with their conjugates
    z* = -i nu (F(z*) = F(z)^dag), support points added in conjugate pairs with real-pair weights so that
    the rational approximant is real on the real axis.  Returns the poles of the approximant."""
    Z = np.concatenate([1j * nu, -1j * nu])
    Fh = np.conj(np.transpose(F, (0, 2, 1)))
    Fm = np.concatenate([F, Fh]).reshape(2 * len(nu), -1)
    N, nh = len(Z), len(nu)
    free = list(range(N))
    zs, fs = [], []
    fit = np.full_like(Fm, Fm.mean())
    weight = None
    for n in range(2, mmax + 1, 2):
        j = int(np.argmax(np.sum(np.abs(Fm - fit) ** 2, axis=1)))
        j2 = (j + nh) % N
        for jj in (j, j2):
            zs.append(Z[jj])
            fs.append(Fm[jj])
            free.remove(jj)
        zv, fv = np.array(zs), np.array(fs)
        C = 1.0 / (Z[free, None] - zv[None, :])
        # Loewner matrix over every matrix entry, then the real parametrisation of conjugate weight pairs
        A = np.concatenate([(Fm[free, e][:, None] - fv[None, :, e]) * C for e in range(Fm.shape[1])], axis=0)
        Al, Ar = A[:, 0::2], A[:, 1::2]
        Ar2 = np.concatenate([Al + Ar, 1j * (Al - Ar)], axis=1)
        Ar2 = np.concatenate([Ar2.real, Ar2.imag], axis=0)
        _, _, Vh = scipy.linalg.svd(Ar2, full_matrices=False)
        wr = Vh[-1].reshape(2, n // 2)
        weight = np.stack([wr[0] + 1j * wr[1], wr[0] - 1j * wr[1]], axis=1).ravel()
        fit = Fm.copy()
        den = C @ weight
        fit[free] = (C @ (weight[:, None] * fv)) / den[:, None]
        if np.max(np.abs(fit - Fm)) <= tol:
            break
    # poles: the finite eigenvalues of the arrowhead pencil of the barycentric denominator
    m = len(weight)
    E = np.zeros((m + 1, m + 1), np.complex128)
    Bm = np.eye(m + 1, dtype=np.complex128)
    Bm[0, 0] = 0.0
    E[0, 1:] = weight
    E[1:, 0] = 1.0
    E[np.arange(1, m + 1), np.arange(1, m + 1)] = zs
    ev = scipy.linalg.eigvals(E, Bm)
    return ev[np.isfinite(ev)]


def residues_tau(poles, it, delta):
    """Least-squares residues W_k of Delta(t_i) = sum_k K(t_i, p_k) W_k (dimensionless poles p_k = beta w_k)."""
    K = kernel(np.asarray(it)[:, None], np.asarray(poles)[None, :])
    W, *_ = np.linalg.lstsq(K, delta.reshape(len(it), -1), rcond=None)
    return W.reshape(len(poles), *delta.shape[1:])


def tau_error(poles, it, delta):
    """RMS over the nodes of the residual of the least-squares fit with these poles, per nonzero entry."""
    W = residues_tau(poles, it, delta)
    K = kernel(np.asarray(it)[:, None], np.asarray(poles)[None, :])
    res = K @ W.reshape(len(poles), -1) - delta.reshape(len(it), -1)
    nz = max(int(np.sum(np.max(np.abs(delta), axis=0) > 1e-12)), 1)
    return float(np.linalg.norm(res) / np.sqrt(len(it)) / nz)


def compress_hybridization(rf, it, beta, delta_tau, tol, max_poles=50):
    """Few-pole representation of Delta (r, n, n) on the DLR nodes (relative times it, DLR frequencies rf).

    Returns (poles, coeffs, error): physical poles w_k (the evaluator multiplies by beta), coefficients
    (p, n, n) with Delta(tau) = sum_k K(tau / beta, beta w_k) coeffs_k, and the imaginary-time fit error."""
    delta = np.asarray(delta_tau, dtype=np.complex128)
    if np.max(np.abs(delta.imag)) == 0.0:
        delta = delta.real
    r = len(it)
    K = kernel(np.asarray(it)[:, None], np.asarray(rf)[None, :])
    coeffs = np.linalg.solve(K, delta.reshape(r, -1)).reshape(delta.shape)
    lam = float(np.max(np.abs(rf)))
    nu = _matsubara_points(lam)
    F = delta_iw(np.asarray(rf), coeffs, nu)
    scale = max(np.max(np.abs(delta)), 1e-300)
    best = None
    for mmax in range(4, max_poles, 2):
        pol = aaa_matrix_real(F, nu, tol=1e-14 * np.max(np.abs(F)), mmax=mmax)
        pol = pol[np.abs(pol.imag) < 1e-3 * max(1.0, np.max(np.abs(pol.real), initial=1.0))].real
        if len(pol) == 0:
            continue
        W = residues_tau(pol, it, delta)
        keep = np.array([np.linalg.norm(w) > tol * scale for w in W])
        pol = pol[keep]
        if len(pol) == 0:
            continue
        res = scipy.optimize.minimize(lambda x: tau_error(x, it, delta), pol, method="L-BFGS-B",
                                      options=dict(gtol=1e-14, ftol=1e-14, maxiter=200))
        x = res.x if res.fun <= tau_error(pol, it, delta) else pol
        err = tau_error(x, it, delta)
        if best is None or err < best[2]:
            best = (x, residues_tau(x, it, delta), err)
        if err < tol:
            break
    if best is None:
        raise ValueError("hybridization compression found no real poles")
    x, W, err = best
    order = np.argsort(x)
    return x[order] / beta, np.asarray(W[order], dtype=np.complex128), err


_FITS = OrderedDict()
_FITS_LOCK = threading.Lock()
FIT_CACHE_SIZE = 64


def compress_hybridization_cached(rf, it, beta, delta_tau, tol, max_poles=50):
    """compress_hybridization, its result kept per exact input (DLR nodes, beta, the values of Delta, tol,
    max_poles; at most FIT_CACHE_SIZE fits, least recently used dropped): the fit is a deterministic function
    of these, so solves that share a bath -- the requests of a served stream at one beta -- share it."""
    h = hashlib.sha1()
    for a in (rf, it, delta_tau):
        h.update(np.ascontiguousarray(a).tobytes())
    h.update(np.array([beta, tol, max_poles], np.float64).tobytes())
    key = h.hexdigest()
    with _FITS_LOCK:
        hit = _FITS.get(key)
        if hit is not None:
            _FITS.move_to_end(key)
    if hit is None:
        hit = compress_hybridization(rf, it, beta, delta_tau, tol, max_poles)
        with _FITS_LOCK:
            _FITS[key] = hit
            while len(_FITS) > FIT_CACHE_SIZE:
                _FITS.popitem(last=False)
    poles, coeffs, err = hit
    return poles.copy(), coeffs.copy(), err
