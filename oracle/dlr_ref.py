"""Oracle (test infrastructure only): numpy restatement of the DLR basis construction.

This module is part of the CPU oracle used by the tests, by ``__graft_entry__.smoke()`` and by
the ``cpu_baseline`` leg of ``bench.py``.  The product never imports it.

The reference calls the third-party library cppdlr (shipped with TRIQS 4.0.x, pinned only to the
4.0.x branch in ``jenkins/Jenkinsfile:9``; not present here) at these call sites:

* ``cppdlr::build_dlr_rf(Lambda, eps)``   ``hyb.cpp:158``, ``block_sparse.cpp:777``
* ``cppdlr::imtime_ops(Lambda, dlr_rf)``  ``block_sparse_backbone.cpp:69``, ``hyb.cpp:159``
* ``cppdlr::k_it(t, om)``                 ``hyb.cpp:98-103``

The restated published algorithm (Kaye, Chen, Parcollet, PRB 105, 235115 (2022); cppdlr JOSS paper):

1. A composite Chebyshev fine grid: in t in [0, 1/2] ``npt = max(ceil(log2 Lambda) - 2, 1)`` dyadic
   panels refined toward 0 with ``p = 24`` first-kind Chebyshev nodes each, mirrored to (1/2, 1]
   and stored in relative format (t < 0 stands for 1 + t); in omega in [-Lambda, Lambda]
   ``npo = max(ceil(log2 Lambda), 1)`` dyadic panels per sign, refined toward 0.
2. Pivoted, reorthogonalised Gram-Schmidt on the frequency columns of K(t, omega) selects the DLR
   frequencies; it stops when the largest residual column has RMS entry below ``eps``.  This rule
   reproduces the rank pinned by the reference test ``test_block_sparse_backbone_eval.cpp:47-50``
   (r = 36 at Lambda = 200, eps = 1e-10).
3. The same procedure on the rows of K(t_fine, omega_dlr) (run to full rank) selects the r
   imaginary-time nodes, returned in ascending absolute time.
"""

import numpy as np

CHEB_P = 24


def k_it(t, om):
    """Fermionic kernel K(t, om) in relative time format (``test/python/pycppdlr.py:29-43``).

    K(t, om) = exp(-t om) / (1 + exp(-om)) for om >= 0 and exp((1 - t) om) / (1 + exp(om)) for
    om < 0; a negative t stands for 1 + t and is evaluated as K(-t, -om) for full accuracy.
    """
    t = float(t)
    om = float(om)
    if t < 0:
        t, om = -t, -om
    if om >= 0:
        return np.exp(-t * om) / (1.0 + np.exp(-om))
    return np.exp((1.0 - t) * om) / (1.0 + np.exp(om))


def k_it_mat(t, om):
    t = np.asarray(t, dtype=float).ravel()
    om = np.asarray(om, dtype=float).ravel()
    out = np.empty((t.size, om.size))
    for i, ti in enumerate(t):
        for j, oj in enumerate(om):
            out[i, j] = k_it(ti, oj)
    return out


def rel2abs(t):
    t = np.asarray(t, dtype=float)
    return np.where(t < 0, 1.0 + t, t)


def _cheb_nodes(p):
    return -np.cos(np.pi * (np.arange(p) + 0.5) / p)


def fine_grids(lam, p=CHEB_P):
    nl = int(np.ceil(np.log(lam) / np.log(2.0)))
    npo = max(nl, 1)
    npt = max(nl - 2, 1)
    xc = _cheb_nodes(p)
    t = []
    for i in range(npt):
        a = 0.0 if i == 0 else 2.0 ** (-(npt - i + 1))
        b = 2.0 ** (-(npt - i))
        t.append(a + (b - a) * (xc + 1) / 2)
    t = np.concatenate(t)
    t = np.concatenate([t, -t[::-1]])
    om = []
    for i in range(npo):
        a = 0.0 if i == 0 else lam * 2.0 ** (-(npo - i))
        b = lam * 2.0 ** (-(npo - i - 1))
        om.append(a + (b - a) * (xc + 1) / 2)
    om = np.concatenate(om)
    om = np.concatenate([-om[::-1], om])
    return t, om


def pivoted_gram_schmidt(a, eps_rms):
    """Pivoted, twice-orthogonalised Gram-Schmidt on the rows of ``a``.

    Returns the pivot row indices in selection order; stops when the largest residual row has
    squared norm below ``eps_rms**2 * a.shape[1]`` (``eps_rms = 0`` runs to full rank).
    """
    a = np.array(a, dtype=float, copy=True)
    m, ncol = a.shape
    norms = np.einsum("ij,ij->i", a, a)
    piv = np.arange(m)
    thresh = eps_rms * eps_rms * ncol
    for j in range(min(m, ncol)):
        k = j + int(np.argmax(norms[j:]))
        if norms[k] <= thresh or norms[k] == 0.0:
            return piv[:j]
        a[[j, k]] = a[[k, j]]
        norms[[j, k]] = norms[[k, j]]
        piv[[j, k]] = piv[[k, j]]
        a[j] /= np.linalg.norm(a[j])
        for _ in range(2):
            a[j + 1:] -= np.outer(a[j + 1:] @ a[j], a[j])
        norms[j + 1:] = np.einsum("ij,ij->i", a[j + 1:], a[j + 1:])
    return piv[:min(m, ncol)]


def build_dlr_rf(lam, eps):
    """DLR real frequencies (dimensionless, ascending) for cutoff ``lam`` and accuracy ``eps``."""
    t, om = fine_grids(lam)
    kmat = k_it_mat(t, om)
    piv = pivoted_gram_schmidt(kmat.T, eps)
    return np.sort(om[piv])


def build_dlr_it(lam, rf):
    """DLR imaginary-time nodes (relative format, ascending absolute time) for frequencies ``rf``."""
    t, _ = fine_grids(lam)
    kmat = k_it_mat(t, rf)
    piv = pivoted_gram_schmidt(kmat, 0.0)
    if len(piv) != len(rf):
        raise RuntimeError("time-node selection lost rank")
    return t[np.sort(piv)]
