"""Pseudo-particle Dyson solver with the reference's Python name
(``python/triqs_xca/dlr_dyson_ppsc.cpp:10-20``: ``DysonItPPSC(beta, itops, g0)``, ``solve(sig, eta)``;
C++ ``cppdlr::dyson_it_ppsc``, ``c++/triqs_xca/dlr_dyson_ppsc.hpp:45-231``).

One object per Fock-space block, as the reference's solver builds them
(``python/triqs_xca/block_sparse_solver.py:136``).  The solve (coefficients, time-ordered convolution,
convolution matrix, LU with partial pivoting, substitution) runs on the GPU in ``libxca_b200.so``.
"""

import ctypes

import numpy as np

from . import _lib


class DysonItPPSC:
    def __init__(self, beta, itops, g0, device=0):
        g0 = np.asarray(g0)
        if g0.ndim != 3 or g0.shape[1] != g0.shape[2]:
            raise ValueError("g0 must have shape (r, d, d)")
        self.beta = float(beta)
        self.rf = np.ascontiguousarray(itops.get_rfnodes(), dtype=float)
        self.it = np.ascontiguousarray(itops.get_itnodes(), dtype=float)
        self.r = len(self.rf)
        if g0.shape[0] != self.r:
            raise ValueError(f"g0 has {g0.shape[0]} time nodes, the basis has rank {self.r}")
        self.d = g0.shape[1]
        lam = float(getattr(itops, "lambda")())
        L = _lib.lib()
        self._ctx = ctypes.c_void_p()
        _lib.check(L.xca_ctx_create(int(device), ctypes.byref(self._ctx)))
        dims = np.array([self.d], np.int32)
        _lib.check(L.xca_basis_setup(self._ctx, self.beta, lam, 0.0, self.r, _lib.as_dp(self.rf), _lib.as_dp(self.it), 1,
                                     _lib.as_ip(dims)))
        g0c = np.ascontiguousarray(g0, dtype=np.complex128)
        _lib.check(L.xca_dyson_setup(self._ctx, _lib.as_dp(g0c.view(np.float64))))
        self.g0 = g0c

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx and _lib._lib is not None:
            _lib._lib.xca_ctx_destroy(ctx)
            self._ctx = None

    def solve(self, sig, eta, hermitize=False):
        """G solving (1 - G0 * (Sigma + eta) *) G = G0 for this block (dlr_dyson_ppsc.hpp:135-168).  With
        ``hermitize`` the result is (G + G^T) / 2, the step solve_dyson adds (block_sparse_solver.py:582-586)."""
        s = np.ascontiguousarray(sig, dtype=np.complex128)
        if s.shape != self.g0.shape:
            raise ValueError(f"sig has shape {s.shape}, expected {self.g0.shape}")
        out = np.empty_like(s)
        _lib.check(_lib.lib().xca_dyson_solve(self._ctx, _lib.as_dp(s.view(np.float64)), float(eta), int(bool(hermitize)),
                                              _lib.as_dp(out.view(np.float64))))
        return out

    def solve_with_op(self, sig, eta, op, hermitize=False):
        """G solving (1 - G0 * (Sigma + eta + op) *) G = G0: the source term gains G0(t) op, as the reference's
        solve_with_op (dlr_dyson_ppsc.hpp:188-216) adds it (``op`` a d x d matrix)."""
        s = np.ascontiguousarray(sig, dtype=np.complex128)
        if s.shape != self.g0.shape:
            raise ValueError(f"sig has shape {s.shape}, expected {self.g0.shape}")
        o = np.ascontiguousarray(op, dtype=np.complex128)
        if o.shape != (self.d, self.d):
            raise ValueError(f"op has shape {o.shape}, expected {(self.d, self.d)}")
        out = np.empty_like(s)
        _lib.check(_lib.lib().xca_dyson_solve_with_op(self._ctx, _lib.as_dp(s.view(np.float64)), float(eta),
                                                      _lib.as_dp(o.view(np.float64)), int(bool(hermitize)),
                                                      _lib.as_dp(out.view(np.float64))))
        return out
