"""DLR basis construction: Python names of the reference's cppdlr binding
(``python/triqs_xca/pycppdlr.wrap.cxx``: ``build_dlr_rf`` :210-214, ``ImTimeOps`` :29-202).

The node selection runs in the C++ library (host set-up, once per (Lambda, eps)).  The mesh class
``MeshDLRImTime`` stands in for ``triqs.gfs.MeshDLRImTime`` as the evaluator's ``tau_mesh`` argument.
"""

import ctypes
import functools

import numpy as np

from . import _lib
from .models import kernel, rel2abs


@functools.lru_cache(maxsize=64)
def _dlr_rf_cached(lam, eps):
    L = _lib.lib()
    buf = np.zeros(4096)
    r = ctypes.c_int(0)
    _lib.check(L.xca_dlr_build_rf(lam, eps, _lib.as_dp(buf), len(buf), ctypes.byref(r)))
    out = buf[: r.value].copy()
    out.setflags(write=False)
    return out


def build_dlr_rf(lam, eps):
    """DLR real frequencies for cutoff ``lam`` = beta * w_max and accuracy ``eps`` (ascending).  The node
    selection is computed once per (lam, eps) in a process (a served stream repeats them)."""
    return _dlr_rf_cached(float(lam), float(eps)).copy()


@functools.lru_cache(maxsize=64)
def _dlr_it_cached(lam, rf_bytes):
    rf = np.frombuffer(rf_bytes, dtype=float).copy()
    it = np.zeros(len(rf))
    _lib.check(_lib.lib().xca_dlr_build_it(lam, _lib.as_dp(rf), len(rf), _lib.as_dp(it)))
    it.setflags(write=False)
    return it


class ImTimeOps:
    """``cppdlr::imtime_ops(lambda, dlr_rf)``: the DLR imaginary-time nodes of a frequency set.

    Holds the nodes and the matrix K(t_i, om_l); the device-side transforms of the hot path use
    the same LU factorisation, built inside the C++ library."""

    def __init__(self, lam, dlr_rf, symmetrize=False):
        if symmetrize:
            raise NotImplementedError("symmetrized DLR nodes are not supported")
        self._lam = float(lam)
        self.rf = np.ascontiguousarray(dlr_rf, dtype=float)
        self.it = _dlr_it_cached(self._lam, self.rf.tobytes()).copy()

    def rank(self):
        return len(self.rf)

    def get_rfnodes(self):
        return self.rf.copy()

    def get_itnodes(self):
        return self.it.copy()

    def get_cf2it(self):
        return kernel(self.it[:, None], self.rf[None, :])

    def __getattr__(self, name):
        if name == "lambda":
            return lambda: self._lam
        raise AttributeError(name)


class MeshDLRImTime:
    """DLR imaginary-time mesh (stand-in for ``triqs.gfs.MeshDLRImTime``): ``beta``, ``w_max``, ``eps``;
    iterating yields the absolute times tau_i = beta * t_i."""

    def __init__(self, beta, statistic="Fermion", w_max=None, eps=None, symmetrize=False):
        if statistic not in ("Fermion", "f", "F"):
            raise NotImplementedError("only fermionic meshes are supported")
        self.beta = float(beta)
        self.w_max = float(w_max)
        self.eps = float(eps)
        self.lam = self.beta * self.w_max
        self.dlr_rf = build_dlr_rf(self.lam, self.eps)
        self.dlr_it = ImTimeOps(self.lam, self.dlr_rf, symmetrize)
        self.dlr_freq = self.dlr_rf

    def __len__(self):
        return len(self.dlr_rf)

    def __iter__(self):
        return iter(self.beta * rel2abs(self.dlr_it.it))

    @property
    def tau(self):
        return self.beta * rel2abs(self.dlr_it.it)
