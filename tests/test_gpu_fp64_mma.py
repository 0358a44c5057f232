"""The FP64 tensor-core operation model the panel kernels rely on.

Their products (W gc, (beta K) Q, (beta K) P', the substitution's rectangular updates and the edge
tables' W fc) run as mma.sync m8n8k4 f64 tiles; the parity of every Sigma item with the CPU oracle
requires that one MMA computes each element as four correctly rounded fused multiply-adds in ascending
k, i.e. exactly the scalar chain of the restatement.  xca_fp64_mma_selftest compares both bit for bit
on random tiles (every fourth one with C cancelling A B).
"""

import ctypes

import pytest

from xca_b200 import _lib

pytestmark = pytest.mark.gpu


def _ctx():
    ctx = ctypes.c_void_p()
    _lib.check(_lib.lib().xca_ctx_create(0, ctypes.byref(ctx)))
    return ctx


@pytest.mark.parametrize("seed", [1, 2024])
def test_fp64_mma_is_the_ascending_fma_chain(seed):
    ctx = _ctx()
    try:
        bad = ctypes.c_long(-1)
        _lib.check(_lib.lib().xca_fp64_mma_selftest(ctx, 1 << 18, seed, ctypes.byref(bad)))
        assert bad.value == 0
    finally:
        _lib.lib().xca_ctx_destroy(ctx)


def test_fp64_mma_probe_reports_a_rate():
    ctx = _ctx()
    try:
        t = ctypes.c_double()
        _lib.check(_lib.lib().xca_fp64_mma_probe(ctx, ctypes.byref(t)))
        assert 1.0 < t.value < 500.0
    finally:
        _lib.lib().xca_ctx_destroy(ctx)
