"""CPU-side checks of the C-ABI library: it loads, exports every symbol the header declares, its
host-side DLR construction matches the oracle's, and device calls fail loudly without a GPU."""

import os
import re

import numpy as np
import pytest

from oracle import dlr_ref
from xca_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "xca_b200.h")).read()
    return sorted(set(re.findall(r"\b(xca_[a-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported():
    L = _lib.lib()
    names = _declared()
    assert len(names) >= 15
    for name in names:
        assert hasattr(L, name), name
        assert name in _lib.SIGNATURES, name


def test_abi_version():
    assert _lib.lib().xca_abi_version() == 1


@pytest.mark.parametrize("lam,eps", [(200.0, 1e-10), (100.0, 1e-10), (200.0, 1e-12), (500.0, 1e-10), (40.0, 1e-8)])
def test_dlr_nodes_match_oracle(lam, eps):
    from xca_b200.pycppdlr import ImTimeOps, build_dlr_rf
    rf = build_dlr_rf(lam, eps)
    rf_o = dlr_ref.build_dlr_rf(lam, eps)
    assert rf.shape == rf_o.shape
    assert np.max(np.abs(rf - rf_o)) <= 1e-12 * lam
    it = ImTimeOps(lam, rf).get_itnodes()
    it_o = dlr_ref.build_dlr_it(lam, rf_o)
    assert np.max(np.abs(it - it_o)) < 1e-14


def test_dlr_rank_pin_product():
    from xca_b200.pycppdlr import build_dlr_rf
    assert len(build_dlr_rf(200.0, 1e-10)) == 36


def test_invalid_lambda_raises():
    from xca_b200.pycppdlr import build_dlr_rf
    with pytest.raises(ValueError):
        build_dlr_rf(-1.0, 1e-10)


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import ctypes
    ctx = ctypes.c_void_p()
    rc = _lib.lib().xca_ctx_create(0, ctypes.byref(ctx))
    assert rc == _lib.XCA_ERR_CUDA
    assert "CUDA" in _lib.lib().xca_last_error().decode() or "device" in _lib.lib().xca_last_error().decode()
