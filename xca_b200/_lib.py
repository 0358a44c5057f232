"""ctypes binding of ``libxca_b200.so`` (the C-ABI declared in ``include/xca_b200.h``).

The library is built in-tree (``python -c "import __graft_entry__ as g; g.build()"``).  Every compute
entry point runs on the GPU; there is no CPU fallback, and a missing library or device raises.
"""

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libxca_b200.so")

XCA_OK = 0
XCA_ERR_INVALID = 1
XCA_ERR_RUNTIME = 2
XCA_ERR_CUDA = 3
XCA_ERR_UNSUPPORTED = 4

# precision / summation modes (xca_set_precision_mode)
XCA_PREC_FP64 = 0
XCA_PREC_FP64_ORDERED = 1
XCA_PREC_FP32 = 2
XCA_ORDERED_UNIT_TUPLES = 64
PRECISION_MODES = {"fp64": XCA_PREC_FP64, "fp64_ordered": XCA_PREC_FP64_ORDERED, "fp32": XCA_PREC_FP32}

# launch-shape parameters (xca_set_tuning)
TUNING = {"unit_batches": 0, "wide_unit_tuples": 1, "wide_ctas_per_sm": 2, "dyson_blocked_min_n": 3}

_lib = None

D = ctypes.c_double
I = ctypes.c_int
L = ctypes.c_long
P = ctypes.c_void_p
dp = ctypes.POINTER(ctypes.c_double)
ip = ctypes.POINTER(ctypes.c_int)
lp = ctypes.POINTER(ctypes.c_long)
dpp = ctypes.POINTER(ctypes.POINTER(ctypes.c_double))

# name -> argtypes (all return int status unless listed in _RESTYPES)
SIGNATURES = {
    "xca_last_error": [],
    "xca_abi_version": [],
    "xca_dlr_build_rf": [D, D, dp, I, ip],
    "xca_dlr_build_it": [D, dp, I, dp],
    "xca_ctx_create": [I, ctypes.POINTER(P)],
    "xca_ctx_destroy": [P],
    "xca_evaluator_setup": [P, D, D, D, I, dp, dp, I, dp, dp, I, lp, I, ip, ip, dp, ip, dp],
    "xca_basis_setup": [P, D, D, D, I, dp, dp, I, ip],
    "xca_dyson_setup": [P, dp],
    "xca_dyson_solve": [P, dp, D, I, dp],
    "xca_dyson_solve_with_op": [P, dp, D, dp, I, dp],
    "xca_dyson_solve_device": [P, P, D, I, P],
    "xca_trace": [P, dp, dp],
    "xca_trace_device": [P, P, dp],
    "xca_normalize_device": [P, P, dp, dp],
    "xca_max_abs_diff_device": [P, P, P, dp],
    "xca_axpby_device": [P, D, P, D, P],
    "xca_num_self_energy_backbones": [P, I, ip, lp],
    "xca_num_single_ptcle_gf_backbones": [P, I, ip, lp],
    "xca_compute_self_energy": [P, dp, I, ip, lp, L, dp],
    "xca_compute_self_energy_device": [P, P, I, ip, D, P],
    "xca_compute_self_energy_device_shard": [P, P, I, ip, D, P, I, I],
    "xca_compute_self_energy_device_batch": [I, ctypes.POINTER(P), ctypes.POINTER(P), ip, ip, dp, ctypes.POINTER(P)],
    "xca_compute_self_energy_device_noalloc": [P, P, I, ip, D, P],
    "xca_compute_single_ptcle_gf": [P, dp, I, ip, lp, L, dp],
    "xca_compute_single_ptcle_gf_device": [P, P, I, ip, D, P],
    "xca_zero_device": [P, P, L],
    "xca_self_energy_items": [P, dp, I, ip, lp, L, lp],
    "xca_self_energy_flops": [P, dp, I, ip, dp, lp],
    "xca_profile": [P, I, dp, lp],
    "xca_event_record": [P, I],
    "xca_event_elapsed": [P, I, I, dp],
    "xca_flush_l2": [P, L],
    "xca_fp64_fma_probe": [P, dp],
    "xca_fp64_mma_probe": [P, dp],
    "xca_fp64_mma_selftest": [P, L, ctypes.c_ulonglong, lp],
    "xca_slab_info": [P, lp, ip],
    "xca_device_buffer": [P, I, L, dpp],
    "xca_copy_to_device": [P, P, dp, L],
    "xca_copy_to_host": [P, dp, P, L],
    "xca_synchronize": [P],
    "xca_kernel_launches": [P, lp],
    "xca_device_allocations": [lp],
    "xca_set_precision_mode": [P, I],
    "xca_set_tuning": [P, I, I],
    "xca_get_tuning": [P, I, ip],
    "xca_compute_one_time_correlator": [P, dp, I, ip, dp, I, ip, dp, I, ip, lp, L, dp],
    "xca_convolve_ppsc": [P, dp, dp, dp],
    "xca_convolve_ppsc_device": [P, P, P, P],
    "xca_expectation_value": [P, dp, ip, dp, dp],
    "xca_get_precision_mode": [P, ip],
}
_RESTYPES = {"xca_last_error": ctypes.c_char_p}


class XcaError(RuntimeError):
    pass


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libxca_b200.so is not built ({LIB_PATH}); run __graft_entry__.build()")
        h = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(h, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, ctypes.c_int)
        _lib = h
    return _lib


def check(rc):
    """Raise the reference's exception type for a failing status (ValueError ~ std::invalid_argument)."""
    if rc == XCA_OK:
        return
    msg = lib().xca_last_error().decode()
    if rc == XCA_ERR_INVALID:
        raise ValueError(msg)
    if rc == XCA_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise XcaError(msg)


def as_dp(a):
    return a.ctypes.data_as(dp)


def as_ip(a):
    return a.ctypes.data_as(ip)


def as_lp(a):
    return a.ctypes.data_as(lp)
