"""The allocation-free Sigma entry point against the allocating one, through the C-ABI.

``xca_compute_self_energy_device_noalloc`` serves callers that may not allocate device memory while
they run (a process that works inside a device memory pool sized up front, or a host framework that
owns the device allocator): its scratch is a fixed 64 MiB array inside the library instead of
context-owned buffers.  Its results must equal those of ``xca_compute_self_energy_device`` on the same
inputs within the tolerance of the other Sigma parity tests (1e-12 relative per tau node, 1e-15
absolute floor; only the order of the atomic accumulation differs), on two calls in a row, the second
with another G and topology order so that it runs on the first call's leftover scratch.  Inputs whose
scratch would exceed the array are refused before any launch.

This file is collected last on purpose (``zz``), so that a stop-at-first-failure run has already run
every other test when it gets here.
"""

import ctypes

import numpy as np
import pytest

from xca_b200 import _lib, models

pytestmark = pytest.mark.gpu

REL = 1e-12
ABS = 1e-15


def _node_rel_err(A, B):
    r = A[0].shape[0]
    worst = 0.0
    for t in range(r):
        num = max(np.max(np.abs(a[t] - b[t])) for a, b in zip(A, B))
        den = max(np.max(np.abs(b[t])) for b in B)
        worst = max(worst, num / (REL * den + ABS))
    return worst


def _evaluator(beta, lam, eps):
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    from xca_b200.pycppdlr import ImTimeOps, build_dlr_rf
    rf = build_dlr_rf(lam, eps)
    it = ImTimeOps(lam, rf).get_itnodes()
    m = models.kanamori_2orb(rf, it, beta, lam, eps)
    Fq = BlockOpSymQuartet(m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks, m.dims)
    return m, DiagramEvaluator.from_arrays(beta, lam, eps, rf, it, m.hyb_poles, m.hyb_coeffs, Fq)


def _allocations():
    out = ctypes.c_long()
    _lib.check(_lib.lib().xca_device_allocations(ctypes.byref(out)))
    return out.value


def _run(ev, fn, G_dev, S_dev, topo, scale):
    t = np.ascontiguousarray(np.asarray(topo, np.int32).reshape(-1, 2))
    ev.zero_device(S_dev, ev.slab)
    _lib.check(getattr(_lib.lib(), fn)(ev._ctx, ctypes.c_void_p(G_dev), t.shape[0], _lib.as_ip(t), float(scale),
                                       ctypes.c_void_p(S_dev)))
    return [x.astype(np.complex128) for x in ev.unpack(ev.to_host(S_dev, ev.slab))]


def test_noalloc_matches_device_entry_on_two_calls():
    m, ev = _evaluator(4.0, 40.0, 1e-8)
    G_dev = ev.device_buffer(0, ev.slab)
    S_dev = ev.device_buffer(1, ev.slab)
    calls = [(models.seeded_G(m, 5), [[0, 2], [1, 3]], -1.0),
             (models.seeded_G(m, 6), [[0, 3], [1, 4], [2, 5]], 0.5)]
    for G, topo, scale in calls:
        ev.to_device(G_dev, ev.pack(G).real)
        ref = _run(ev, "xca_compute_self_energy_device", G_dev, S_dev, topo, scale)
        before = _allocations()
        got = _run(ev, "xca_compute_self_energy_device_noalloc", G_dev, S_dev, topo, scale)
        assert _allocations() == before  # the call itself allocated no device memory
        assert max(np.max(np.abs(b)) for b in ref) > 0.0
        assert _node_rel_err(got, ref) <= 1.0, topo


def test_noalloc_full_size_second_order_and_refusal():
    # the 2-orbital Kanamori model on its full basis (beta = 20, Lambda = 200, eps = 1e-12): OCA fits in the
    # fixed scratch, TCA (edge tables ~ 1 + 2p + 4p^2 signatures) does not and is refused
    m, ev = _evaluator(20.0, 200.0, 1e-12)
    G_dev = ev.device_buffer(0, ev.slab)
    S_dev = ev.device_buffer(1, ev.slab)
    ev.to_device(G_dev, ev.pack(models.seeded_G(m, 0)).real)
    topo = [[0, 2], [1, 3]]
    ref = _run(ev, "xca_compute_self_energy_device", G_dev, S_dev, topo, 1.0)
    got = _run(ev, "xca_compute_self_energy_device_noalloc", G_dev, S_dev, topo, 1.0)
    assert _node_rel_err(got, ref) <= 1.0
    with pytest.raises(ValueError, match="scratch"):
        _run(ev, "xca_compute_self_energy_device_noalloc", G_dev, S_dev, [[0, 3], [1, 4], [2, 5]], 1.0)
