"""The five-orbital d shell (10 spin-orbitals restricted to N = 4..6: 672 states in 16 (N_up, N_dn) blocks of
dimension up to 100, Slater-Condon F0 = 4, J = 0.7, F4 / F2 = 0.625, beta = 20, Lambda = 200, eps = 1e-8,
diagonal Bethe hybridization): block chains too wide for a shared-memory panel run on the wide-chain kernel.

Parity against golden values of the oracle on seeded random flat-index subsets
(``tests/golden/make_sigma_golden.py dshell_subsets``; the CPU restatement needs hours for every flat index):
bit for bit in the ordered mode, 1e-12 relative per tau node in the fast mode."""

import os
import time

import numpy as np
import pytest

from oracle import oracle as O
from xca_b200 import models

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sigma_dshell_subsets_ordered.npz")


def _setup():
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    if not os.path.exists(GOLDEN):
        pytest.skip("golden file not generated")
    fx = np.load(GOLDEN)
    beta, lam, eps = float(fx["beta"]), float(fx["lam"]), float(fx["eps"])
    m = models.dshell_5orb(fx["rf"], fx["it"], beta, lam, eps)
    assert np.array_equal(m.dims, fx["dims"]) and max(m.dims) == 100
    Fq = BlockOpSymQuartet(m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks, m.dims)
    ev = DiagramEvaluator.from_arrays(beta, lam, eps, fx["rf"], fx["it"], m.hyb_poles, m.hyb_coeffs, Fq)
    return fx, m, ev, ev.unpack(fx["G"].astype(np.complex128))


def _per_node_rel(ev, a, b):
    r = ev.r
    num, den, off = np.zeros(r), np.zeros(r), 0
    for d in ev.dims:
        sz = r * d * d
        num = np.maximum(num, np.max(np.abs(a[off:off + sz] - b[off:off + sz]).reshape(r, -1), axis=1))
        den = np.maximum(den, np.max(np.abs(b[off:off + sz]).reshape(r, -1), axis=1))
        off += sz
    return float(np.max(num / np.maximum(den, 1e-300)))


@pytest.mark.parametrize("mode", ["fp64_ordered", "fp64"])
def test_dshell_sigma_subsets_vs_oracle(mode):
    fx, m, ev, G = _setup()
    ev.precision_mode = mode
    for k in range(int(fx["n_topologies"])):
        topo, gold, fix = fx[f"topo_{k}"], fx[f"sigma_{k}"], fx[f"fix_{k}"]
        got = np.concatenate([s.real.ravel() for s in ev.compute_self_energy(G, topo, f_ix=fix)])
        assert np.max(np.abs(gold)) > 0
        if mode == "fp64_ordered":
            assert np.array_equal(got, gold), (topo.tolist(), float(np.max(np.abs(got - gold))))
        else:
            rel = _per_node_rel(ev, got, gold)
            print(f"d shell {topo.tolist()} ({len(fix)} flat indices): fast mode per-node error {rel:.2e}")
            assert rel <= 1e-12


def test_dshell_full_oca_both_modes():
    # every flat index of the second-order topology through the device-resident path, fast vs ordered mode
    fx, m, ev, G = _setup()
    topo = [[0, 2], [1, 3]]
    bg = ev.device_buffer(30, ev.slab)
    bs = ev.device_buffer(31, ev.slab)
    ev.to_device(bg, ev.pack(G).real)
    res = {}
    for mode in ("fp64", "fp64_ordered"):
        ev.precision_mode = mode
        ev.zero_device(bs, ev.slab)
        ev.compute_self_energy_device(bg, topo, 1.0, bs)  # warm-up (work list, edge tables)
        ev.zero_device(bs, ev.slab)
        ev.synchronize()
        t0 = time.perf_counter()
        ev.compute_self_energy_device(bg, topo, 1.0, bs)
        ev.synchronize()
        res[mode] = (ev.to_host(bs, ev.slab), time.perf_counter() - t0)
    fl, items = ev.self_energy_flops(G, topo)
    rel = _per_node_rel(ev, res["fp64"][0], res["fp64_ordered"][0])
    print(f"d shell OCA, all {items} items: fast {res['fp64'][1] * 1e3:.1f} ms ({fl / res['fp64'][1] / 1e12:.2f} TFLOP/s), "
          f"ordered {res['fp64_ordered'][1] * 1e3:.1f} ms; modes differ by {rel:.2e} per node")
    assert rel <= 1e-12


@pytest.mark.parametrize("block", [1, 6])
def test_dshell_blocked_dyson_vs_oracle(block):
    # systems of dimension r d = 31 x 50 and 31 x 25 (> 512: the blocked LU) against the oracle's getrf / getrs
    from xca_b200.dlr_dyson_ppsc import DysonItPPSC
    from xca_b200.pycppdlr import ImTimeOps, build_dlr_rf
    beta, lam, eps = 20.0, 200.0, 1e-8
    itops = ImTimeOps(lam, build_dlr_rf(lam, eps))
    d = O.Dlr(lam, eps, rf=itops.get_rfnodes(), it=itops.get_itnodes())
    m = models.dshell_5orb(d.rf, d.it, beta, lam, eps)
    g0 = m.G0[block]
    assert g0.shape[1] * d.r > 512
    sig = 0.2 * models.seeded_G(m, 9)[block]
    for eta in (0.0, 0.3):
        t0 = time.perf_counter()
        dev = DysonItPPSC(beta, itops, g0).solve(sig, eta)
        t1 = time.perf_counter()
        ref = d.dyson_solve(beta, g0, sig, eta)
        rel = float(np.max(np.abs(dev - ref)) / np.max(np.abs(ref)))
        print(f"Dyson d = {g0.shape[1]} (N = {g0.shape[1] * d.r}), eta = {eta}: {rel:.2e}, device {1e3 * (t1 - t0):.1f} ms")
        assert rel <= 1e-12
