"""GPU parity of the single-particle Green's function backbones (compute_single_ptcle_gf) against the
CPU oracle, through the C-ABI.

Tolerance as for Sigma: per tau node, max_{mu, ka} |g_gpu - g_oracle| <= 1e-12 * max_{mu, ka} |g_oracle(tau)|
+ 1e-15.  Every flat index's contribution is evaluated in the oracle's operation order; only the order in
which contributions are summed differs.
"""

import numpy as np
import pytest

from oracle import oracle as O
from xca_b200 import models

pytestmark = pytest.mark.gpu

REL = 1e-12
ABS = 1e-15

TOPOS = [[[0, 1]], [[0, 2], [1, 3]], [[0, 2], [1, 4], [3, 5]], [[0, 3], [1, 4], [2, 5]], [[0, 3], [1, 5], [2, 4]],
         [[0, 4], [1, 3], [2, 5]]]


def _node_rel_err(a, b):
    worst = 0.0
    for t in range(a.shape[0]):
        num = np.max(np.abs(a[t] - b[t]))
        den = np.max(np.abs(b[t]))
        worst = max(worst, num / (REL * den + ABS))
    return worst


def _pair(model, dlr):
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    Fq = BlockOpSymQuartet(model.labels, model.F_index, model.F_blocks, model.Fd_index, model.Fd_blocks, model.dims)
    dev = DiagramEvaluator.from_arrays(model.beta, model.lam, model.eps, dlr.rf, dlr.it, model.hyb_poles, model.hyb_coeffs, Fq)
    ora = O.Evaluator(dlr, model.beta, model.hyb_poles, model.hyb_coeffs, model.dims, model.labels, model.F_index,
                      model.F_blocks, model.Fd_index, model.Fd_blocks)
    return dev, ora


@pytest.mark.parametrize("pole", [0.0, 0.8, -1.3])
def test_one_fermion_all_topologies(pole):
    beta, lam, eps = 2.0, 40.0, 1e-10
    d = O.Dlr(lam, eps)
    m = models.one_fermion(d.rf, d.it, beta, lam, eps, hyb_pole=pole)
    dev, ora = _pair(m, d)
    nonzero = 0
    for topo in TOPOS:
        assert dev.get_num_single_ptcle_gf_backbones(topo) == ora.num_single_ptcle_gf_backbones(np.array(topo))
        a = dev.compute_single_ptcle_gf(m.G0, topo)
        b = ora.compute_single_ptcle_gf(m.G0, topo)
        nonzero += np.max(np.abs(b)) > 0  # one spin-orbital: only NCA and one TCA topology contribute
        assert _node_rel_err(a, b) <= 1.0, topo
    assert nonzero == 2


def test_two_fermion_interacting():
    beta, lam, eps = 2.0, 40.0, 1e-12
    d = O.Dlr(lam, eps)
    m = models.two_fermion(d.rf, d.it, beta, lam, eps, U=3.0, mu=0.7, hyb_pole=-1.5)
    dev, ora = _pair(m, d)
    for topo in TOPOS:
        a = dev.compute_single_ptcle_gf(m.G0, topo)
        b = ora.compute_single_ptcle_gf(m.G0, topo)
        assert _node_rel_err(a, b) <= 1.0, topo


def test_kanamori_small_basis_full_eval():
    beta, lam, eps = 4.0, 40.0, 1e-8
    d = O.Dlr(lam, eps)
    m = models.kanamori_2orb(d.rf, d.it, beta, lam, eps)
    G = models.seeded_G(m, 0)
    dev, ora = _pair(m, d)
    for topo in TOPOS:
        a = dev.compute_single_ptcle_gf(G, topo)
        b = ora.compute_single_ptcle_gf(G, topo)
        assert _node_rel_err(a, b) <= 1.0, topo


def test_kanamori_full_config_subset_and_zero_block():
    d = O.Dlr(200.0, 1e-12)
    m = models.kanamori_2orb(d.rf, d.it)
    G = models.seeded_G(m, 0)
    G[5] = np.zeros_like(G[5])  # a zero block prunes chains (the 1e-16 zero-block rule)
    dev, ora = _pair(m, d)
    rng = np.random.default_rng(12)
    for topo in TOPOS:
        nmax = ora.num_single_ptcle_gf_backbones(np.array(topo))
        fix = np.sort(rng.choice(nmax, size=min(nmax, 800), replace=False))
        a = dev.compute_single_ptcle_gf(G, topo, f_ix=fix)
        b = ora.compute_single_ptcle_gf(G, topo, f_ix=fix)
        assert _node_rel_err(a, b) <= 1.0, topo


def test_device_accumulation_matches_host_call():
    beta, lam, eps = 4.0, 40.0, 1e-8
    d = O.Dlr(lam, eps)
    m = models.kanamori_2orb(d.rf, d.it, beta, lam, eps)
    G = models.seeded_G(m, 1)
    dev, _ = _pair(m, d)
    gbuf = dev.device_buffer(0, dev.slab)
    obuf = dev.device_buffer(1, dev.r * dev.n * dev.n)
    dev.to_device(gbuf, dev.pack(G).real)
    dev.zero_device(obuf, dev.r * dev.n * dev.n)
    ref = np.zeros((dev.r, dev.n, dev.n))
    for k, topo in enumerate(TOPOS[:3]):
        dev.compute_single_ptcle_gf_device(gbuf, topo, 0.5 + k, obuf)
        ref += (0.5 + k) * dev.compute_single_ptcle_gf(G, topo).real
    got = dev.to_host(obuf, dev.r * dev.n * dev.n).reshape(ref.shape)
    assert _node_rel_err(got, ref) <= 1.0


def test_out_of_range_flat_index_raises():
    d = O.Dlr(40.0, 1e-8)
    m = models.kanamori_2orb(d.rf, d.it, 4.0, 40.0, 1e-8)
    dev, _ = _pair(m, d)
    nmax = dev.get_num_single_ptcle_gf_backbones([[0, 2], [1, 3]])
    from xca_b200._lib import XcaError
    with pytest.raises(XcaError):
        dev.compute_single_ptcle_gf(m.G0, [[0, 2], [1, 3]], f_ix=[nmax])
