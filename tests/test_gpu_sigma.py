"""GPU parity of the Sigma backbone evaluation against the CPU oracle, through the C-ABI.

Tolerance (FP64 plain path): per tau node, max_{block, i, j} |Sigma_gpu - Sigma_oracle| <= 1e-12 *
max_{block, i, j} |Sigma_oracle(tau)| + 1e-15, i.e. 1e-12 relative per tau node with an absolute floor
at the double-precision round-off of the O(1) inputs.  Item lists are compared bit-exactly.
"""

import numpy as np
import pytest

from oracle import oracle as O
from xca_b200 import models

pytestmark = pytest.mark.gpu

REL = 1e-12
ABS = 1e-15


def _node_rel_err(A, B):
    """max over tau nodes of ||A(t) - B(t)||_max / (||B(t)||_max) with an absolute floor."""
    r = A[0].shape[0]
    worst = 0.0
    for t in range(r):
        num = max(np.max(np.abs(a[t] - b[t])) for a, b in zip(A, B))
        den = max(np.max(np.abs(b[t])) for b in B)
        worst = max(worst, num / (REL * den + ABS))
    return worst  # <= 1 passes


def _pair(model, dlr):
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    Fq = BlockOpSymQuartet(model.labels, model.F_index, model.F_blocks, model.Fd_index, model.Fd_blocks, model.dims)
    dev = DiagramEvaluator.from_arrays(model.beta, model.lam, model.eps, dlr.rf, dlr.it, model.hyb_poles, model.hyb_coeffs, Fq)
    ora = O.Evaluator(dlr, model.beta, model.hyb_poles, model.hyb_coeffs, model.dims, model.labels, model.F_index,
                      model.F_blocks, model.Fd_index, model.Fd_blocks)
    return dev, ora


TOPOS = [[[0, 1]], [[0, 2], [1, 3]], [[0, 2], [1, 4], [3, 5]], [[0, 3], [1, 4], [2, 5]], [[0, 3], [1, 5], [2, 4]],
         [[0, 4], [1, 3], [2, 5]]]


@pytest.mark.parametrize("pole", [0.0, 0.8, -1.3])
def test_one_fermion_all_topologies(pole):
    beta, lam, eps = 2.0, 40.0, 1e-10
    d = O.Dlr(lam, eps)
    m = models.one_fermion(d.rf, d.it, beta, lam, eps, hyb_pole=pole)
    dev, ora = _pair(m, d)
    for topo in TOPOS:
        a = dev.compute_self_energy(m.G0, topo)
        b = ora.compute_self_energy(m.G0, topo)
        assert _node_rel_err(a, b) <= 1.0, topo


def test_two_fermion_interacting():
    beta, lam, eps = 2.0, 40.0, 1e-12
    d = O.Dlr(lam, eps)
    m = models.two_fermion(d.rf, d.it, beta, lam, eps, U=3.0, mu=0.7, hyb_pole=-1.5)
    dev, ora = _pair(m, d)
    for topo in TOPOS:
        a = dev.compute_self_energy(m.G0, topo)
        b = ora.compute_self_energy(m.G0, topo)
        assert _node_rel_err(a, b) <= 1.0, topo


def test_kanamori_small_basis_full_eval():
    # the 2-orbital Kanamori model on a reduced basis (Lambda = 40, eps = 1e-8): every flat index
    beta, lam, eps = 4.0, 40.0, 1e-8
    d = O.Dlr(lam, eps)
    m = models.kanamori_2orb(d.rf, d.it, beta, lam, eps)
    G = models.seeded_G(m, 0)
    dev, ora = _pair(m, d)
    for topo in TOPOS:
        a = dev.compute_self_energy(G, topo)
        b = ora.compute_self_energy(G, topo)
        assert _node_rel_err(a, b) <= 1.0, topo


def test_kanamori_full_config_subset():
    # the benchmark configuration (beta = 20, Lambda = 200, eps = 1e-12) on a seeded subset of flat indices
    d = O.Dlr(200.0, 1e-12)
    m = models.kanamori_2orb(d.rf, d.it)
    G = models.seeded_G(m, 0)
    dev, ora = _pair(m, d)
    rng = np.random.default_rng(11)
    for topo in TOPOS:
        nmax = ora.num_self_energy_backbones(np.array(topo))
        assert dev.get_num_self_energy_backbones(topo) == nmax
        fix = np.sort(rng.choice(nmax, size=min(nmax, 1500), replace=False))
        a = dev.compute_self_energy(G, topo, f_ix=fix)
        b = ora.compute_self_energy(G, topo, f_ix=fix)
        assert _node_rel_err(a, b) <= 1.0, topo


def test_item_list_bit_exact():
    d = O.Dlr(200.0, 1e-12)
    m = models.kanamori_2orb(d.rf, d.it)
    G = models.seeded_G(m, 0)
    G[3] = np.zeros_like(G[3])  # a zero block prunes paths (the 1e-16 zero-block rule)
    dev, ora = _pair(m, d)
    for topo in TOPOS[:4]:
        nmax = ora.num_self_energy_backbones(np.array(topo))
        k = min(nmax, 30000)
        a = dev.self_energy_items(G, topo, max_rows=None)
        b = ora.item_list(G, np.array(topo), 0, nmax)
        assert a.shape == b.shape and np.array_equal(a, b), topo
        assert k > 0


def test_out_of_range_flat_index_raises():
    d = O.Dlr(40.0, 1e-8)
    m = models.kanamori_2orb(d.rf, d.it, 4.0, 40.0, 1e-8)
    dev, _ = _pair(m, d)
    nmax = dev.get_num_self_energy_backbones([[0, 2], [1, 3]])
    from xca_b200._lib import XcaError
    with pytest.raises(XcaError):
        dev.compute_self_energy(m.G0, [[0, 2], [1, 3]], f_ix=[nmax])


def test_rejects_cross_set_coefficients():
    d = O.Dlr(40.0, 1e-8)
    m = models.kanamori_2orb(d.rf, d.it, 4.0, 40.0, 1e-8)
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    Fq = BlockOpSymQuartet(m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks, m.dims)
    bad = m.hyb_coeffs.copy()
    bad[:, 0, 2] = 0.1  # orbitals 0 and 2 are in different symmetry sets
    with pytest.raises(ValueError):
        DiagramEvaluator.from_arrays(m.beta, m.lam, m.eps, d.rf, d.it, m.hyb_poles, bad, Fq)


@pytest.mark.parametrize("n_shards", [1, 3])
def test_shards_partition_the_work(n_shards):
    # the work-unit shards of every rank, evaluated one after another on one GPU, add up to the full Sigma
    from xca_b200.distributed import sigma_terms
    d = O.Dlr(40.0, 1e-8)
    m = models.kanamori_2orb(d.rf, d.it, 4.0, 40.0, 1e-8)
    G = models.seeded_G(m, 2)
    dev, _ = _pair(m, d)
    gbuf = dev.device_buffer(0, dev.slab)
    full = dev.device_buffer(1, dev.slab)
    part = dev.device_buffer(2, dev.slab)
    dev.to_device(gbuf, dev.pack(G).real)
    dev.zero_device(full, dev.slab)
    dev.zero_device(part, dev.slab)
    for _, topo, fac in sigma_terms(3):
        dev.compute_self_energy_device(gbuf, topo, fac, full)
        for s in range(n_shards):
            dev.compute_self_energy_device_shard(gbuf, topo, fac, part, s, n_shards)
    a = dev.unpack(dev.to_host(part, dev.slab))
    b = dev.unpack(dev.to_host(full, dev.slab))
    assert _node_rel_err(a, b) <= 1.0


def test_t2g_three_orbital_subset():
    # three-orbital t2g Kanamori (U = 3, J = 0.3, beta = 50, Lambda = 500, eps = 1e-10; 16 blocks up to 9 x 9,
    # orbital-off-diagonal hybridization) on a seeded subset of flat indices of every topology
    d = O.Dlr(500.0, 1e-10)
    m = models.t2g_3orb(d.rf, d.it)
    G = models.seeded_G(m, 0)
    dev, ora = _pair(m, d)
    rng = np.random.default_rng(13)
    for topo in TOPOS:
        nmax = ora.num_self_energy_backbones(np.array(topo))
        fix = np.sort(rng.choice(nmax, size=min(nmax, 300), replace=False))
        a = dev.compute_self_energy(G, topo, f_ix=fix)
        b = ora.compute_self_energy(G, topo, f_ix=fix)
        assert _node_rel_err(a, b) <= 1.0, topo
