"""The solver's state I/O on the host (no GPU): __reduce_to_dict__ / __factory_from_dict__ and the .npz round
trip keep every array and scalar (block_sparse_solver.py:1133-1204)."""

import numpy as np

from xca_b200 import models


def test_state_round_trip(tmp_path):
    from xca_b200.block_sparse_solver import BlockSparseSolver
    from xca_b200.pycppdlr import MeshDLRImTime
    beta, lam, eps = 10.0, 100.0, 1e-10
    mesh = MeshDLRImTime(beta=beta, statistic="Fermion", w_max=lam / beta, eps=eps)
    m = models.kanamori_2orb(mesh.dlr_rf, mesh.dlr_it.it, beta, lam, eps)
    S = BlockSparseSolver(m.ad, beta, lam / beta, eps, precision="fp64_ordered")
    S.G = models.seeded_G(m, 3)
    S.eta = 0.123
    S.n_ppsc_iter = 7
    S.diff_G = 1e-9
    S.Delta_tau[:, 0, 0] = 0.25
    path = str(tmp_path / "s.npz")
    S.save(path)
    R = BlockSparseSolver.load(path)
    assert R == S
    assert R.precision == "fp64_ordered"
    assert R.ad.get_subspace_dims() == S.ad.get_subspace_dims()
    assert all(np.array_equal(a, b) for a, b in zip(R.G, S.G))
    R.eta = 0.5
    assert not (R == S)
