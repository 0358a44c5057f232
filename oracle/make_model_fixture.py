"""Writes the benchmark model as plain arrays for the CPU reference leg of ``bench.py`` (test and
measurement infrastructure): the two-orbital Kanamori model (U = 4, J = 0.5, half filling, beta = 20,
diagonal Bethe hybridization t = 1 fitted on the DLR poles) on the oracle's DLR basis (Lambda = 200,
eps = 1e-12), its field operators in (N_up, N_dn) blocks and the seeded propagator G (numpy
default_rng(0)).  The CPU leg loads this file and the oracle only, so no library of the product is
mapped into that process.

    python oracle/make_model_fixture.py
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import dlr_ref  # noqa: E402
from oracle.oracle import pack_ops  # noqa: E402
from xca_b200 import models  # noqa: E402

PATH = os.path.join(HERE, "fixtures", "kanamori_2orb_beta20_L200_eps1e-12.npz")


def main():
    beta, lam, eps = 20.0, 200.0, 1e-12
    rf = dlr_ref.build_dlr_rf(lam, eps)
    it = dlr_ref.build_dlr_it(lam, rf)
    m = models.kanamori_2orb(rf, it, beta, lam, eps)
    G = models.seeded_G(m, 0)
    fi, fd = pack_ops(m.dims, m.F_index, m.F_blocks)
    gi, gd = pack_ops(m.dims, m.Fd_index, m.Fd_blocks)
    os.makedirs(os.path.dirname(PATH), exist_ok=True)
    np.savez_compressed(PATH, beta=beta, lam=lam, eps=eps, rf=rf, it=it, dims=m.dims, labels=m.labels, F_index=fi, F_data=fd,
                        Fd_index=gi, Fd_data=gd, hyb_poles=m.hyb_poles, hyb_coeffs=m.hyb_coeffs,
                        G=np.concatenate([g.ravel() for g in G]))
    print("wrote", PATH)


if __name__ == "__main__":
    main()
