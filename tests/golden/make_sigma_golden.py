"""Generates the golden Sigma fixtures of the full-size parity tests with the oracle (CPU restatement).

Each fixture holds the DLR basis the oracle built, the seeded pseudo-particle propagator G and, per
topology, the oracle's compute_self_energy(G, topology) over every flat index, summed in the fixed order
of the device's ordered mode (``Evaluator.compute_self_energy_ordered``, unit = 64 pole tuples), or over a
listed subset of flat indices (``fix_k``) summed in list order; the device must reproduce either bit for
bit in that mode.  Real parts are stored (every model here is real).

    python tests/golden/make_sigma_golden.py kanamori_2orb      # two-orbital Kanamori, orders 1-3 (minutes)
    python tests/golden/make_sigma_golden.py t2g_oca            # three-orbital t2g, orders 1-2
    python tests/golden/make_sigma_golden.py t2g_tca            # t2g, one third-order topology (about an hour on 8 cores)
    python tests/golden/make_sigma_golden.py dshell_subsets     # five-orbital d shell, random flat-index subsets
"""

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from xca_b200 import models  # noqa: E402

CONFIGS = {
    # name: (model builder, beta, Lambda, eps, topologies (None: all of orders 1..3))
    "kanamori_2orb": (models.kanamori_2orb, 20.0, 200.0, 1e-12, None),
    "t2g_oca": (models.t2g_3orb, 50.0, 500.0, 1e-10, [[[0, 1]], [[0, 2], [1, 3]]]),
    "t2g_tca": (models.t2g_3orb, 50.0, 500.0, 1e-10, [[[0, 3], [1, 4], [2, 5]]]),
    # five-orbital d shell (blocks up to 100 x 100): every flat index of orders 1 and 2 would take the CPU
    # restatement hours, so these are seeded random flat-index subsets, summed in list order
    "dshell_subsets": (models.dshell_5orb, 20.0, 200.0, 1e-8,
                       [([[0, 1]], None), ([[0, 2], [1, 3]], 40), ([[0, 3], [1, 4], [2, 5]], 120), ([[0, 4], [1, 3], [2, 5]], 120)]),
}


def generate(name, nthreads=0):
    build, beta, lam, eps, topos = CONFIGS[name]
    d = O.Dlr(lam, eps)
    m = build(d.rf, d.it, beta, lam, eps)
    G = models.seeded_G(m, 0)
    ev = O.Evaluator(d, beta, m.hyb_poles, m.hyb_coeffs, m.dims, m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks)
    if topos is None:
        topos = [topo for order in (1, 2, 3) for _, topo in O.connected_pairings(order)]
    out = {"rf": d.rf, "it": d.it, "G": np.concatenate([g.real.ravel() for g in G]), "dims": m.dims,
           "beta": beta, "lam": lam, "eps": eps, "n_topologies": len(topos)}
    rng = np.random.default_rng(11)
    for k, topo in enumerate(topos):
        t0 = time.time()
        if isinstance(topo, tuple):  # (topology, number of random flat indices or None for all)
            topo, nsub = topo
            t = np.array(topo, np.int32)
            nmax = ev.num_self_energy_backbones(t)
            fix = np.arange(nmax) if nsub is None else np.sort(rng.choice(nmax, size=nsub, replace=False))
            S = ev.compute_self_energy_list_ordered(G, t, fix, nthreads=nthreads)
            out[f"fix_{k}"] = fix
        else:
            S = ev.compute_self_energy_ordered(G, np.array(topo, np.int32), unit=64, nthreads=nthreads)
        out[f"topo_{k}"] = np.array(topo, np.int32)
        out[f"sigma_{k}"] = np.concatenate([s.real.ravel() for s in S])
        assert max(np.max(np.abs(s.imag)) for s in S) == 0.0
        print(f"{name} topology {topo}: {time.time() - t0:.1f} s", flush=True)
    path = os.path.join(HERE, f"sigma_{name}_ordered.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("config", choices=sorted(CONFIGS))
    ap.add_argument("--threads", type=int, default=0)
    a = ap.parse_args()
    generate(a.config, a.threads)
