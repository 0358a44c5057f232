"""The launch-shape autotuner: it chooses a setting no slower than the default, records it, re-applies it,
and the ordered-mode result does not depend on the setting (bit for bit)."""

import numpy as np
import pytest

from oracle import oracle as O
from xca_b200 import autotune, models

pytestmark = pytest.mark.gpu


def test_autotune_kanamori(tmp_path):
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    beta, lam, eps = 20.0, 200.0, 1e-12
    d = O.Dlr(lam, eps)
    m = models.kanamori_2orb(d.rf, d.it, beta, lam, eps)
    Fq = BlockOpSymQuartet(m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks, m.dims)
    ev = DiagramEvaluator.from_arrays(beta, lam, eps, d.rf, d.it, m.hyb_poles, m.hyb_coeffs, Fq)
    G = models.seeded_G(m, 0)
    bg, bs = ev.device_buffer(30, ev.slab), ev.device_buffer(31, ev.slab)
    ev.to_device(bg, ev.pack(G).real)
    terms = [(np.array(t, np.int32), (-1) ** 3 * s * (-1) ** 4) for s, t in O.connected_pairings(3)]
    cache = str(tmp_path / "tuning.json")
    setting, table = autotune.tune_sigma(ev, bg, bs, terms, reps=1, params=["unit_batches"], cache_path=cache, device_name="test")
    start_ms = table[0][2]
    best_ms = min(ms for _, _, ms in table)
    print("autotune:", setting, [(n, v, round(ms, 2)) for n, v, ms in table])
    assert ev.get_tuning() == setting
    ev.set_tuning(unit_batches=4)
    assert autotune.apply_cached(ev, terms, cache_path=cache, device_name="test") == setting
    assert best_ms <= start_ms
    # ordered mode: the same bits for every setting
    ev.precision_mode = "fp64_ordered"
    res = []
    for ub in (1, 16):
        ev.set_tuning(unit_batches=ub)
        ev.zero_device(bs, ev.slab)
        ev.compute_self_energy_device(bg, terms[0][0], 1.0, bs)
        res.append(ev.to_host(bs, ev.slab))
    assert np.array_equal(res[0], res[1])
