"""The solve server: results do not depend on what else runs, the memory budget is enforced.

Each admitted solve owns its evaluator context (stream, device state), so a request's result in a mix of
concurrent solves must equal its result alone up to the summation order of the Sigma items on the
device (well-conditioned single-orbital Anderson requests: 1e-10 on G, eta and G(tau)).
"""

import numpy as np
import pytest

from xca_b200.serving import SolveServer, footprint_bytes, synthetic_request

pytestmark = pytest.mark.gpu


def _close(a, b, tol=1e-10):
    assert abs(a.eta - b.eta) < tol
    for x, y in zip(a.G, b.G):
        assert np.max(np.abs(x - y)) < tol
    assert np.max(np.abs(a.G_tau - b.G_tau)) < tol


@pytest.mark.parametrize("batched", [False, True])
def test_result_same_alone_and_in_mix(batched):
    probe = synthetic_request("anderson", 10.0, 2.5, 2, tag="probe")
    others = [synthetic_request("kanamori", 10.0, 4.0, 2, tag="k2"),
              synthetic_request("anderson", 20.0, 3.0, 3, tag="a3"),
              synthetic_request("kanamori", 20.0, 2.0, 1, tag="k1"),
              synthetic_request("anderson", 50.0, 1.5, 1, tag="a1")]
    srv = SolveServer(max_concurrent=1)
    alone = srv.submit(probe).result()
    srv.shutdown()
    srv = SolveServer(max_concurrent=4, batched=batched)
    futs = [srv.submit(r) for r in others[:2]] + [srv.submit(probe)] + [srv.submit(r) for r in others[2:]]
    results = [f.result() for f in futs]
    srv.shutdown()
    mixed = results[2]
    assert mixed.tag == "probe"
    assert alone.diff_G < probe.tol and mixed.diff_G < probe.tol
    assert alone.n_iter == mixed.n_iter
    _close(alone, mixed)
    for r in results:
        assert r.diff_G < 1e-8


def test_memory_budget_refuses_oversized_request():
    req = synthetic_request("anderson", 10.0, 2.0, 1)
    need = footprint_bytes(req.atom_diag, req.delta_tau.shape[0], req.delta_tau.shape[0], req.max_order)
    srv = SolveServer(max_concurrent=2, hbm_budget=need - 1)
    fut = srv.submit(req)
    with pytest.raises(MemoryError):
        fut.result()
    srv.shutdown()
