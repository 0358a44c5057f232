"""Serving of whole self-consistent pseudo-particle solves on one GPU.

Requests (a local problem, its hybridization and the solve parameters of BlockSparseSolver.solve,
``python/triqs_xca/block_sparse_solver.py:240-355``) arrive at any time.  The server admits a request
when its device-memory footprint fits into what the running solves leave of the budget, runs every
admitted solve in its own worker thread with its own evaluator context — its own CUDA stream, its G, Σ
and Dyson state resident on the device for the whole solve — so that the device work of concurrent
solves overlaps, and completes a future with the converged result and its timings (queue wait, time to
converged solve).  Solves never share device state, so a result does not depend on what else runs.
"""

import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

from .block_sparse_solver import BlockSparseSolver


@dataclass
class SolveRequest:
    atom_diag: object            # xca_b200.atom_diag.AtomDiag
    beta: float
    w_max: float
    eps: float
    delta_tau: np.ndarray        # (r, n, n) hybridization on the DLR nodes of (beta, w_max, eps)
    max_order: int = 1
    tol: float = 1e-8
    maxiter: int = 100
    mix: float = 1.0
    tag: object = None


@dataclass
class SolveResult:
    tag: object
    G: list
    Sigma: list
    eta: float
    G_tau: np.ndarray
    n_iter: int
    diff_G: float
    t_submit: float
    t_start: float
    t_done: float
    extra: dict = field(default_factory=dict)

    @property
    def latency(self):
        """Time from arrival to converged solve (s)."""
        return self.t_done - self.t_submit


def footprint_bytes(atom_diag, r, n_poles, max_order=3):
    """Device memory of one solve: G, Σ and Dyson slabs, edge tables, Dyson system matrices, operators."""
    dims = np.asarray(atom_diag.get_subspace_dims(), dtype=np.int64)
    slab = int(r * np.sum(dims ** 2))
    # edge tables of the orders the solve evaluates (1 + 2p signatures, 1 + 2p + 4p^2 for third order)
    nsig = 1 + 2 * n_poles + (4 * n_poles * n_poles if max_order >= 3 else 0)
    tables = nsig * 2 * slab
    mats = int(np.sum((r * dims) ** 2))
    n = atom_diag.n
    ops = int(np.sum(dims) ** 2) * n * (2 + 2 * n_poles)
    return 8 * (12 * slab + tables + mats + ops + 6 * slab) + (64 << 20)


class SolveServer:
    """Admits solve requests by device-memory budget and runs up to ``max_concurrent`` at a time."""

    def __init__(self, max_concurrent=8, hbm_budget=48 << 30, device=0):
        self.max_concurrent = max_concurrent
        self.budget = int(hbm_budget)
        self.device = device
        self._used = 0
        self._running = 0
        self._cv = threading.Condition()
        self._queue = []
        self._threads = []
        self._closed = False
        self._dispatcher = threading.Thread(target=self._dispatch, daemon=True)
        self._dispatcher.start()

    def submit(self, req: SolveRequest) -> Future:
        fut = Future()
        with self._cv:
            if self._closed:
                raise RuntimeError("server is shut down")
            self._queue.append((req, fut, time.perf_counter()))
            self._cv.notify_all()
        return fut

    def shutdown(self):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        self._dispatcher.join()
        for t in self._threads:
            t.join()

    def _dispatch(self):
        while True:
            with self._cv:
                while True:
                    if self._closed and not self._queue:
                        return
                    if self._queue and self._running < self.max_concurrent:
                        req, fut, t_sub = self._queue[0]
                        need = self._need(req)
                        if need > self.budget:
                            self._queue.pop(0)
                            fut.set_exception(MemoryError(f"solve needs {need} bytes, the budget is {self.budget}"))
                            continue
                        if self._used + need <= self.budget:
                            self._queue.pop(0)
                            self._used += need
                            self._running += 1
                            break
                    self._cv.wait()
            th = threading.Thread(target=self._run, args=(req, fut, t_sub, need), daemon=True)
            self._threads.append(th)
            th.start()

    @staticmethod
    def _need(req):
        r = req.delta_tau.shape[0]
        return footprint_bytes(req.atom_diag, r, r, req.max_order)

    def _run(self, req, fut, t_sub, need):
        t_start = time.perf_counter()
        try:
            S = BlockSparseSolver(req.atom_diag, req.beta, req.w_max, req.eps, device=self.device)
            if S.Delta_tau.shape != req.delta_tau.shape:
                raise ValueError(f"delta_tau has shape {req.delta_tau.shape}, the DLR mesh needs {S.Delta_tau.shape}")
            S.Delta_tau = np.asarray(req.delta_tau, dtype=np.complex128)
            S.solve(max_order=req.max_order, tol=req.tol, maxiter=req.maxiter, mix=req.mix)
            res = SolveResult(req.tag, S.G, S.Sigma, S.eta, S.G_tau, S.n_ppsc_iter, S.diff_G, t_sub, t_start,
                              time.perf_counter(), {"footprint_bytes": need})
            del S
            fut.set_result(res)
        except BaseException as e:  # the future carries the failure to the caller
            fut.set_exception(e)
        finally:
            with self._cv:
                self._used -= need
                self._running -= 1
                self._cv.notify_all()


def synthetic_request(kind, beta, U, order, eps=1e-10, tol=1e-8, maxiter=100, tag=None):
    """A request of the mixed serving stream: single-orbital Anderson or two-orbital Kanamori (J = U / 8)
    at half filling with a Bethe hybridization (t = 1), Lambda = 10 beta (w_max = 10)."""
    from . import models
    from .pycppdlr import MeshDLRImTime
    mesh = MeshDLRImTime(beta=beta, statistic="Fermion", w_max=10.0, eps=eps)
    rf, it = mesh.dlr_rf, mesh.dlr_it.it
    if kind == "anderson":
        m = models.anderson(rf, it, beta, 10.0 * beta, eps, U=U, mu=U / 2)
    else:
        m = models.kanamori_diag_bethe(rf, it, 2, beta, 10.0 * beta, eps, U, U / 8, "kanamori_2orb")
    delta = np.zeros((len(rf), m.n, m.n), np.complex128)
    dv = models.bethe_delta(beta, it)
    for i in range(m.n):
        delta[:, i, i] = dv
    return SolveRequest(m.ad, beta, 10.0, eps, delta, max_order=order, tol=tol, maxiter=maxiter, tag=tag)
