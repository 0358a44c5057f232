"""Serving of whole self-consistent pseudo-particle solves on one GPU.

Requests (a local problem, its hybridization and the solve parameters of BlockSparseSolver.solve,
``python/triqs_xca/block_sparse_solver.py:240-355``) arrive at any time.  The server admits a request
when its device-memory footprint fits into what the running solves leave of the budget and completes a
future with the converged result and its timings (queue wait, time to converged solve).  Every admitted
solve has its own evaluator context — its own CUDA stream, its G, Σ and Dyson state resident on the
device for the whole solve — so a result does not depend on what else runs (up to the summation order
of the Σ items).  Two ways to run them:

- lock step (``batched=True``): one scheduler thread runs an iteration of every live solve at a time,
  the Σ of all of them (every topology of every solve, grouped by padded DLR rank) in ONE job-batched
  launch (``DiagramEvaluator.compute_self_energy_device_batch``), then their Dyson solves, then their
  normalisations and convergence tests.  Set-up (hybridization fit, evaluator) and the final
  single-particle Green's function run in helper threads beside it; a solve joins the next iteration
  when its set-up is done and leaves when it converges;
- threads (``batched=False``, the default): each solve iterates in its own worker thread; the device work
  of concurrent solves overlaps through their streams, and each solve's own topologies share one batched
  launch per iteration.

Which is faster depends on the stream, measured: one batched launch ties its solves to the slowest of
them, so the lock step wins when the solves are alike and small (43 vs 29 solves/s on a stream of small
Anderson and Kanamori solves) and loses when their costs spread (5.2 vs 5.5 solves/s on the stream of
bench.py, which mixes t2g and beta = 100 third-order solves with small ones; 4.3 vs 5.8 at 16 concurrent).
"""

import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

from .block_sparse import DiagramEvaluator
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
    hyb_comp: bool = True        # compress the hybridization to a few poles (the reference's default)
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


@dataclass
class _Live:
    """A solve of the lock-step scheduler."""
    req: SolveRequest
    fut: Future
    t_submit: float
    t_start: float
    need: int
    solver: BlockSparseSolver
    it: int = 0


class SolveServer:
    """Admits solve requests by device-memory budget and runs up to ``max_concurrent`` at a time, each in
    its own thread or (``batched``) all in lock step with one Σ launch per iteration."""

    def __init__(self, max_concurrent=8, hbm_budget=48 << 30, device=0, batched=False):
        self.max_concurrent = max_concurrent
        self.budget = int(hbm_budget)
        self.device = device
        self.batched = bool(batched)
        self._used = 0
        self._running = 0
        self._cv = threading.Condition()
        self._queue = []
        self._threads = []
        self._arrived = []  # set up, waiting for the next lock-step iteration
        self._closed = False
        self.iterations = 0  # lock-step iterations run (batched)
        self._dispatcher = threading.Thread(target=self._dispatch, daemon=True)
        self._dispatcher.start()
        self._stepper = None
        if self.batched:
            self._stepper = threading.Thread(target=self._step_loop, daemon=True)
            self._stepper.start()

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
        if self._stepper is not None:
            self._stepper.join()
        for t in list(self._threads):
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
            th = threading.Thread(target=self._setup if self.batched else self._run, args=(req, fut, t_sub, need), daemon=True)
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
            S.solve(max_order=req.max_order, tol=req.tol, maxiter=req.maxiter, mix=req.mix, hyb_comp=req.hyb_comp)
            res = SolveResult(req.tag, S.G, S.Sigma, S.eta, S.G_tau, S.n_ppsc_iter, S.diff_G, t_sub, t_start,
                              time.perf_counter(), {"footprint_bytes": need})
            del S
            fut.set_result(res)
        except BaseException as e:  # the future carries the failure to the caller
            fut.set_exception(e)
        finally:
            self._release(need)

    def _release(self, need):
        with self._cv:
            self._used -= need
            self._running -= 1
            self._cv.notify_all()

    # ---------------------------------------------------------------- lock step (batched=True)
    def _setup(self, req, fut, t_sub, need):
        t_start = time.perf_counter()
        try:
            S = BlockSparseSolver(req.atom_diag, req.beta, req.w_max, req.eps, device=self.device)
            if S.Delta_tau.shape != req.delta_tau.shape:
                raise ValueError(f"delta_tau has shape {req.delta_tau.shape}, the DLR mesh needs {S.Delta_tau.shape}")
            S.Delta_tau = np.asarray(req.delta_tau, dtype=np.complex128)
            S.begin(req.max_order, tol=req.tol, hyb_comp=req.hyb_comp)
            S.d.synchronize()
        except BaseException as e:
            fut.set_exception(e)
            self._release(need)
            return
        with self._cv:
            self._arrived.append(_Live(req, fut, t_sub, t_start, need, S))
            self._cv.notify_all()

    def _step_loop(self):
        live = []
        while True:
            with self._cv:
                while not live and not self._arrived:
                    if self._closed and self._running == 0 and not self._queue:
                        return
                    self._cv.wait()
                live.extend(self._arrived)
                self._arrived.clear()
            self._iterate(live)
            self.iterations += 1

    def _fail(self, live, L, e):
        live.remove(L)
        L.solver = None
        L.fut.set_exception(e)
        self._release(L.need)

    def _iterate(self, live):
        """One iteration of every live solve: their Σ in one launch per padded rank, Dyson solves queued on every
        stream, then normalisation and convergence test per solve; converged solves leave for a finisher."""
        groups = {}
        for L in live:
            groups.setdefault(L.solver.d.padded_rank, []).append(L)
        for grp in groups.values():
            try:
                jobs = []
                for L in grp:
                    jobs += L.solver.sigma_jobs(L.req.max_order)
                DiagramEvaluator.compute_self_energy_device_batch(jobs)
            except BaseException as e:
                for L in grp:
                    self._fail(live, L, e)
        for L in list(live):
            try:
                L.solver.launch_dyson()
            except BaseException as e:
                self._fail(live, L, e)
        for L in list(live):
            L.it += 1
            try:
                done = L.solver.end_iteration(L.it, L.req.tol, L.req.mix, dyson_launched=True) or L.it >= L.req.maxiter
            except BaseException as e:
                self._fail(live, L, e)
                continue
            if done:
                live.remove(L)
                th = threading.Thread(target=self._finish, args=(L,), daemon=True)
                self._threads.append(th)
                th.start()

    def _finish(self, L):
        try:
            S = L.solver.finish()
            L.solver = None
            res = SolveResult(L.req.tag, S.G, S.Sigma, S.eta, S.G_tau, S.n_ppsc_iter, S.diff_G, L.t_submit, L.t_start,
                              time.perf_counter(), {"footprint_bytes": L.need, "batched": True})
            del S
            L.fut.set_result(res)
        except BaseException as e:
            L.fut.set_exception(e)
        finally:
            self._release(L.need)


# DLR accuracy of each model family of the served stream (the accuracy its single-solve configuration uses)
STREAM_EPS = {"anderson": 1e-10, "kanamori": 1e-12, "t2g": 1e-10}


def synthetic_request(kind, beta, U, order, eps=None, tol=1e-8, maxiter=100, tag=None, hyb_comp=True):
    """A request of the mixed serving stream, Lambda = 10 beta (w_max = 10), at half filling:
    'anderson': single-orbital Anderson with a Bethe hybridization (t = 1);
    'kanamori': two-orbital Kanamori (J = U / 8) with a diagonal Bethe hybridization;
    't2g': three-orbital t2g Kanamori (J = U / 10) with the off-diagonal 8-pole bath of numpy default_rng(1)
    (poles w_k ~ U(-2, 2), weights V_k V_k^T, V_k ~ N(0, 0.3^2)).  eps defaults to STREAM_EPS[kind]."""
    from . import models
    from .pycppdlr import MeshDLRImTime
    eps = STREAM_EPS[kind] if eps is None else eps
    mesh = MeshDLRImTime(beta=beta, statistic="Fermion", w_max=10.0, eps=eps)
    rf, it = mesh.dlr_rf, mesh.dlr_it.it
    if kind == "t2g":
        m = models.t2g_3orb(rf, it, beta, 10.0 * beta, eps, U=U, J=U / 10)
        delta = np.asarray(m.extra["delta"], np.complex128)
    else:
        if kind == "anderson":
            m = models.anderson(rf, it, beta, 10.0 * beta, eps, U=U, mu=U / 2)
        elif kind == "kanamori":
            m = models.kanamori_diag_bethe(rf, it, 2, beta, 10.0 * beta, eps, U, U / 8, "kanamori_2orb")
        else:
            raise ValueError(f"unknown model family {kind!r}")
        delta = np.zeros((len(rf), m.n, m.n), np.complex128)
        dv = models.bethe_delta(beta, it)
        for i in range(m.n):
            delta[:, i, i] = dv
    return SolveRequest(m.ad, beta, 10.0, eps, delta, max_order=order, tol=tol, maxiter=maxiter, hyb_comp=hyb_comp, tag=tag)
