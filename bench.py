"""Benchmark: TCA pseudo-particle self-energy evaluations per second on the two-orbital
Hubbard-Kanamori model (4 spin-orbitals, 9 (N_up, N_dn) blocks of size <= 4, U = 4, J = 0.5,
U' = 3, half filling mu = 4.75, beta = 20, DLR Lambda = 200, eps = 1e-12, diagonal Bethe
hybridization t = 1 fitted on the DLR poles, fixed seeded G_pp from numpy default_rng(0)).

One step = one full Sigma evaluation: orders 1..3, every connected topology, every flat index,
every block, accumulated with the reference's signs (python/triqs_xca/block_sparse_solver.py:597-640).

  python bench.py [--gpus N --steps K --warmup W] [--impl xca|reference]

Under torchrun (N > 1) every rank evaluates an interleaved shard of the work units of each topology
and the partial Sigma slabs are summed with one NCCL all-reduce per step (strong scaling).
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "TCA Sigma(tau) evals/s (FP64 plain)"
UNIT = "evals/s"
CONFIG_NAME = "kanamori_2orb_beta20_L200_eps1e-12_TCA"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="xca", choices=["xca", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="bounded CPU sample length")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end host-API measurement (profiling runs)")
    ap.add_argument("--serving", action="store_true",
                    help="instead of the Sigma metric: a Poisson stream of whole self-consistent solves through the solve server")
    ap.add_argument("--serving-requests", type=int, default=256)
    ap.add_argument("--serving-concurrency", type=int, default=8, help="solves the server runs at once")
    ap.add_argument("--no-serving", action="store_true", help="skip the served-solves measurement of the default line")
    ap.add_argument("--dshell", action="store_true",
                    help="instead of the Sigma metric: OCA Sigma of the five-orbital d shell (wide-chain kernel)")
    ap.add_argument("--dshell-stride", type=int, default=1,
                    help="with --dshell: evaluate every n-th flat index only (a small case, e.g. for a kernel profile)")
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-shape autotuner")
    ap.add_argument("--no-variants", action="store_true", help="skip the compressed-hybridization variant")
    return ap.parse_args()


def topologies(max_order=3):
    from xca_b200.distributed import sigma_terms
    return [(order, np.array(topo, np.int32), fac) for order, topo, fac in sigma_terms(max_order)]


def build_model():
    from xca_b200 import models
    from xca_b200.pycppdlr import ImTimeOps, build_dlr_rf
    rf = build_dlr_rf(200.0, 1e-12)
    it = ImTimeOps(200.0, rf).get_itnodes()
    m = models.kanamori_2orb(rf, it)
    G = models.seeded_G(m, 0)
    return m, G


MODEL_FIXTURE = os.path.join(ROOT, "oracle", "fixtures", "kanamori_2orb_beta20_L200_eps1e-12.npz")


def cpu_model():
    """(CPU model name, logical CPUs usable by this process) of the host."""
    name = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                name = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count()
    return name, usable


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index):
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix="xca_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, smax, reasons = [], [], set()
        lines = open(self.path).read().splitlines()
        os.unlink(self.path)
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_sigma_sample(seconds, nthreads=0, seed=7):
    """The oracle (CPU restatement of the reference's path) on a bounded random sample of flat indices of
    every topology of the benchmark model, loaded from the oracle's model file (no product library is
    mapped).  Returns (evals/s extrapolated to the full evaluation, wall seconds of the sample, threads,
    sample description)."""
    from oracle import oracle as O
    _, ev, G = O.Evaluator.from_fixture(MODEL_FIXTURE)
    topos = [np.array(t, np.int32) for order in (1, 2, 3) for _, t in O.connected_pairings(order)]
    rng = np.random.default_rng(seed)
    nmax = [ev.num_self_energy_backbones(t) for t in topos]
    per_topo = seconds / len(topos)
    total_est, wall, sampled = 0.0, 0.0, 0
    for t, nm in zip(topos, nmax):
        k = min(nm, 64)
        while True:
            fix = np.sort(rng.choice(nm, size=k, replace=False))
            t0 = time.perf_counter()
            ev.compute_self_energy(G, t, f_ix=fix, nthreads=nthreads)
            dt = time.perf_counter() - t0
            wall += dt
            if dt > 0.2 * per_topo or k == nm:
                break
            k = min(nm, max(k * 2, int(k * 0.5 * per_topo / max(dt, 1e-6))))
        total_est += dt * nm / k
        sampled += k
    threads = nthreads or int(os.environ.get("OMP_NUM_THREADS", cpu_model()[1]))
    return (1.0 / total_est, wall, threads,
            f"{sampled} random flat indices over {len(topos)} topologies, time extrapolated to all {sum(nmax)} flat indices")


def cpu_baseline_object(seconds):
    """cpu_baseline of the GPU arm: all host threads, plus a 1-thread figure on a shorter sample."""
    v, wall, cores, sample = cpu_sigma_sample(seconds)
    v1, _, _, _ = cpu_sigma_sample(max(seconds / 4, 2.0), nthreads=1, seed=8)
    name, usable = cpu_model()
    return {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample, "value_1thread": v1,
            "cpu_model": name, "host_cpus": usable, "sample_wall_s": wall}


def run_serving(args, batched=False):
    """Served solves/s and p50 / p99 time to converged solve for a mixed request stream: Poisson arrivals
    (mean gap 5 ms, numpy default_rng(2)); each request draws a model family (single-orbital Anderson,
    two-orbital Kanamori, three-orbital t2g with its 8-pole off-diagonal bath), beta in {10, 20, 50, 100},
    Lambda = 10 beta, U ~ U(1, 6), an order in {NCA, OCA, TCA} (t2g: NCA, OCA) and tolerance 1e-8, at most
    100 iterations, the hybridization compressed as the reference's solve does by default.  Up to
    --serving-concurrency solves (default 8) run concurrently, each with its own context and stream, in lock
    step with one Sigma launch per iteration for all of them (``batched``) or in worker threads."""
    from xca_b200.serving import SolveServer, STREAM_EPS, synthetic_request
    rng = np.random.default_rng(2)
    n = args.serving_requests
    gaps = rng.exponential(0.005, n)
    kinds = ("anderson", "kanamori", "t2g")
    reqs = []
    for i in range(n):
        kind = kinds[int(rng.integers(0, 3))]
        beta = float(rng.choice([10.0, 20.0, 50.0, 100.0]))
        U = float(rng.uniform(1.0, 6.0))
        order = int(rng.integers(1, 3 if kind == "t2g" else 4))
        reqs.append(synthetic_request(kind, beta, U, order, tag=(kind, beta, order)))
    srv = SolveServer(max_concurrent=args.serving_concurrency, batched=batched)
    for kind, order in (("anderson", 3), ("kanamori", 3), ("t2g", 2)):  # warm-up: module load and first-use set-up
        srv.submit(synthetic_request(kind, 10.0, 2.0, order)).result()
    t0 = time.perf_counter()
    futs = []
    t_next = t0
    for req, gap in zip(reqs, gaps):
        t_next += gap
        wait = t_next - time.perf_counter()
        if wait > 0:
            time.sleep(wait)
        futs.append(srv.submit(req))
    res = [f.result() for f in futs]
    t1 = max(r.t_done for r in res)
    srv.shutdown()
    lat = np.array([r.latency for r in res])
    out = {"metric": "served solves/s (FP64 plain, mixed stream)", "value": n / (t1 - t0), "unit": "solves/s", "n_gpus": 1,
           "higher_is_better": True, "dtype": "f64", "data": "synthetic",
           "config": {"workload": "poisson_stream", "requests": n, "mean_gap_ms": 5.0, "max_concurrent": args.serving_concurrency,
                      "mode": "lock step, one batched Sigma launch per iteration" if batched else "worker threads",
                      "models": "anderson, kanamori_2orb, t2g_3orb (U ~ U(1, 6))", "orders": "1-3; t2g 1-2",
                      "t2g_tca_excluded": "a t2g TCA solve alone takes 41-172 s (0.45 s per iteration, up to 100 iterations)",
                      "beta": [10, 20, 50, 100], "lambda": "10 beta", "eps": STREAM_EPS, "tol": 1e-8, "maxiter": 100,
                      "hyb_comp": True},
           "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
           "mean_iterations": float(np.mean([r.n_iter for r in res])),
           "converged": int(sum(r.diff_G < 1e-8 for r in res)), "wall_s": t1 - t0}
    return out


def _per_node_rel(ev, a, b):
    """max over tau nodes of max |a - b| / max |b| at that node (all blocks)."""
    num, den, off = np.zeros(ev.r), np.zeros(ev.r), 0
    for d in ev.dims:
        sz = ev.r * d * d
        num = np.maximum(num, np.max(np.abs(a[off:off + sz] - b[off:off + sz]).reshape(ev.r, -1), axis=1))
        den = np.maximum(den, np.max(np.abs(b[off:off + sz]).reshape(ev.r, -1), axis=1))
        off += sz
    return float(np.max(num / np.maximum(den, 1e-300)))


def precision_variants(m, G, device):
    """The same evaluation (1) with the Bethe hybridization compressed to a few poles inside the band
    (fit_hybridization(compression=True), xca_b200.hyb_fit, tolerance 1e-10) in place of one pole per DLR
    frequency, and (2) with FP32 block products (the mixed form's bulk arithmetic, evaluator mode 'fp32'), for
    both pole sets: evals/s and the change of Sigma against FP64 (per tau node, relative to the node's largest
    entry).  (3) The mixed solve against the FP64 one: the same model from its atomic G0, TCA with the
    compressed hybridization, to 1e-10: time, iterations and the difference of the converged G(tau)."""
    import torch
    from xca_b200 import hyb_fit, models
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    from xca_b200.block_sparse_solver import BlockSparseSolver
    from xca_b200.distributed import self_energy_sharded
    dv = models.bethe_delta(m.beta, m.it)
    delta = np.zeros((m.r, m.n, m.n))
    for i in range(m.n):
        delta[:, i, i] = dv
    poles, coeffs, err = hyb_fit.compress_hybridization(m.rf, m.it, m.beta, delta, 1e-10)
    Fq = BlockOpSymQuartet(m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks, m.dims)
    res = {}
    for name, (p, c) in (("dlr", (m.hyb_poles, m.hyb_coeffs)), ("compressed", (poles, coeffs))):
        ev = DiagramEvaluator.from_arrays(m.beta, m.lam, m.eps, m.rf, m.it, p, c, Fq, device=device)
        dev = torch.device("cuda", device)
        G_t = torch.tensor(np.concatenate([g.real.ravel() for g in G]), dtype=torch.float64, device=dev)
        S_t = torch.zeros(ev.slab, dtype=torch.float64, device=dev)
        terms = topologies()
        for mode in ("fp64", "fp32"):
            ev.precision_mode = mode
            for _ in range(2):
                self_energy_sharded(ev, G_t.data_ptr(), S_t.data_ptr(), terms, 0, 1)
            ms = []
            for _ in range(3):
                ev.flush_l2(256 << 20)
                ev.event_record(0)
                self_energy_sharded(ev, G_t.data_ptr(), S_t.data_ptr(), terms, 0, 1)
                ev.event_record(1)
                ms.append(ev.event_elapsed(0, 1))
            res[(name, mode)] = (float(np.median(ms)), S_t.cpu().numpy())
        res[name] = ev
    ref = res[("dlr", "fp64")][1]
    diff = float(np.max(np.abs(res[("compressed", "fp64")][1] - ref)) / np.max(np.abs(ref)))
    out = {"compressed_hybridization": {"value": 1000.0 / res[("compressed", "fp64")][0], "unit": UNIT, "poles": int(len(poles)),
                                        "fit_error": float(err), "sigma_rel_change_vs_dlr_poles": diff,
                                        "ms_per_step": res[("compressed", "fp64")][0]}}
    mixed = {}
    for name in ("dlr", "compressed"):
        t32, s32 = res[(name, "fp32")]
        t64, s64 = res[(name, "fp64")]
        mixed[f"fp32_sigma_{name}_poles"] = {"value": 1000.0 / t32, "unit": UNIT, "ms_per_step": t32, "fp64_ms_per_step": t64,
                                             "per_node_rel_err_vs_fp64": _per_node_rel(res[name], s32, s64),
                                             "input": "seeded G (default_rng(0))"}
    solves = {}
    for precision in ("fp64", "mixed"):
        S = BlockSparseSolver(m.ad, m.beta, m.lam / m.beta, m.eps, device=device, precision=precision)
        S.Delta_tau = delta.astype(np.complex128)
        S.solve(max_order=3, tol=1e-10, maxiter=60, hyb_comp=True, hyb_tol=1e-11)
        solves[precision] = S
    a, b = solves["mixed"], solves["fp64"]
    mixed["solve"] = {"model": "kanamori_2orb TCA from G0, compressed hybridization", "tol": 1e-10,
                      "fp64_solve_loop_s": b.timings["solve_loop_s"], "mixed_solve_loop_s": a.timings["solve_loop_s"],
                      "fp64_iterations": int(b.n_ppsc_iter), "mixed_fp32_iterations": int(a.n_fp32_iter),
                      "mixed_fp64_iterations": int(a.n_ppsc_iter - a.n_fp32_iter),
                      "max_abs_diff_G_tau_vs_fp64": float(np.max(np.abs(a.G_tau - b.G_tau))),
                      "max_abs_diff_G_vs_fp64": max(float(np.max(np.abs(x - y))) for x, y in zip(a.G, b.G))}
    out["mixed"] = mixed
    return out


def run_dshell(args):
    """OCA Sigma evaluations per second of the five-orbital d shell (10 spin-orbitals, N = 4..6: 672 states in
    16 (N_up, N_dn) blocks up to 100 x 100; Slater F0 = 4, J = 0.7, F4 / F2 = 0.625; beta = 20, Lambda = 200,
    eps = 1e-8, r = 31; diagonal Bethe hybridization on the DLR poles; seeded G from default_rng(0)).  Every
    chain is wider than a shared-memory panel, so the wide-chain kernel does the work.  One step is the
    device-resident evaluation of the OCA topology over every flat index, or with --dshell-stride n over every
    n-th flat index (through the host API's flat-index list)."""
    from xca_b200 import models
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    from xca_b200.pycppdlr import ImTimeOps, build_dlr_rf
    lam, eps, beta = 200.0, 1e-8, 20.0
    rf = build_dlr_rf(lam, eps)
    it = ImTimeOps(lam, rf).get_itnodes()
    m = models.dshell_5orb(rf, it, beta, lam, eps)
    G = models.seeded_G(m, 0)
    Fq = BlockOpSymQuartet(m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks, m.dims)
    ev = DiagramEvaluator.from_arrays(beta, lam, eps, rf, it, m.hyb_poles, m.hyb_coeffs, Fq)
    topo = np.array([[0, 2], [1, 3]], np.int32)
    flops, items = ev.self_energy_flops(G, topo)
    stride = max(1, args.dshell_stride)
    if stride > 1:
        fix = np.arange(0, ev.get_num_self_energy_backbones(topo), stride)

        def step():
            ev.compute_self_energy(G, topo, f_ix=fix)
        frac = len(fix) / ev.get_num_self_energy_backbones(topo)
    else:
        bg, bs = ev.device_buffer(30, ev.slab), ev.device_buffer(31, ev.slab)
        ev.to_device(bg, ev.pack(G).real)

        def step():
            ev.zero_device(bs, ev.slab)
            ev.compute_self_energy_device(bg, topo, 1.0, bs)
        frac = 1.0
    for _ in range(args.warmup):
        step()
    ms = []
    for _ in range(args.steps):
        ev.flush_l2(256 << 20)
        ev.event_record(0)
        step()
        ev.event_record(1)
        ms.append(ev.event_elapsed(0, 1))
    t = float(np.median(ms))
    return {"metric": "d-shell OCA Sigma(tau) evals/s (FP64 plain)", "value": 1000.0 / t / frac, "unit": "evals/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "dshell_5orb_beta20_L200_eps1e-8_OCA", "r": int(len(rf)),
                                            "flat_index_stride": stride, "l2": "flushed (256 MB write) before each step"},
            "items_full": int(items), "tflops": flops * frac / (t * 1e-3) / 1e12}


def run_reference(args, rank):
    """--impl reference: the CPU restatement of the reference's path (oracle) on the host cores.  One step is
    a bounded random sample of the benchmark evaluation; its time is extrapolated to the full evaluation."""
    if rank != 0:
        return
    per_step = args.cpu_seconds / max(args.steps, 1)
    for w in range(args.warmup):
        cpu_sigma_sample(min(per_step, 2.0) / 2, seed=100 + w)
    vals, walls = [], []
    sample = ""
    cores = 0
    for k in range(args.steps):
        v, wall, cores, sample = cpu_sigma_sample(per_step, seed=200 + k)
        vals.append(v)
        walls.append(wall)
    v = float(np.median(vals))
    v1, _, _, _ = cpu_sigma_sample(min(per_step, 4.0), nthreads=1, seed=300)
    name, usable = cpu_model()
    out = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": 1000.0 * float(np.mean(walls)), "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
           "dtype": "c128", "data": "synthetic", "impl": "reference",
           "config": {"workload": CONFIG_NAME, "l2": "inputs < L2; CPU run",
                      "step": "one bounded random sample of the evaluation; value = 1 / (sample time extrapolated to all flat indices)"},
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample, "value_1thread": v1,
                            "cpu_model": name, "host_cpus": usable},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.dshell:
        if rank == 0:
            print(json.dumps(run_dshell(args)), flush=True)
        return
    if args.serving:
        if rank == 0:
            print(json.dumps(run_serving(args, batched=True)), flush=True)
            print(json.dumps(run_serving(args, batched=False)), flush=True)
        return
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from xca_b200.block_sparse import BlockOpSymQuartet, DiagramEvaluator
    m, G = build_model()
    Fq = BlockOpSymQuartet(m.labels, m.F_index, m.F_blocks, m.Fd_index, m.Fd_blocks, m.dims)
    ev = DiagramEvaluator.from_arrays(m.beta, m.lam, m.eps, m.rf, m.it, m.hyb_poles, m.hyb_coeffs, Fq, device=local)
    topos = topologies()
    dev = torch.device("cuda", local)
    greal = np.concatenate([g.real.ravel() for g in G])
    G_t = torch.tensor(greal, dtype=torch.float64, device=dev)
    S_t = torch.zeros(ev.slab, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    from xca_b200.distributed import self_energy_sharded

    def allreduce():
        dist.all_reduce(S_t)
        torch.cuda.synchronize()

    def step():
        self_energy_sharded(ev, G_t.data_ptr(), S_t.data_ptr(), topos, rank, world, allreduce if world > 1 else None)

    tuning = None
    if world == 1 and not args.no_tune:
        # launch shapes of the panel kernel for this workload (xca_b200.autotune), before the warm-up steps
        from xca_b200 import autotune
        setting, table = autotune.tune_sigma(ev, G_t.data_ptr(), S_t.data_ptr(), [(t, f) for _, t, f in topos], reps=1,
                                             params=["unit_batches"])
        tuning = {"setting": setting, "sweep_ms": [[n, v, round(ms, 3)] for n, v, ms in table[1:]],
                  "default_ms": round(table[0][2], 3)}
    for _ in range(args.warmup):
        step()
    ev.synchronize()
    # algorithmic work of one step
    alg_flops, items = 0.0, 0
    for _, t, _ in topos:
        f, n = ev.self_energy_flops(G, t)
        alg_flops += f
        items += n
    launches0 = ev.kernel_launches()
    clocks = ClockSampler(local)
    ev.profile(True)
    ev.profile(True)  # reset counters
    step_ms = []
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    for _ in range(args.steps):
        ev.flush_l2(256 << 20)  # 256 MiB write: evicts the 126 MB L2 between timed steps
        ev.event_record(0)
        step()
        ev.event_record(1)
        step_ms.append(ev.event_elapsed(0, 1))
    ev.synchronize()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    sigma_ms, sigma_launches = ev.profile(False)
    clk = clocks.stop()
    launches = ev.kernel_launches() - launches0 - args.steps  # minus the L2 flushes
    t_step = float(np.sum(step_ms)) / args.steps
    if dist is not None:
        tt = torch.tensor([t_step], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_step = float(tt.item())
    value = 1000.0 / t_step

    # end to end through the public host API: host G in, host Sigma out, every step (rank 0 only)
    e2e = None
    if rank == 0 and not args.no_e2e:
        def host_eval():
            acc = [np.zeros_like(g) for g in G]
            for _, t, fac in topos:
                part = ev.compute_self_energy(G, t)
                for b in range(len(acc)):
                    acc[b] += fac * part[b]
            return acc
        host_eval()
        t0 = time.perf_counter()
        ne = max(1, min(args.steps, 3))
        for _ in range(ne):
            host_eval()
        te = (time.perf_counter() - t0) / ne
        e2e = {"value": 1.0 / te, "unit": UNIT, "h2d_bytes_per_step": int(len(topos) * ev.slab * 8),
               "d2h_bytes_per_step": int(len(topos) * ev.slab * 8)}

    peak_fma = ev.fp64_fma_peak()
    peak_mma = ev.fp64_mma_peak()
    peak = max(peak_fma, peak_mma)
    kernel_s = sigma_ms * 1e-3 / max(args.steps, 1)
    achieved = alg_flops / world / kernel_s / 1e12 if kernel_s > 0 else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_object(args.cpu_seconds)
    variants = None
    if rank == 0 and world == 1 and not args.no_variants:
        variants = precision_variants(m, G, local)
    serving = None
    if rank == 0 and world == 1 and not args.no_serving:
        serving = {"batched": run_serving(args, batched=True), "threads": run_serving(args, batched=False)}
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": t_step, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
               "data": "synthetic",
               "config": {"workload": CONFIG_NAME, "r": int(ev.r), "poles": int(ev.p), "items_per_step": int(items),
                          "alg_gflop_per_step": alg_flops / 1e9, "l2": "flushed (256 MiB write) before every timed step"},
               "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                            "frac": (achieved / peak) if achieved else None, "traffic": None,
                            "kernel": "sigma_panel_kernel",
                            "peak_source": "max of the FP64 FMA (xca_fp64_fma_probe) and FP64 tensor-core MMA "
                                           "(xca_fp64_mma_probe) throughputs measured on this GPU",
                            "peak_fp64_fma": peak_fma, "peak_fp64_mma": peak_mma,
                            "kernel_ms_per_step": sigma_ms / max(args.steps, 1), "launches_per_step": sigma_launches / max(args.steps, 1)},
               "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "clocks": clk,
               "tuning": tuning, "variants": variants, "serving": serving}
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
