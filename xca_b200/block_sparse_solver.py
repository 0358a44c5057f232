"""Self-consistent pseudo-particle solve with the reference's Python interface
(``BlockSparseSolver``, ``python/triqs_xca/block_sparse_solver.py:36-355``), device resident.

The pseudo-particle propagator, self-energy and Dyson state stay in GPU memory across iterations; each
iteration launches the Sigma evaluation of every order and topology (accumulated with the reference's
signs, :597-640), the Dyson solve with hermitization (:572-590), the 'classic' normalisation
(:427-449) and the convergence test (:338, :1379-1380); only three scalars per iteration (Z, deta,
diff_G) come back to the host.

TRIQS is not available here, so the local problem is given as an ``xca_b200.atom_diag.AtomDiag`` and the
hybridization as a dense ``(r, n, n)`` array of Delta(tau) on the DLR nodes (``Delta_tau``); with
``hyb_comp=False`` the solver fits it on the DLR poles exactly as the reference does (:171-176), with
``hyb_comp=True`` it compresses it to a few poles (``xca_b200.hyb_fit``, in place of adapol, :151-169).
"""

import time

import numpy as np

from . import diag
from .atom_diag import atomic_pseudo_particle_greens_function
from .block_sparse import BlockOpSymQuartet, DiagramEvaluator
from .hyb_fit import compress_hybridization_cached
from .models import dlr_fit_hybridization, rel2abs
from .pycppdlr import MeshDLRImTime

# device buffer slots of the solver's slabs (the evaluator's buffers 0..9 stay free for callers)
_SLOTS = {"G": 10, "Gn": 11, "S": 12, "Sa": 13, "Gt": 14, "W1": 15, "W2": 16}

NORMALIZATIONS = ("classic", "root", "ode+classic", "ode+root")


class BlockSparseSolver:
    def __init__(self, atom_diag, beta, w_max, eps, device=0, verbose=False, precision="fp64", mixed_tol=1e-5):
        """``precision``: 'fp64' (Sigma items summed with atomics), 'fp64_ordered' (fixed summation order: the
        solve is reproducible bit for bit) or 'mixed': the early iterations evaluate the NCA Sigma only, with
        FP32 block products (the evaluator's 'fp32' mode), until diff_G falls below ``mixed_tol`` or makes no
        new low for three iterations; then the full order in FP64 until convergence, which is only accepted in that phase.  FP32
        is confined to NCA because every higher diagram passes through the DLR convolution of an edge, whose
        closed form (K^-1 with cond ~ 1/eps, then sums over W_lk = K(0, om_k) / (om_k - om_l) that cancel)
        loses all FP32 digits.  The Dyson solve, the normalisation and G(tau) are FP64 throughout."""
        if precision not in ("fp64", "fp64_ordered", "mixed"):
            raise ValueError(f"precision must be 'fp64', 'fp64_ordered' or 'mixed', got {precision!r}")
        self.ad = atom_diag
        self.precision = precision
        self.mixed_tol = float(mixed_tol)
        self.beta = float(beta)
        self.w_max = float(w_max)
        self.eps = float(eps)
        self.device = device
        self.verbose = verbose
        self.mesh_tau = MeshDLRImTime(beta=self.beta, statistic="Fermion", w_max=self.w_max, eps=self.eps)
        self.rf = self.mesh_tau.dlr_rf
        self.it = self.mesh_tau.dlr_it.it
        self.r = len(self.rf)
        self.n = atom_diag.n
        self.tau = self.beta * rel2abs(self.it)
        self.Delta_tau = np.zeros((self.r, self.n, self.n), np.complex128)
        self.G0, self.eta0 = atomic_pseudo_particle_greens_function(atom_diag, self.beta, self.tau)
        self.G = [g.copy() for g in self.G0]
        self.Sigma = [np.zeros_like(g) for g in self.G0]
        self.eta = 0.0
        self.Fq = BlockOpSymQuartet.from_atom_diag(atom_diag)
        self.d = None
        self.G_tau = None
        self.timings = {}

    # -- hybridization (fit_hybridization, block_sparse_solver.py:146-185): one pole per DLR frequency, or with
    # ``compression`` a few real poles fitted to tolerance ``tol`` (xca_b200.hyb_fit); fit_error as the reference
    def fit_hybridization(self, tol=None, compression=False):
        if compression:
            if tol is None or tol <= 0:
                raise ValueError("tol must be provided and positive when compression is enabled")
            self.hyb_poles, self.hyb_coeffs, self.hyb_fit_error = compress_hybridization_cached(self.rf, self.it, self.beta,
                                                                                                self.Delta_tau, tol)
        else:
            self.hyb_poles, self.hyb_coeffs = dlr_fit_hybridization(self.rf, self.it, self.beta, self.Delta_tau)
            self.hyb_fit_error = self.eps
        self.hyb_compression = bool(compression)

    def init_diagram_evaluator(self):
        self.d = DiagramEvaluator.from_arrays(self.beta, self.beta * self.w_max, self.eps, self.rf, self.it, self.hyb_poles,
                                              self.hyb_coeffs, self.Fq, device=self.device)
        self.d.precision_mode = "fp32" if self.precision == "mixed" else self.precision
        self.d.dyson_setup(self.G0)
        self._buf = {k: self.d.device_buffer(slot, self.d.slab) for k, slot in _SLOTS.items()}

    def _ensure_evaluator(self):
        if self.d is None:
            self.fit_hybridization()
            self.init_diagram_evaluator()

    def _upload(self, key, blocks):
        self.d.to_device(self._buf[key], np.concatenate([np.asarray(g).real.ravel() for g in blocks]))

    def _download(self, key):
        return [x.astype(np.complex128) for x in self.d.unpack(self.d.to_host(self._buf[key], self.d.slab))]

    def sigma_jobs(self, max_order):
        """Zeroes the device Sigma and returns the iteration's Sigma evaluations as jobs (evaluator, G, topology,
        scale, Sigma) of DiagramEvaluator.compute_self_energy_device_batch: every connected topology of orders
        1..max_order with the reference's signs (block_sparse_solver.py:597-640)."""
        d = self.d
        d.zero_device(self._buf["S"], d.slab)
        jobs = []
        for order in range(1, max_order + 1):
            for sign, topo in diag.all_connected_pairings(order):
                # (-1)^order * parity * (-1)^(order+1): the order loop's and the topology loop's signs
                fac = (-1) ** order * sign * (-1) ** (order + 1)
                jobs.append((d, self._buf["G"], topo, float(fac), self._buf["S"]))
        return jobs

    def _sigma_device(self, max_order):
        jobs = self.sigma_jobs(max_order)
        if self.d.precision_mode == "fp64":
            # every topology in one launch over the shared edge tables of the highest order
            DiagramEvaluator.compute_self_energy_device_batch(jobs)
        else:
            # the fixed summation order (one ordered evaluation per topology, accumulated in topology order), or
            # the FP32 products of a mixed solve's early iterations
            for _, G, topo, fac, S in jobs:
                self.d.compute_self_energy_device(G, topo, fac, S)

    def begin(self, max_order, tol=1e-4, hyb_tol=None, hyb_comp=True, normalization="classic", spgf_max_order=None):
        """The set-up of solve (block_sparse_solver.py:240-300): hybridization fit, evaluator, G on the device."""
        if normalization not in NORMALIZATIONS:
            raise NotImplementedError(f"normalization {normalization!r} is not available on the device path "
                                      f"(available: {', '.join(NORMALIZATIONS)})")
        self.normalization = normalization
        self.max_order = max_order
        self.spgf_max_order = spgf_max_order if spgf_max_order is not None else max_order
        # compression is skipped for NCA, whose backbones use no pole representation (block_sparse_solver.py:289)
        self.hyb_tol = hyb_tol if hyb_tol is not None else 0.1 * tol
        self.fit_hybridization(tol=self.hyb_tol, compression=hyb_comp and max_order > 1)
        self.init_diagram_evaluator()
        self._upload("G", self.G)

    def launch_dyson(self):
        """The Dyson solve of an iteration whose Sigma is on the device, for the 'classic' normalisation
        (queued on the evaluator's stream)."""
        self.d.dyson_solve_device(self._buf["S"], self.eta, self._buf["Gn"], hermitize=True)

    def end_iteration(self, it, tol, mix, verbose=False, dyson_launched=False, accept=True):
        """The rest of one iteration after its Sigma (block_sparse_solver.py:300-345): eta, Dyson solve,
        normalisation, diff_G; mixes G unless converged.  Returns True when diff_G < tol (never with
        ``accept`` False, as in the FP32 phase of a mixed solve)."""
        d = self.d
        normalization = self.normalization
        if normalization in ("ode+classic", "ode+root"):
            self.solve_ppsc_chempot_adiabatic_ode(tol=100 * self.eps)
        if normalization in ("root", "ode+root"):
            self.solve_ppsc_chempot_newton(xtol=10 * self.eps)
        if not dyson_launched:
            d.dyson_solve_device(self._buf["S"], self.eta, self._buf["Gn"], hermitize=True)
        if normalization in ("classic", "ode+classic"):
            Z, deta = d.normalize_device(self._buf["Gn"])
            self.eta += deta
        else:
            Z = -d.trace_device(self._buf["Gn"]).real
        self.diff_G = d.max_abs_diff_device(self._buf["Gn"], self._buf["G"])
        self.n_ppsc_iter = it
        if verbose:
            print(f"iter = {it}, diff_G = {self.diff_G:2.2E}, Z = {Z:+2.6E}, eta = {self.eta:2.2E}")
        if accept and self.diff_G < tol:
            return True
        d.axpby_device(mix, self._buf["Gn"], 1.0 - mix, self._buf["G"])
        return False

    def finish(self):
        """The end of solve: G and Sigma back to the host, the single-particle Green's function."""
        self.d.synchronize()
        self.G = self._download("G")
        self.Sigma = self._download("S")
        self.G_tau = None
        if self.spgf_max_order > 0:
            self.G_tau = self.eval_single_particle_greens_function(self.G, self.spgf_max_order)
        return self

    def solve(self, max_order, tol=1e-4, maxiter=10, mix=1.0, hyb_tol=None, hyb_comp=True, normalization="classic",
              spgf_max_order=None, verbose=None):
        """BlockSparseSolver.solve (block_sparse_solver.py:240-355), with its defaults: the hybridization is
        compressed to a few poles (hyb_comp=True, tolerance hyb_tol = 0.1 tol) for orders above NCA."""
        verbose = self.verbose if verbose is None else verbose
        self.begin(max_order, tol, hyb_tol, hyb_comp, normalization, spgf_max_order)
        t0 = time.perf_counter()
        self.n_ppsc_iter = 0
        self.n_fp32_iter = 0
        fp32_phase = self.precision == "mixed"
        best, stalled = np.inf, 0
        for it in range(1, maxiter + 1):
            self._sigma_device(1 if fp32_phase else max_order)
            done = self.end_iteration(it, tol, mix, verbose, accept=not fp32_phase)
            if fp32_phase:
                self.n_fp32_iter += 1
                if self.diff_G < best:
                    best, stalled = self.diff_G, 0
                else:
                    stalled += 1
                # below mixed_tol, three iterations without a new best, or not finite: the full order in FP64
                if self.diff_G < self.mixed_tol or stalled >= 3 or not np.isfinite(self.diff_G):
                    fp32_phase = False
                    self.d.precision_mode = "fp64"
            if done:
                break
        self.d.synchronize()
        self.timings["solve_loop_s"] = time.perf_counter() - t0
        return self.finish()

    # -- eta from Z(eta) = 1 ('root' / 'ode' normalizations, block_sparse_solver.py:744-1030).  G_alpha solves the
    # Dyson equation with alpha * Sigma (the current Sigma on the device) at eta; every Dyson solve, convolution
    # and trace runs on the device, the scalar root / ODE iteration on the host with scipy, as the reference.
    def _g_alpha(self, alpha, eta):
        d = self.d
        src = self._buf["S"]
        if alpha != 1.0:
            d.zero_device(self._buf["Sa"], d.slab)
            d.axpby_device(alpha, self._buf["S"], 0.0, self._buf["Sa"])
            src = self._buf["Sa"]
        d.dyson_solve_device(src, float(eta), self._buf["Gt"], hermitize=True)
        return self._buf["Gt"]

    def Z_alpha_minus_one_and_derivative_and_2nd_derivative(self, alpha, eta):
        """Z_alpha - 1 and its first two eta derivatives: Z = -Tr G(beta), dZ/deta = -Tr (G * G)(beta),
        d2Z/deta2 = -2 Tr ((G * G) * G)(beta) (block_sparse_solver.py:800-816)."""
        d = self.d
        G = self._g_alpha(alpha, eta)
        Za = -d.trace_device(G).real
        d.convolve_ppsc_device(G, G, self._buf["W1"])
        dZ = -d.trace_device(self._buf["W1"]).real
        d.convolve_ppsc_device(self._buf["W1"], G, self._buf["W2"])
        d2Z = -2 * d.trace_device(self._buf["W2"]).real
        return Za - 1, dZ, d2Z

    def deta_dalpha(self, alpha, eta):
        """d eta / d alpha = -Tr[G_a * Sigma * G_a] / Tr[G_a * G_a] (block_sparse_solver.py:819-838)."""
        d = self.d
        G = self._g_alpha(alpha, eta)
        d.convolve_ppsc_device(G, G, self._buf["W1"])
        tr_gg = -d.trace_device(self._buf["W1"])
        d.convolve_ppsc_device(self._buf["S"], G, self._buf["W1"])
        d.convolve_ppsc_device(G, self._buf["W1"], self._buf["W2"])
        tr_gsg = -d.trace_device(self._buf["W2"])
        return -tr_gsg / tr_gg

    def solve_ppsc_chempot_newton(self, **kwargs):
        """eta with Z(eta) = 1 by Halley's method from the current eta (solve_ppsc_chempot_newton,
        block_sparse_solver.py:1000-1029)."""
        from scipy.optimize import root_scalar
        sol = root_scalar(lambda eta: self.Z_alpha_minus_one_and_derivative_and_2nd_derivative(1.0, eta), x0=self.eta, fprime=True,
                          fprime2=True, method="halley", **kwargs)
        self.eta = float(sol.root)
        return sol

    def solve_ppsc_chempot_adiabatic_ode(self, tol=1e-9, method="RK23"):
        """eta(alpha = 1) from d eta / d alpha along alpha in [0, 1], eta(0) = 0 (solve_ppsc_chempot_adiabatic_ode,
        block_sparse_solver.py:896-923)."""
        from scipy.integrate import solve_ivp
        sol = solve_ivp(lambda t, y: self.deta_dalpha(t, y[0]).real, (0.0, 1.0), np.array([0.0]), atol=tol, method=method,
                        dense_output=True)
        self.eta = float(sol.y[0, -1])
        return sol

    # -- state I/O (__reduce_to_dict__ / __factory_from_dict__, block_sparse_solver.py:1178-1204): everything but
    # the device evaluator; h5 is not available here, so the state goes to a numpy .npz archive
    _STATE_ARRAYS = ("G", "Sigma", "G0", "Delta_tau", "hyb_poles", "hyb_coeffs", "G_tau")
    _STATE_SCALARS = ("beta", "w_max", "eps", "eta", "eta0", "n_ppsc_iter", "diff_G", "max_order", "spgf_max_order", "precision",
                      "normalization", "verbose", "hyb_tol", "hyb_fit_error", "hyb_compression", "mixed_tol", "n_fp32_iter")

    def __reduce_to_dict__(self):
        out = {"atom_diag": self.ad.to_dict()}
        for k in self._STATE_ARRAYS + self._STATE_SCALARS:
            if hasattr(self, k):
                v = getattr(self, k)
                out[k] = [np.array(g) for g in v] if isinstance(v, list) else v
        return out

    @classmethod
    def __factory_from_dict__(cls, name, d):
        from .atom_diag import AtomDiag
        ret = cls(AtomDiag.from_dict(d["atom_diag"]), d["beta"], d["w_max"], d["eps"], verbose=False,
                  precision=d.get("precision", "fp64"))
        for k in cls._STATE_ARRAYS + cls._STATE_SCALARS:
            if k in d:
                setattr(ret, k, d[k])
        return ret

    def __eq__(self, other):
        a, b = self.__reduce_to_dict__(), other.__reduce_to_dict__()
        if a.keys() != b.keys():
            return False

        def same(x, y):
            if isinstance(x, dict):
                return x.keys() == y.keys() and all(same(x[k], y[k]) for k in x)
            if isinstance(x, (list, tuple)):
                return len(x) == len(y) and all(same(u, v) for u, v in zip(x, y))
            if isinstance(x, np.ndarray) or isinstance(y, np.ndarray):
                return np.array_equal(np.asarray(x), np.asarray(y))
            return x == y

        return all(same(a[k], b[k]) for k in a)

    def save(self, path):
        """Write the solver state to ``path`` (.npz)."""
        flat = {}

        def put(prefix, v):
            if isinstance(v, dict):
                for k, x in v.items():
                    put(f"{prefix}{k}/", x)
            elif isinstance(v, list):
                flat[f"{prefix}len"] = np.array(len(v))
                for i, x in enumerate(v):
                    put(f"{prefix}{i}/", x)
            else:
                flat[prefix.rstrip("/")] = np.asarray(v) if v is not None else np.array("None")

        put("", self.__reduce_to_dict__())
        np.savez_compressed(path, **flat)

    @classmethod
    def load(cls, path):
        """Solver rebuilt from a file written by ``save``; a later ``solve`` continues from its G and eta."""
        z = np.load(path, allow_pickle=False)
        tree = {}
        for key in z.files:
            parts = key.split("/")
            node = tree
            for p in parts[:-1]:
                node = node.setdefault(p, {})
            node[parts[-1]] = z[key]

        def build(node):
            if isinstance(node, dict):
                if "len" in node and set(node) == {"len"} | {str(i) for i in range(int(node["len"]))}:
                    return [build(node[str(i)]) for i in range(int(node["len"]))]
                return {k: build(v) for k, v in node.items()}
            if node.dtype.kind == "U":
                s = str(node)
                return None if s == "None" else s
            return node.item() if node.ndim == 0 else node

        d = build(tree)
        return cls.__factory_from_dict__(cls.__name__, d)

    def eval_pseudo_particle_self_energy(self, G, max_order):
        """Sigma of orders 1..max_order for a host G (block_sparse_solver.py:597-640)."""
        self._ensure_evaluator()
        self._upload("G", G)
        self._sigma_device(max_order)
        self.d.synchronize()
        return self._download("S")

    def solve_dyson(self, Sigma, eta):
        """solve_dyson (block_sparse_solver.py:572-590): per-block Dyson solve, hermitized."""
        self._ensure_evaluator()
        self._upload("S", Sigma)
        self.d.dyson_solve_device(self._buf["S"], eta, self._buf["Gn"], hermitize=True)
        self.d.synchronize()
        return self._download("Gn")

    def eval_single_particle_greens_function(self, G, max_order):
        """Single-particle G(tau) of orders 1..max_order (block_sparse_solver.py:657-698)."""
        self._ensure_evaluator()
        g = np.zeros((self.r, self.n, self.n), np.complex128)
        for order in range(1, max_order + 1):
            for sign, topo in diag.all_connected_pairings(order):
                g += (-1) ** order * sign * self.d.compute_single_ptcle_gf(G, topo)
        return g

    def partition_function_from_ppgf(self, G):
        """Z = -Re sum_b Tr G_b(beta) (block_sparse_solver.py:482-487)."""
        self._ensure_evaluator()
        return -self.d.trace(G).real
