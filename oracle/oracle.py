"""Oracle (test infrastructure only): ctypes front end of the CPU restatement in ``xca_oracle.cpp``
plus a numpy restatement of the reference's Python solve loop.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py`` use this module, as the checker or the timed CPU reference; the product never imports it.

Layout conventions (shared with the product's C-ABI):

* a block Green's function is a list of ``(r, d_b, d_b)`` complex arrays, one per Fock-space block;
* an operator set ``s`` is ``(index[s, b], blocks[s][b])`` with ``blocks[s][b]`` of shape
  ``(q_s, d_index, d_b)`` (``BlockOpSymSet``, ``c++/triqs_xca/block_sparse.hpp:181-200``).
"""

import ctypes
import math
import os

import numpy as np

from . import dlr_ref

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: run `make -C {_HERE}`")
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        D = ctypes.c_double
        I = ctypes.c_int
        LG = ctypes.c_long
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        lp = ctypes.POINTER(ctypes.c_long)
        L.ora_last_error.restype = ctypes.c_char_p
        L.ora_dlr_new.restype = P
        L.ora_dlr_new.argtypes = [I, dp, dp]
        L.ora_dlr_free.argtypes = [P]
        for name in ("ora_vals2coefs", "ora_coefs2vals", "ora_reflect"):
            getattr(L, name).argtypes = [P, LG, dp, dp]
        L.ora_coefs2eval.argtypes = [P, LG, dp, D, dp]
        L.ora_convolve.argtypes = [P, D, I, I, I, dp, dp, I, dp]
        L.ora_convmat.argtypes = [P, D, I, dp, I, dp]
        L.ora_dyson_solve.argtypes = [P, D, I, dp, dp, D, dp]
        L.ora_dyson_solve_op.argtypes = [P, D, I, dp, dp, D, dp, dp]
        L.ora_eval_new.restype = P
        L.ora_eval_new.argtypes = [P, D, I, dp, dp, I, lp, I, ip, ip, dp, ip, dp]
        L.ora_eval_free.argtypes = [P]
        L.ora_num_sigma_backbones.restype = LG
        L.ora_num_sigma_backbones.argtypes = [P, I, ip]
        L.ora_num_spgf_backbones.restype = LG
        L.ora_num_spgf_backbones.argtypes = [P, I, ip]
        L.ora_sigma.argtypes = [P, dp, I, ip, lp, LG, I, dp, lp, dp]
        L.ora_sigma_ordered.argtypes = [P, dp, I, ip, LG, I, dp, lp]
        L.ora_sigma_list_ordered.argtypes = [P, dp, I, ip, lp, LG, I, dp]
        L.ora_items.restype = LG
        L.ora_items.argtypes = [P, dp, I, ip, LG, LG, lp, LG]
        L.ora_spgf.argtypes = [P, dp, I, ip, lp, LG, I, dp]
        L.ora_hyb_values.argtypes = [P, dp, dp]
        L.ora_correlator.argtypes = [P, dp, I, ip, lp, LG, I, I, ip, dp, I, ip, dp, dp]
        L.ora_expectation.argtypes = [P, I, ip, dp, ip, dp, dp]
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _lp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_long))


def _c(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().ora_last_error().decode())


class Dlr:
    """cppdlr ``imtime_ops`` restated (third-party; call sites listed in ``xca_oracle.cpp``)."""

    def __init__(self, lam, eps, rf=None, it=None):
        self.lam = lam
        self.eps = eps
        self.rf = np.ascontiguousarray(dlr_ref.build_dlr_rf(lam, eps) if rf is None else rf, dtype=float)
        self.it = np.ascontiguousarray(dlr_ref.build_dlr_it(lam, self.rf) if it is None else it, dtype=float)
        self.r = len(self.rf)
        self._h = lib().ora_dlr_new(self.r, _dp(self.rf), _dp(self.it))

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.ora_dlr_free(self._h)
            self._h = None

    def tau(self, beta):
        return beta * dlr_ref.rel2abs(self.it)

    def _map(self, fn, g):
        g = _c(g)
        out = np.empty_like(g)
        _check(getattr(lib(), fn)(self._h, g.size // self.r, _dp(g), _dp(out)))
        return out

    def vals2coefs(self, g):
        return self._map("ora_vals2coefs", g)

    def coefs2vals(self, g):
        return self._map("ora_coefs2vals", g)

    def reflect(self, g):
        return self._map("ora_reflect", g)

    def coefs2eval(self, gc, t):
        gc = _c(gc)
        out = np.empty(gc.shape[1:], dtype=np.complex128)
        _check(lib().ora_coefs2eval(self._h, gc.size // self.r, _dp(gc), float(t), _dp(out)))
        return out

    def convolve(self, beta, fc, gc, time_order=False):
        fc = _c(fc)
        gc = _c(gc)
        a, b = fc.shape[1:]
        b2, c = gc.shape[1:]
        assert b == b2
        out = np.empty((self.r, a, c), dtype=np.complex128)
        _check(lib().ora_convolve(self._h, beta, a, b, c, _dp(fc), _dp(gc), int(bool(time_order)), _dp(out)))
        return out

    def convmat(self, beta, fc, time_order=True):
        fc = _c(fc)
        n = fc.shape[1]
        out = np.empty((self.r * n, self.r * n), dtype=np.complex128)
        _check(lib().ora_convmat(self._h, beta, n, _dp(fc), int(bool(time_order)), _dp(out)))
        return out

    def dyson_solve(self, beta, g0, sig, eta, op=None):
        """``dyson_it_ppsc(beta, itops, g0).solve(sig, eta)`` (``c++/triqs_xca/dlr_dyson_ppsc.hpp:135-168``), or with
        ``op`` (n x n) ``solve_with_op(sig, eta, op)`` (``dlr_dyson_ppsc.hpp:188-216``)."""
        g0 = _c(g0)
        sig = _c(sig)
        n = g0.shape[1]
        out = np.empty_like(g0)
        if op is None:
            _check(lib().ora_dyson_solve(self._h, beta, n, _dp(g0), _dp(sig), float(eta), _dp(out)))
        else:
            o = _c(op)
            assert o.shape == (n, n)
            _check(lib().ora_dyson_solve_op(self._h, beta, n, _dp(g0), _dp(sig), float(eta), _dp(o), _dp(out)))
        return out


def pack_ops(dims, index, blocks):
    """Pack operator slabs of every set in (set, block column) order, skipping absent columns."""
    index = np.ascontiguousarray(index, dtype=np.int32)
    parts = []
    for s in range(index.shape[0]):
        for b in range(index.shape[1]):
            if index[s, b] >= 0:
                blk = np.asarray(blocks[s][b])
                assert blk.shape[1:] == (dims[index[s, b]], dims[b]), (s, b, blk.shape)
                parts.append(_c(blk).ravel())
    data = np.concatenate(parts) if parts else np.zeros(1, np.complex128)
    return index, np.ascontiguousarray(data)


class Evaluator:
    """TRIQS-free ``DiagramEvaluator(beta, Lambda, eps, hyb_poles, hyb_coeffs, Fq)`` restated
    (``c++/triqs_xca/block_sparse_backbone.cpp:63-85``)."""

    def __init__(self, dlr, beta, hyb_poles, hyb_coeffs, dims, sym_set_labels, F_index, F_blocks, Fd_index, Fd_blocks):
        self.dlr = dlr
        self.beta = float(beta)
        self.dims = np.ascontiguousarray(dims, dtype=np.int32)
        self.labels = np.ascontiguousarray(sym_set_labels, dtype=np.int64)
        self.n = len(self.labels)
        self.poles = np.ascontiguousarray(hyb_poles, dtype=float)
        self.coeffs = _c(hyb_coeffs)
        self.p = len(self.poles)
        assert self.coeffs.shape == (self.p, self.n, self.n)
        self._fi, self._fd = pack_ops(self.dims, F_index, F_blocks)
        self._gi, self._gd = pack_ops(self.dims, Fd_index, Fd_blocks)
        self._h = lib().ora_eval_new(dlr._h, self.beta, self.p, _dp(self.poles), _dp(self.coeffs), self.n, _lp(self.labels),
                                     len(self.dims), _ip(self.dims), _ip(self._fi), _dp(self._fd), _ip(self._gi), _dp(self._gd))
        if not self._h:
            raise ValueError(lib().ora_last_error().decode())
        self.r = dlr.r

    @classmethod
    def from_fixture(cls, path):
        """(Dlr, Evaluator, G) of a model written by ``oracle/make_model_fixture.py`` (packed operator arrays)."""
        z = np.load(path)
        dlr = Dlr(float(z["lam"]), float(z["eps"]), rf=z["rf"], it=z["it"])
        self = cls.__new__(cls)
        self.dlr = dlr
        self.beta = float(z["beta"])
        self.dims = np.ascontiguousarray(z["dims"], dtype=np.int32)
        self.labels = np.ascontiguousarray(z["labels"], dtype=np.int64)
        self.n = len(self.labels)
        self.poles = np.ascontiguousarray(z["hyb_poles"], dtype=float)
        self.coeffs = _c(z["hyb_coeffs"])
        self.p = len(self.poles)
        self._fi = np.ascontiguousarray(z["F_index"], dtype=np.int32)
        self._fd = _c(z["F_data"])
        self._gi = np.ascontiguousarray(z["Fd_index"], dtype=np.int32)
        self._gd = _c(z["Fd_data"])
        self._h = lib().ora_eval_new(dlr._h, self.beta, self.p, _dp(self.poles), _dp(self.coeffs), self.n, _lp(self.labels),
                                     len(self.dims), _ip(self.dims), _ip(self._fi), _dp(self._fd), _ip(self._gi), _dp(self._gd))
        if not self._h:
            raise ValueError(lib().ora_last_error().decode())
        self.r = dlr.r
        return dlr, self, self.unpack(_c(z["G"]))

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.ora_eval_free(self._h)
            self._h = None

    def pack(self, G):
        return np.ascontiguousarray(np.concatenate([_c(g).ravel() for g in G]))

    def unpack(self, flat):
        out, off = [], 0
        for d in self.dims:
            sz = self.r * d * d
            out.append(flat[off:off + sz].reshape(self.r, d, d).copy())
            off += sz
        return out

    def num_self_energy_backbones(self, topology):
        t = np.ascontiguousarray(topology, dtype=np.int32)
        return lib().ora_num_sigma_backbones(self._h, t.shape[0], _ip(t))

    def num_single_ptcle_gf_backbones(self, topology):
        t = np.ascontiguousarray(topology, dtype=np.int32)
        return lib().ora_num_spgf_backbones(self._h, t.shape[0], _ip(t))

    def compute_self_energy(self, G, topology, f_ix=None, nthreads=0, stats=None):
        t = np.ascontiguousarray(topology, dtype=np.int32)
        g = self.pack(G)
        out = np.empty_like(g)
        items = np.zeros(1, np.int64)
        flops = np.zeros(1, float)
        if f_ix is None:
            fix_p, nfix = None, 0
        else:
            fix = np.ascontiguousarray(np.atleast_1d(f_ix), dtype=np.int64)
            fix_p, nfix = _lp(fix), len(fix)
        _check(lib().ora_sigma(self._h, _dp(g), t.shape[0], _ip(t), fix_p, nfix, int(nthreads), _dp(out), _lp(items), _dp(flops)))
        if stats is not None:
            stats["items"] = stats.get("items", 0) + int(items[0])
            stats["flops"] = stats.get("flops", 0.0) + float(flops[0])
        return self.unpack(out)

    def compute_self_energy_ordered(self, G, topology, unit=64, nthreads=0):
        """``compute_self_energy(G, topology)`` with the additions into Sigma in the fixed order of the
        device's ordered mode (path classes in order, runs of ``unit`` pole tuples, items in order)."""
        t = np.ascontiguousarray(topology, dtype=np.int32)
        g = self.pack(G)
        out = np.empty_like(g)
        items = np.zeros(1, np.int64)
        _check(lib().ora_sigma_ordered(self._h, _dp(g), t.shape[0], _ip(t), int(unit), int(nthreads), _dp(out), _lp(items)))
        return self.unpack(out)

    def compute_self_energy_list_ordered(self, G, topology, f_ix, nthreads=0):
        """``compute_self_energy(G, topology, f_ix_vec)`` with the additions into Sigma in list order (the
        order of the device's ordered mode for a flat-index list); the items are evaluated in parallel."""
        t = np.ascontiguousarray(topology, dtype=np.int32)
        g = self.pack(G)
        out = np.empty_like(g)
        fix = np.ascontiguousarray(np.atleast_1d(f_ix), dtype=np.int64)
        _check(lib().ora_sigma_list_ordered(self._h, _dp(g), t.shape[0], _ip(t), _lp(fix), len(fix), int(nthreads), _dp(out)))
        return self.unpack(out)

    def item_list(self, G, topology, f0=0, f1=None):
        t = np.ascontiguousarray(topology, dtype=np.int32)
        m = t.shape[0]
        if f1 is None:
            f1 = self.num_self_energy_backbones(t)
        g = self.pack(G)
        width = 3 + 2 * m - 1
        n = lib().ora_items(self._h, _dp(g), m, _ip(t), f0, f1, None, 0)
        out = np.zeros((max(n, 1), width), np.int64)
        lib().ora_items(self._h, _dp(g), m, _ip(t), f0, f1, _lp(out), n)
        return out[:n]

    def compute_single_ptcle_gf(self, G, topology, f_ix=None, nthreads=0):
        t = np.ascontiguousarray(topology, dtype=np.int32)
        g = self.pack(G)
        out = np.zeros((self.r, self.n, self.n), dtype=np.complex128)
        if f_ix is None:
            fix_p, nfix = None, 0
        else:
            fix = np.ascontiguousarray(np.atleast_1d(f_ix), dtype=np.int64)
            fix_p, nfix = _lp(fix), len(fix)
        _check(lib().ora_spgf(self._h, _dp(g), t.shape[0], _ip(t), fix_p, nfix, int(nthreads), _dp(out)))
        return out

    def compute_one_time_correlator(self, G, ops_tau, ops_0, topology, f_ix=None, nthreads=0):
        """``compute_one_time_correlator`` (``c++/triqs_xca/block_sparse_backbone.cpp:843-866``) with block operators
        ``(index[nb], blocks[nb])`` (blocks[b] of shape (d_index[b], d_b), None where index[b] == -1)."""
        t = np.ascontiguousarray(topology, dtype=np.int32)
        g = self.pack(G)

        def packed(ops):
            idx = np.ascontiguousarray(np.concatenate([np.asarray(i, np.int32) for i, _ in ops]), dtype=np.int32)
            parts = [_c(blk).ravel() for i, blks in ops for b, blk in zip(i, blks) if b >= 0]
            data = np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros(1, np.complex128))
            return idx, data

        mi, md = packed(ops_tau)
        ki, kd = packed(ops_0)
        out = np.zeros((self.r, len(ops_tau), len(ops_0)), np.complex128)
        if f_ix is None:
            fix_p, nfix = None, 0
        else:
            fix = np.ascontiguousarray(np.atleast_1d(f_ix), dtype=np.int64)
            fix_p, nfix = _lp(fix), len(fix)
        _check(lib().ora_correlator(self._h, _dp(g), t.shape[0], _ip(t), fix_p, nfix, int(nthreads), len(ops_tau), _ip(mi), _dp(md),
                                    len(ops_0), _ip(ki), _dp(kd), _dp(out)))
        return out

    def hyb_values(self):
        v = np.zeros((self.r, self.n, self.n), np.complex128)
        vr = np.zeros_like(v)
        lib().ora_hyb_values(self._h, _dp(v), _dp(vr))
        return v, vr


# ------------------------------------------------------------------ restated Python solve loop
def connected_pairings(order):
    """``diag.all_connected_pairings`` (``python/triqs_xca/diag.py:48-71, 110-127``) restated."""

    def rec(parity, partial, unpaired):
        if not unpaired:
            yield parity, partial
            return
        for i in range(1, len(unpaired)):
            pair = (unpaired[0], unpaired[i])
            rest = [x for k, x in enumerate(unpaired) if k not in (0, i)]
            yield from rec(-parity if i % 2 == 0 else parity, partial + [pair], rest)

    def crossing(p1, p2):
        return (p1[0] < p2[0] < p1[1] < p2[1]) or (p2[0] < p1[0] < p2[1] < p1[1])

    for parity, pairing in rec(1, [], list(range(2 * order))):
        stack = [p for p in pairing if (p[0] <= 0) != (p[1] <= 0)]
        rest = [p for p in pairing if (p[0] <= 0) == (p[1] <= 0)]
        while stack:
            pc = stack.pop(0)
            for idx in reversed(range(len(rest))):
                if crossing(pc, rest[idx]):
                    stack.append(rest.pop(idx))
        if not rest:
            yield parity, pairing


def sigma_total(ev, G, max_order, nthreads=0, stats=None, orders=None, ordered=False):
    """``BlockSparseSolver.eval_pseudo_particle_self_energy`` (``block_sparse_solver.py:597-640``):
    Sigma = sum_order sum_topology (-1)^order * parity * (-1)^(order+1) * compute_self_energy.
    ``ordered``: each topology summed in the fixed order of the device's ordered mode."""
    Sig = [np.zeros_like(_c(g)) for g in G]
    for order in (orders if orders is not None else range(1, max_order + 1)):
        for sign, topo in connected_pairings(order):
            if ordered:
                part = ev.compute_self_energy_ordered(G, np.array(topo, np.int32), nthreads=nthreads)
            else:
                part = ev.compute_self_energy(G, np.array(topo, np.int32), nthreads=nthreads, stats=stats)
            fac = (-1) ** order * sign * (-1) ** (order + 1)
            for b in range(len(Sig)):
                Sig[b] += fac * part[b]
    return Sig


def spgf_total(ev, G, max_order, nthreads=0):
    """``BlockSparseSolver.eval_single_particle_greens_function`` (``block_sparse_solver.py:657-698``)."""
    g = np.zeros((ev.r, ev.n, ev.n), np.complex128)
    for order in range(1, max_order + 1):
        for sign, topo in connected_pairings(order):
            g += (-1) ** order * sign * ev.compute_single_ptcle_gf(G, np.array(topo, np.int32), nthreads=nthreads)
    return g


def trace_beta(dlr, G):
    """``trace`` (``c++/triqs_xca/block_sparse.cpp:852-861``): sum_b Tr G_b(beta) by DLR evaluation, the
    diagonal and the blocks summed one after another from zero (``nda::trace`` and ``trace +=``)."""
    tot = 0.0 + 0.0j
    for g in G:
        gb = dlr.coefs2eval(dlr.vals2coefs(g), 1.0)
        tr = 0.0 + 0.0j
        for x in range(gb.shape[0]):
            tr += complex(gb[x, x])
        tot += tr
    return tot


def convolve_ppsc(dlr, beta, G1, G2):
    """``convolve_ppsc`` (``c++/triqs_xca/block_sparse.cpp:832-850``): per block the time-ordered convolution."""
    return [dlr.convolve(beta, dlr.vals2coefs(a), dlr.vals2coefs(b), time_order=True) for a, b in zip(G1, G2)]


def expectation_value(dlr, G, op_index, op_blocks):
    """``expectation_value`` (``c++/triqs_xca/block_sparse.cpp:797-818``) of a block-diagonal operator given as
    (op_index[nb], op_blocks[nb]) in the Fock basis."""
    dims = np.ascontiguousarray([g.shape[1] for g in G], dtype=np.int32)
    idx = np.ascontiguousarray(op_index, dtype=np.int32)
    parts = [_c(o).ravel() for i, o in zip(idx, op_blocks) if i >= 0]
    data = np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros(1, np.complex128))
    g = np.ascontiguousarray(np.concatenate([_c(x).ravel() for x in G]))
    out = np.zeros(2)
    _check(lib().ora_expectation(dlr._h, len(G), _ip(dims), _dp(g), _ip(idx), _dp(data), _dp(out)))
    return complex(out[0], out[1])


def solve_dyson(dlr, beta, G0, Sig, eta):
    """``solve_dyson`` (``block_sparse_solver.py:572-590``): per-block Dyson solve, then hermitize."""
    out = []
    for g0, s in zip(G0, Sig):
        g = dlr.dyson_solve(beta, g0, s, eta)
        out.append(0.5 * (g + np.conj(np.transpose(g, (0, 2, 1)))))
    return out


def normalize(dlr, beta, G, eta):
    """``normalize_pseudo_particle_gf`` (``block_sparse_solver.py:427-449``)."""
    Z = -trace_beta(dlr, G).real
    deta = math.log(abs(Z)) / beta
    tabs = dlr_ref.rel2abs(dlr.it)
    fac = np.array([math.exp(-((beta * float(t)) * deta)) for t in tabs])
    return [g * fac[:, None, None] for g in G], eta + deta


def z_alpha_minus_one_and_derivatives(dlr, beta, G0, Sig, alpha, eta):
    """``Z_alpha_minus_one_and_derivative_and_2nd_derivative`` (``block_sparse_solver.py:800-816``)."""
    Ga = solve_dyson(dlr, beta, G0, Sig if alpha == 1.0 else [alpha * s for s in Sig], eta)
    Za = -trace_beta(dlr, Ga).real
    G2 = convolve_ppsc(dlr, beta, Ga, Ga)
    dZ = -trace_beta(dlr, G2).real
    d2Z = -2 * trace_beta(dlr, convolve_ppsc(dlr, beta, G2, Ga)).real
    return Za - 1, dZ, d2Z


def deta_dalpha(dlr, beta, G0, Sig, alpha, eta):
    """``deta_dalpha`` (``block_sparse_solver.py:819-838``): -Tr[G_a * Sigma * G_a] / Tr[G_a * G_a]."""
    Ga = solve_dyson(dlr, beta, G0, Sig if alpha == 1.0 else [alpha * s for s in Sig], eta)
    tr_gg = -trace_beta(dlr, convolve_ppsc(dlr, beta, Ga, Ga))
    tr_gsg = -trace_beta(dlr, convolve_ppsc(dlr, beta, Ga, convolve_ppsc(dlr, beta, Sig, Ga)))
    return -tr_gsg / tr_gg


def chempot_newton(dlr, beta, G0, Sig, eta, **kwargs):
    """``solve_ppsc_chempot_newton`` (``block_sparse_solver.py:1000-1029``): Halley's method on Z(eta) - 1."""
    from scipy.optimize import root_scalar
    sol = root_scalar(lambda e: z_alpha_minus_one_and_derivatives(dlr, beta, G0, Sig, 1.0, e), x0=eta, fprime=True, fprime2=True,
                      method="halley", **kwargs)
    return float(sol.root)


def chempot_adiabatic_ode(dlr, beta, G0, Sig, tol, method="RK23"):
    """``solve_ppsc_chempot_adiabatic_ode`` (``block_sparse_solver.py:896-923``)."""
    from scipy.integrate import solve_ivp
    sol = solve_ivp(lambda t, y: deta_dalpha(dlr, beta, G0, Sig, t, y[0]).real, (0.0, 1.0), np.array([0.0]), atol=tol, method=method,
                    dense_output=True)
    return float(sol.y[0, -1])


def solve(dlr, ev, beta, G0, max_order, tol, maxiter, mix=1.0, spgf_max_order=None, nthreads=0, verbose=False, ordered=False,
          G_init=None, eta_init=0.0, normalization="classic", eps=None):
    """``BlockSparseSolver.solve`` (``block_sparse_solver.py:240-355``) with the 'classic', 'root', 'ode+classic'
    or 'ode+root' normalization (``eps`` = the DLR accuracy, which sets the root / ODE tolerances).
    ``ordered``: Sigma summed in the fixed order of the device's ordered mode.  ``G_init``/``eta_init``:
    start from a previous solution (the reference's solver keeps self.G and self.eta between solves).

    Returns (G, Sigma, eta, g_spgf, n_iter, diff_G)."""
    G = [g.copy() for g in (G0 if G_init is None else G_init)]
    eta = eta_init
    it = 0
    diff = np.inf
    Sig = None
    for it in range(1, maxiter + 1):
        Sig = sigma_total(ev, G, max_order, nthreads=nthreads, ordered=ordered)
        if normalization in ("ode+classic", "ode+root"):
            eta = chempot_adiabatic_ode(dlr, beta, G0, Sig, tol=100 * eps)
        if normalization in ("root", "ode+root"):
            eta = chempot_newton(dlr, beta, G0, Sig, eta, xtol=10 * eps)
        Gn = solve_dyson(dlr, beta, G0, Sig, eta)
        if normalization in ("classic", "ode+classic"):
            Gn, eta = normalize(dlr, beta, Gn, eta)
        diff = max(np.max(np.abs(a - b)) for a, b in zip(Gn, G))
        if verbose:
            print(f"iter = {it}, diff_G = {diff:2.2E}, eta = {eta:2.2E}")
        if diff < tol:
            break
        G = [mix * a + (1 - mix) * b for a, b in zip(Gn, G)]
    g = spgf_total(ev, G, spgf_max_order or max_order, nthreads=nthreads)
    return G, Sig, eta, g, it, diff
