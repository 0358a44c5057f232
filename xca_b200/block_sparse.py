"""Python face of the device evaluator, with the reference's names
(``python/triqs_xca/block_sparse.wrap.cxx``: ``DiagramEvaluator`` and its methods,
``c++/triqs_xca/block_sparse_backbone.hpp:23-165``).

A block Green's function is passed as a list of ``(r, d_b, d_b)`` arrays, as objects with a ``.data``
attribute, or as an iterable of ``(name, g)`` pairs (the shape of a TRIQS ``BlockGf``); results come
back as a list of ``(r, d_b, d_b)`` complex arrays.  All evaluation runs in ``libxca_b200.so`` on the
GPU.
"""

import ctypes

import numpy as np

from . import _lib
from .atom_diag import AtomDiag, get_operators


class BlockOpSymQuartet:
    """Field operators grouped in symmetry sets (``c++/triqs_xca/block_sparse.hpp:270-291``): the
    F and F^dag slabs per set and block column; the barred operators are formed by the library."""

    def __init__(self, sym_set_labels, F_index, F_blocks, Fd_index, Fd_blocks, dims):
        self.sym_set_labels = np.ascontiguousarray(sym_set_labels, dtype=np.int64)
        self.F_index = np.ascontiguousarray(F_index, dtype=np.int32)
        self.F_blocks = F_blocks
        self.Fd_index = np.ascontiguousarray(Fd_index, dtype=np.int32)
        self.Fd_blocks = Fd_blocks
        self.dims = np.ascontiguousarray(dims, dtype=np.int32)

    @classmethod
    def from_atom_diag(cls, ad):
        labels, Fi, Fb, Fdi, Fdb = get_operators(ad)
        return cls(labels, Fi, Fb, Fdi, Fdb, ad.get_subspace_dims())

    def packed(self):
        def pack(index, blocks):
            parts = []
            for s in range(index.shape[0]):
                for b in range(index.shape[1]):
                    if index[s, b] >= 0:
                        parts.append(np.ascontiguousarray(blocks[s][b], dtype=np.complex128).ravel())
            data = np.concatenate(parts) if parts else np.zeros(1, np.complex128)
            return np.ascontiguousarray(data).view(np.float64)

        return pack(self.F_index, self.F_blocks), pack(self.Fd_index, self.Fd_blocks)


def _blocks_of(G):
    out = []
    for g in G:
        if isinstance(g, tuple) and len(g) == 2:
            g = g[1]
        if hasattr(g, "data"):
            g = g.data
        out.append(np.asarray(g))
    return out


class DiagramEvaluator:
    """Evaluator of the pseudo-particle self-energy backbones on one GPU.

    ``DiagramEvaluator(hyb_poles, hyb_coeffs, tau_mesh, atom_diag)`` (bsb.hpp:144-147) or
    ``DiagramEvaluator(beta, Lambda, eps, hyb_poles, hyb_coeffs, Fq)`` (bsb.hpp:158-162).
    ``device`` selects the CUDA device.
    """

    def __init__(self, *args, device=0):
        if len(args) == 4:
            hyb_poles, hyb_coeffs, mesh, ad = args
            if not isinstance(ad, AtomDiag):
                raise TypeError("atom_diag must be an xca_b200.atom_diag.AtomDiag")
            beta, lam, eps = mesh.beta, mesh.lam, mesh.eps
            rf, it = mesh.dlr_rf, mesh.dlr_it.it
            Fq = BlockOpSymQuartet.from_atom_diag(ad)
        elif len(args) == 6:
            beta, lam, eps, hyb_poles, hyb_coeffs, Fq = args
            from .pycppdlr import ImTimeOps, build_dlr_rf
            rf = build_dlr_rf(lam, eps)
            it = ImTimeOps(lam, rf).it
        else:
            raise TypeError("DiagramEvaluator(hyb_poles, hyb_coeffs, tau_mesh, atom_diag) or "
                            "DiagramEvaluator(beta, Lambda, eps, hyb_poles, hyb_coeffs, Fq)")
        self._setup(float(beta), float(lam), float(eps), np.asarray(rf, float), np.asarray(it, float),
                    hyb_poles, hyb_coeffs, Fq, device)

    @classmethod
    def from_arrays(cls, beta, lam, eps, rf, it, hyb_poles, hyb_coeffs, Fq, device=0):
        self = cls.__new__(cls)
        self._setup(float(beta), float(lam), float(eps), np.asarray(rf, float), np.asarray(it, float),
                    hyb_poles, hyb_coeffs, Fq, device)
        return self

    def _setup(self, beta, lam, eps, rf, it, hyb_poles, hyb_coeffs, Fq, device):
        L = _lib.lib()
        self._ctx = ctypes.c_void_p()
        _lib.check(L.xca_ctx_create(int(device), ctypes.byref(self._ctx)))
        self.beta = beta
        self.r = len(rf)
        self.rf = np.ascontiguousarray(rf, dtype=float)
        self.it = np.ascontiguousarray(it, dtype=float)
        poles = np.ascontiguousarray(hyb_poles, dtype=float)
        coeffs = np.ascontiguousarray(hyb_coeffs, dtype=np.complex128)
        n = len(Fq.sym_set_labels)
        if coeffs.shape != (len(poles), n, n):
            raise ValueError(f"DiagramEvaluator: hyb_coeffs must have shape (p, n, n) with p = {len(poles)} and n = {n}, "
                             f"got {coeffs.shape}")
        self.n = n
        self.q = int(Fq.sym_set_labels.max()) + 1
        self.dims = np.ascontiguousarray(Fq.dims, dtype=np.int32)
        self.Nmax = int(self.dims.max())
        self.p = len(poles)
        self.Fq = Fq
        fdata, fddata = Fq.packed()
        self._keep = (poles, coeffs, fdata, fddata)
        _lib.check(L.xca_evaluator_setup(self._ctx, beta, lam, eps, self.r, _lib.as_dp(self.rf), _lib.as_dp(self.it),
                                         self.p, _lib.as_dp(poles), _lib.as_dp(coeffs.view(np.float64)), n,
                                         _lib.as_lp(Fq.sym_set_labels), len(self.dims), _lib.as_ip(self.dims),
                                         _lib.as_ip(Fq.F_index), _lib.as_dp(fdata), _lib.as_ip(Fq.Fd_index), _lib.as_dp(fddata)))
        nd = ctypes.c_long()
        rr = ctypes.c_int()
        _lib.check(L.xca_slab_info(self._ctx, ctypes.byref(nd), ctypes.byref(rr)))
        self.slab = nd.value

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx and _lib._lib is not None:
            _lib._lib.xca_ctx_destroy(ctx)
            self._ctx = None

    # ---------------------------------------------------------------- packing
    def pack(self, G):
        blocks = _blocks_of(G)
        if len(blocks) != len(self.dims):
            raise ValueError(f"expected {len(self.dims)} blocks, got {len(blocks)}")
        for g, d in zip(blocks, self.dims):
            if g.shape != (self.r, d, d):
                raise ValueError(f"block of shape {g.shape}, expected {(self.r, d, d)}")
        return np.ascontiguousarray(np.concatenate([np.asarray(g, np.complex128).ravel() for g in blocks]))

    def unpack(self, flat):
        out, off = [], 0
        for d in self.dims:
            sz = self.r * d * d
            out.append(flat[off:off + sz].reshape(self.r, d, d).copy())
            off += sz
        return out

    @staticmethod
    def _topo(topology):
        t = np.ascontiguousarray(np.asarray(topology, dtype=np.int32).reshape(-1, 2))
        return t, t.shape[0]

    # ---------------------------------------------------------------- reference API
    def get_num_self_energy_backbones(self, topology):
        t, m = self._topo(topology)
        out = ctypes.c_long()
        _lib.check(_lib.lib().xca_num_self_energy_backbones(self._ctx, m, _lib.as_ip(t), ctypes.byref(out)))
        return out.value

    def get_num_single_ptcle_gf_backbones(self, topology):
        t, m = self._topo(topology)
        out = ctypes.c_long()
        _lib.check(_lib.lib().xca_num_single_ptcle_gf_backbones(self._ctx, m, _lib.as_ip(t), ctypes.byref(out)))
        return out.value

    def compute_self_energy(self, G_ppsc, topology, f_ix=None):
        """Sigma contribution of one topology (all flat indices, one, or a list), bsb.cpp:369-459."""
        t, m = self._topo(topology)
        g = self.pack(G_ppsc)
        out = np.zeros_like(g)
        if f_ix is None:
            fp, nf = None, 0
        else:
            fix = np.ascontiguousarray(np.atleast_1d(f_ix), dtype=np.int64)
            fp, nf = _lib.as_lp(fix), len(fix)
        _lib.check(_lib.lib().xca_compute_self_energy(self._ctx, _lib.as_dp(g.view(np.float64)), m, _lib.as_ip(t), fp, nf,
                                                      _lib.as_dp(out.view(np.float64))))
        return self.unpack(out)

    def compute_single_ptcle_gf(self, G_ppsc, topology, f_ix=None):
        """Single-particle correlator g(tau)[mu][ka] of one topology, (r, n, n) complex (bsb.cpp:779-821)."""
        t, m = self._topo(topology)
        g = self.pack(G_ppsc)
        out = np.zeros((self.r, self.n, self.n), np.complex128)
        if f_ix is None:
            fp, nf = None, 0
        else:
            fix = np.ascontiguousarray(np.atleast_1d(f_ix), dtype=np.int64)
            fp, nf = _lib.as_lp(fix), len(fix)
        _lib.check(_lib.lib().xca_compute_single_ptcle_gf(self._ctx, _lib.as_dp(g.view(np.float64)), m, _lib.as_ip(t), fp, nf,
                                                          _lib.as_dp(out.view(np.float64))))
        return out

    def compute_single_ptcle_gf_device(self, G_dev, topology, scale, g_dev):
        t, m = self._topo(topology)
        _lib.check(_lib.lib().xca_compute_single_ptcle_gf_device(self._ctx, ctypes.c_void_p(G_dev), m, _lib.as_ip(t), float(scale),
                                                                 ctypes.c_void_p(g_dev)))

    def self_energy_items(self, G_ppsc, topology, max_rows=None):
        """Valid (f_ix, b_ix, p_kap, ind_path...) items of find_path_self_energy in flat-index order."""
        t, m = self._topo(topology)
        g = self.pack(G_ppsc)
        n = ctypes.c_long()
        L = _lib.lib()
        _lib.check(L.xca_self_energy_items(self._ctx, _lib.as_dp(g.view(np.float64)), m, _lib.as_ip(t), None, 0, ctypes.byref(n)))
        rows_n = n.value if max_rows is None else min(n.value, max_rows)
        rows = np.zeros((max(rows_n, 1), 3 + 2 * m - 1), np.int64)
        _lib.check(L.xca_self_energy_items(self._ctx, _lib.as_dp(g.view(np.float64)), m, _lib.as_ip(t), _lib.as_lp(rows),
                                           rows_n, ctypes.byref(n)))
        return rows[:rows_n]

    def compute_one_time_correlator(self, G_ppsc, ops_tau, ops_0, ad, topology, f_ix=None):
        """C(tau)[mu][ka] of one topology with the operators ops_tau at tau and ops_0 at 0, (r, len(ops_tau),
        len(ops_0)) complex (``compute_one_time_correlator``, bsb.cpp:843-866).  An operator is a dense Fock-space
        matrix (converted with ``ad.get_op_mat``) or already in block form ``(index, blocks)``."""
        t, m = self._topo(topology)
        g = self.pack(G_ppsc)

        def blocked(ops):
            idx, parts = [], []
            for op in ops:
                i, blks = op if isinstance(op, tuple) else ad.get_op_mat(op)
                i = np.asarray(i, np.int32)
                if i.shape != (len(self.dims),):
                    raise ValueError(f"operator block index of shape {i.shape}, expected ({len(self.dims)},)")
                idx.append(i)
                for b, tb in enumerate(i):
                    if tb >= 0:
                        blk = np.asarray(blks[b], np.complex128)
                        if blk.shape != (self.dims[tb], self.dims[b]):
                            raise ValueError(f"operator block {b} has shape {blk.shape}, expected {(self.dims[tb], self.dims[b])}")
                        parts.append(blk.ravel())
            data = np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros(1, np.complex128))
            return np.ascontiguousarray(np.concatenate(idx)), data

        mi, md = blocked(ops_tau)
        ki, kd = blocked(ops_0)
        out = np.zeros((self.r, len(ops_tau), len(ops_0)), np.complex128)
        if f_ix is None:
            fp, nf = None, 0
        else:
            fix = np.ascontiguousarray(np.atleast_1d(f_ix), dtype=np.int64)
            fp, nf = _lib.as_lp(fix), len(fix)
        _lib.check(_lib.lib().xca_compute_one_time_correlator(
            self._ctx, _lib.as_dp(g.view(np.float64)), len(ops_tau), _lib.as_ip(mi), _lib.as_dp(md.view(np.float64)), len(ops_0),
            _lib.as_ip(ki), _lib.as_dp(kd.view(np.float64)), m, _lib.as_ip(t), fp, nf, _lib.as_dp(out.view(np.float64))))
        return out

    def convolve_ppsc(self, G1, G2):
        """Per block the time-ordered DLR convolution (G1 * G2)(tau) (``convolve_ppsc``, block_sparse.cpp:832-850)."""
        a, b = self.pack(G1), self.pack(G2)
        out = np.zeros_like(a)
        _lib.check(_lib.lib().xca_convolve_ppsc(self._ctx, _lib.as_dp(a.view(np.float64)), _lib.as_dp(b.view(np.float64)),
                                                _lib.as_dp(out.view(np.float64))))
        return self.unpack(out)

    def expectation_value(self, op, ad, G_ppsc):
        """-sum_b Tr[O_b G_b(beta)] of a block-diagonal Fock-space operator (``expectation_value``,
        block_sparse.cpp:797-818); ``op`` a dense Fock-space matrix or ``(index, blocks)``."""
        idx, blks = op if isinstance(op, tuple) else ad.get_op_mat(op)
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        parts = [np.asarray(blks[b], np.complex128).ravel() for b in range(len(idx)) if idx[b] >= 0]
        data = np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros(1, np.complex128))
        g = self.pack(G_ppsc)
        out = np.zeros(2)
        _lib.check(_lib.lib().xca_expectation_value(self._ctx, _lib.as_dp(g.view(np.float64)), _lib.as_ip(idx),
                                                    _lib.as_dp(data.view(np.float64)), _lib.as_dp(out)))
        return complex(out[0], out[1])

    def trace(self, G_ppsc):
        """sum_b Tr G_b(beta) from the DLR expansion of each block (``trace``, block_sparse.cpp:852-861)."""
        g = self.pack(G_ppsc)
        out = np.zeros(2)
        _lib.check(_lib.lib().xca_trace(self._ctx, _lib.as_dp(g.view(np.float64)), _lib.as_dp(out)))
        return complex(out[0], out[1])

    @property
    def padded_rank(self):
        """Register-column width the Sigma kernels are compiled for: the DLR rank rounded up to 32, 48 or 64
        (evaluators batched into one launch share it)."""
        return 32 if self.r <= 32 else (48 if self.r <= 48 else 64)

    @property
    def precision_mode(self):
        """'fp64' (items summed with atomics) or 'fp64_ordered' (fixed summation order, reproducible bit for bit)."""
        out = ctypes.c_int()
        _lib.check(_lib.lib().xca_get_precision_mode(self._ctx, ctypes.byref(out)))
        return {v: k for k, v in _lib.PRECISION_MODES.items()}[out.value]

    @precision_mode.setter
    def precision_mode(self, mode):
        if mode not in _lib.PRECISION_MODES:
            raise NotImplementedError(f"precision mode {mode!r} is not available ({sorted(_lib.PRECISION_MODES)})")
        _lib.check(_lib.lib().xca_set_precision_mode(self._ctx, _lib.PRECISION_MODES[mode]))

    def set_tuning(self, **params):
        """Launch-shape parameters (unit_batches, wide_unit_tuples, wide_ctas_per_sm of the Sigma kernels; dyson_blocked_min_n of the Dyson solve)."""
        for k, v in params.items():
            if k not in _lib.TUNING:
                raise ValueError(f"unknown tuning parameter {k!r} ({sorted(_lib.TUNING)})")
            _lib.check(_lib.lib().xca_set_tuning(self._ctx, _lib.TUNING[k], int(v)))

    def get_tuning(self):
        out = {}
        for k, i in _lib.TUNING.items():
            v = ctypes.c_int()
            _lib.check(_lib.lib().xca_get_tuning(self._ctx, i, ctypes.byref(v)))
            out[k] = v.value
        return out

    # ---------------------------------------------------------------- device-resident use
    def dyson_setup(self, G0):
        """Dyson solvers of every block for the atomic propagator G0 (``DysonItPPSC(beta, itops, G0_b)`` for each
        block, block_sparse_solver.py:136)."""
        g0 = self.pack(G0)
        _lib.check(_lib.lib().xca_dyson_setup(self._ctx, _lib.as_dp(g0.view(np.float64))))

    def dyson_solve_device(self, Sigma_dev, eta, G_dev, hermitize=True):
        _lib.check(_lib.lib().xca_dyson_solve_device(self._ctx, ctypes.c_void_p(Sigma_dev), float(eta), int(bool(hermitize)),
                                                     ctypes.c_void_p(G_dev)))

    def normalize_device(self, G_dev):
        """Classic normalisation of a device slab in place; returns (Z, deta)."""
        Z, de = ctypes.c_double(), ctypes.c_double()
        _lib.check(_lib.lib().xca_normalize_device(self._ctx, ctypes.c_void_p(G_dev), ctypes.byref(Z), ctypes.byref(de)))
        return Z.value, de.value

    def convolve_ppsc_device(self, G1_dev, G2_dev, H_dev):
        _lib.check(_lib.lib().xca_convolve_ppsc_device(self._ctx, ctypes.c_void_p(G1_dev), ctypes.c_void_p(G2_dev), ctypes.c_void_p(H_dev)))

    def trace_device(self, G_dev):
        out = np.zeros(2)
        _lib.check(_lib.lib().xca_trace_device(self._ctx, ctypes.c_void_p(G_dev), _lib.as_dp(out)))
        return complex(out[0], out[1])

    def max_abs_diff_device(self, a_dev, b_dev):
        out = ctypes.c_double()
        _lib.check(_lib.lib().xca_max_abs_diff_device(self._ctx, ctypes.c_void_p(a_dev), ctypes.c_void_p(b_dev),
                                                      ctypes.byref(out)))
        return out.value

    def axpby_device(self, alpha, x_dev, beta, y_dev):
        _lib.check(_lib.lib().xca_axpby_device(self._ctx, float(alpha), ctypes.c_void_p(x_dev), float(beta),
                                               ctypes.c_void_p(y_dev)))

    def device_buffer(self, slot, n_doubles):
        ptr = ctypes.POINTER(ctypes.c_double)()
        _lib.check(_lib.lib().xca_device_buffer(self._ctx, int(slot), int(n_doubles) * 8, ctypes.byref(ptr)))
        return ctypes.cast(ptr, ctypes.c_void_p).value

    def to_device(self, dev_ptr, host_real):
        a = np.ascontiguousarray(host_real, dtype=np.float64)
        _lib.check(_lib.lib().xca_copy_to_device(self._ctx, ctypes.c_void_p(dev_ptr), _lib.as_dp(a), a.size))

    def to_host(self, dev_ptr, n_doubles):
        a = np.zeros(n_doubles)
        _lib.check(_lib.lib().xca_copy_to_host(self._ctx, _lib.as_dp(a), ctypes.c_void_p(dev_ptr), a.size))
        return a

    def compute_self_energy_device(self, G_dev, topology, scale, Sigma_dev):
        t, m = self._topo(topology)
        _lib.check(_lib.lib().xca_compute_self_energy_device(self._ctx, ctypes.c_void_p(G_dev), m, _lib.as_ip(t), float(scale),
                                                             ctypes.c_void_p(Sigma_dev)))

    @staticmethod
    def compute_self_energy_device_batch(jobs):
        """Job-batched compute_self_energy_device: jobs is a list of (evaluator, G_dev, topology, scale,
        Sigma_dev); every job adds scale * Sigma(topology) of its evaluator into its Sigma_dev, the panel work of
        all jobs in one launch on the first evaluator's stream (every evaluator's stream is ordered after it).
        The evaluators share a device and a padded DLR rank and sum with atomics (precision 'fp64'); the jobs
        of one evaluator share its G."""
        n = len(jobs)
        if n == 0:
            return
        P = ctypes.c_void_p
        ctxs = (P * n)(*[j[0]._ctx for j in jobs])
        Gs = (P * n)(*[j[1] for j in jobs])
        Ss = (P * n)(*[j[4] for j in jobs])
        orders = np.zeros(n, np.int32)
        topo = np.zeros((n, 6), np.int32)
        for k, j in enumerate(jobs):
            t, m = DiagramEvaluator._topo(j[2])
            orders[k] = m
            topo[k, :2 * m] = t.ravel()
        scales = np.ascontiguousarray([float(j[3]) for j in jobs], dtype=np.float64)
        _lib.check(_lib.lib().xca_compute_self_energy_device_batch(n, ctxs, Gs, _lib.as_ip(orders), _lib.as_ip(topo),
                                                                   _lib.as_dp(scales), Ss))

    def compute_self_energy_device_shard(self, G_dev, topology, scale, Sigma_dev, shard, n_shards):
        t, m = self._topo(topology)
        _lib.check(_lib.lib().xca_compute_self_energy_device_shard(self._ctx, ctypes.c_void_p(G_dev), m, _lib.as_ip(t),
                                                                   float(scale), ctypes.c_void_p(Sigma_dev), int(shard),
                                                                   int(n_shards)))

    def zero_device(self, dev_ptr, n_doubles):
        _lib.check(_lib.lib().xca_zero_device(self._ctx, ctypes.c_void_p(dev_ptr), int(n_doubles)))

    def self_energy_flops(self, G_ppsc, topology):
        """(algorithmic real flops, number of items) of one full compute_self_energy(G, topology)."""
        t, m = self._topo(topology)
        g = self.pack(G_ppsc)
        fl = ctypes.c_double()
        n = ctypes.c_long()
        _lib.check(_lib.lib().xca_self_energy_flops(self._ctx, _lib.as_dp(g.view(np.float64)), m, _lib.as_ip(t),
                                                    ctypes.byref(fl), ctypes.byref(n)))
        return fl.value, n.value

    def profile(self, enable):
        """Enable/disable per-launch CUDA-event timing; returns (Sigma kernel ms, launches) recorded so far."""
        ms = ctypes.c_double()
        n = ctypes.c_long()
        _lib.check(_lib.lib().xca_profile(self._ctx, int(bool(enable)), ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def event_record(self, slot):
        _lib.check(_lib.lib().xca_event_record(self._ctx, int(slot)))

    def event_elapsed(self, a, b):
        ms = ctypes.c_double()
        _lib.check(_lib.lib().xca_event_elapsed(self._ctx, int(a), int(b), ctypes.byref(ms)))
        return ms.value

    def fp64_fma_peak(self):
        """Measured FP64 FMA throughput of the device in TFLOP/s."""
        out = ctypes.c_double()
        _lib.check(_lib.lib().xca_fp64_fma_probe(self._ctx, ctypes.byref(out)))
        return out.value

    def fp64_mma_peak(self):
        """Measured FP64 tensor-core (mma.sync m8n8k4 f64) throughput of the device in TFLOP/s."""
        out = ctypes.c_double()
        _lib.check(_lib.lib().xca_fp64_mma_probe(self._ctx, ctypes.byref(out)))
        return out.value

    def flush_l2(self, nbytes=256 << 20):
        _lib.check(_lib.lib().xca_flush_l2(self._ctx, int(nbytes)))

    def synchronize(self):
        _lib.check(_lib.lib().xca_synchronize(self._ctx))

    def kernel_launches(self):
        out = ctypes.c_long()
        _lib.check(_lib.lib().xca_kernel_launches(self._ctx, ctypes.byref(out)))
        return out.value


# ---------------------------------------------------------------- free functions of the reference's module
class _BlockBasis:
    """Device context holding only a DLR basis and a block structure (the state the free functions need)."""

    def __init__(self, beta, lam, eps, rf, it, dims, device=0):
        L = _lib.lib()
        self._ctx = ctypes.c_void_p()
        _lib.check(L.xca_ctx_create(int(device), ctypes.byref(self._ctx)))
        self.rf = np.ascontiguousarray(rf, dtype=float)
        self.it = np.ascontiguousarray(it, dtype=float)
        self.dims = np.ascontiguousarray(dims, dtype=np.int32)
        self.r = len(self.rf)
        _lib.check(L.xca_basis_setup(self._ctx, float(beta), float(lam), float(eps), self.r, _lib.as_dp(self.rf), _lib.as_dp(self.it),
                                     len(self.dims), _lib.as_ip(self.dims)))

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx and _lib._lib is not None:
            _lib._lib.xca_ctx_destroy(ctx)
            self._ctx = None


_BASES = {}


def _basis_for(G, mesh):
    blocks = _blocks_of(G)
    dims = tuple(int(g.shape[1]) for g in blocks)
    key = (mesh.beta, mesh.lam, mesh.eps, dims)
    if key not in _BASES:
        _BASES[key] = _BlockBasis(mesh.beta, mesh.lam, mesh.eps, mesh.dlr_rf, mesh.dlr_it.it, dims)
    return _BASES[key], blocks


def _packed(blocks):
    return np.ascontiguousarray(np.concatenate([np.asarray(g, np.complex128).ravel() for g in blocks]))


def _unpacked(flat, dims, r):
    out, off = [], 0
    for d in dims:
        out.append(flat[off:off + r * d * d].reshape(r, d, d).copy())
        off += r * d * d
    return out


def convolve_ppsc(G1, G2, mesh):
    """``convolve_ppsc(G1, G2)`` (``c++/triqs_xca/block_sparse.cpp:832-850``) on the DLR mesh ``mesh``
    (TRIQS Gfs carry their mesh; here it is passed alongside the blocks)."""
    B, b1 = _basis_for(G1, mesh)
    b2 = _blocks_of(G2)
    a, b = _packed(b1), _packed(b2)
    if a.shape != b.shape:
        raise ValueError("convolve_ppsc: G1 and G2 have different block structures")
    out = np.zeros_like(a)
    _lib.check(_lib.lib().xca_convolve_ppsc(B._ctx, _lib.as_dp(a.view(np.float64)), _lib.as_dp(b.view(np.float64)),
                                            _lib.as_dp(out.view(np.float64))))
    return _unpacked(out, B.dims, B.r)


def trace(G, mesh):
    """``trace(G)`` = sum_b Tr G_b(beta) (``c++/triqs_xca/block_sparse.cpp:852-861``)."""
    B, blocks = _basis_for(G, mesh)
    g = _packed(blocks)
    out = np.zeros(2)
    _lib.check(_lib.lib().xca_trace(B._ctx, _lib.as_dp(g.view(np.float64)), _lib.as_dp(out)))
    return complex(out[0], out[1])


def expectation_value(op, ad, G, mesh):
    """``expectation_value(op, ad, G)`` = -sum_b Tr[O_b G_b(beta)] (``c++/triqs_xca/block_sparse.cpp:797-818``)."""
    B, blocks = _basis_for(G, mesh)
    idx, blks = op if isinstance(op, tuple) else ad.get_op_mat(op)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    parts = [np.asarray(blks[b], np.complex128).ravel() for b in range(len(idx)) if idx[b] >= 0]
    data = np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros(1, np.complex128))
    g = _packed(blocks)
    out = np.zeros(2)
    _lib.check(_lib.lib().xca_expectation_value(B._ctx, _lib.as_dp(g.view(np.float64)), _lib.as_ip(idx), _lib.as_dp(data.view(np.float64)),
                                                _lib.as_dp(out)))
    return complex(out[0], out[1])
