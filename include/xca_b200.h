/*
 * xca_b200: C-ABI of the B200-native pseudo-particle strong-coupling hot path.
 *
 * The reference (TRIQS/xca) exposes this path as C++ classes bound to Python with c2py.  Each entry
 * point below replaces one reference interface; the comment names it by file:line within TRIQS/xca
 * (cppdlr, the third-party DLR library, is cited through TRIQS/xca's binding of it).
 *
 * Conventions
 *  - Every function returns an int status: XCA_OK or one of the error codes; xca_last_error() gives
 *    the message of the last failing call on the calling thread.  No C++ exception crosses the ABI.
 *    XCA_ERR_INVALID maps the reference's std::invalid_argument, XCA_ERR_RUNTIME its
 *    std::runtime_error.
 *  - Host buffers are owned by the caller.  The context owns its device memory and one CUDA stream.
 *    One context per thread; a context is not thread safe (as the reference's evaluator).
 *  - Complex arrays are complex128, interleaved (re, im), row-major.  Block Green's functions are
 *    packed slabs: the blocks in block order, block b an (r, d_b, d_b) array.  The device path
 *    computes in real FP64 and rejects inputs with a non-zero imaginary part (XCA_ERR_UNSUPPORTED).
 *  - Imaginary-time nodes are in cppdlr's relative format (t < 0 stands for 1 + t, t = tau / beta);
 *    real frequencies are dimensionless (omega * beta).
 */
#ifndef XCA_B200_H
#define XCA_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define XCA_OK 0
#define XCA_ERR_INVALID 1
#define XCA_ERR_RUNTIME 2
#define XCA_ERR_CUDA 3
#define XCA_ERR_UNSUPPORTED 4

/* Precision / summation modes of the Sigma evaluation (xca_set_precision_mode). */
#define XCA_PREC_FP64 0          /* FP64, items summed into Sigma with atomics (fastest; order varies run to run) */
#define XCA_PREC_FP64_ORDERED 1  /* FP64, fixed summation order: reproducible bit for bit from run to run */
#define XCA_PREC_FP32 2          /* FP32 block products on the CUDA cores, FP64 prefactors and atomic accumulation */

/* Pole tuples per work unit in XCA_PREC_FP64_ORDERED (part of the definition of its summation order). */
#define XCA_ORDERED_UNIT_TUPLES 64

typedef struct xca_ctx xca_ctx;

/* Message of the last failing call on this thread (empty string if none). */
const char *xca_last_error(void);

/* ABI version of this library. */
int xca_abi_version(void);

/* cppdlr::build_dlr_rf(lambda, eps): DLR real frequencies, ascending.
 * Replaces python/triqs_xca/pycppdlr.wrap.cxx:210-214 (build_dlr_rf).  rf_out has room for max_r. */
int xca_dlr_build_rf(double lambda, double eps, double *rf_out, int max_r, int *r_out);

/* cppdlr::imtime_ops(lambda, dlr_rf).get_itnodes(): DLR imaginary-time nodes, relative format,
 * ascending absolute time.  Replaces python/triqs_xca/pycppdlr.wrap.cxx:44-47, 111-112. */
int xca_dlr_build_it(double lambda, const double *rf, int r, double *it_out);

/* Context on CUDA device `device`.  Replaces the construction of a DiagramEvaluator's owned state
 * (c++/triqs_xca/block_sparse_backbone.hpp:80-84). */
int xca_ctx_create(int device, xca_ctx **out);
int xca_ctx_destroy(xca_ctx *ctx);

/* DiagramEvaluator(beta, Lambda, eps, hyb_poles, hyb_coeffs, Fq): TRIQS-free constructor,
 * c++/triqs_xca/block_sparse_backbone.hpp:158-162 (and the atom_diag constructor :144-147 once the
 * caller has built Fq).  Uploads the DLR basis (r, rf, it), the hybridization (p physical poles, the
 * evaluator multiplies them by beta; coefficients p x n x n complex), the symmetry-set labels of the
 * n orbitals and the field operators as BlockOpSymSet slabs (c++/triqs_xca/block_sparse.hpp:181-200):
 * F_index[s * n_blocks + b] is the target block of set s acting on block b (-1: none); F_data packs,
 * in (s, b) order over present columns, a (q_s, d_target, d_b) complex slab.  The library forms the
 * barred operators of BlockOpSymQuartet (c++/triqs_xca/block_sparse.cpp:496-577) and uploads them.
 * Validation as check_sym_set_block_diagonal (c++/triqs_xca/block_sparse.cpp:443-492). */
int xca_evaluator_setup(xca_ctx *ctx, double beta, double lambda, double eps, int r, const double *rf, const double *it,
                        int p, const double *hyb_poles, const double *hyb_coeffs, int n, const long *sym_set_labels,
                        int n_blocks, const int *block_dims, const int *F_index, const double *F_data,
                        const int *Fd_index, const double *Fd_data);

/* DLR basis only (no hybridization, no operators): the state a standalone Dyson solver needs.
 * dyson_it_ppsc's imtime_ops argument (c++/triqs_xca/dlr_dyson_ppsc.hpp:91-101; Python
 * DysonItPPSC(beta, itops, g0), python/triqs_xca/dlr_dyson_ppsc.cpp:10-20) for n_blocks blocks of
 * dimensions block_dims.  xca_evaluator_setup sets the same basis up as part of the evaluator. */
int xca_basis_setup(xca_ctx *ctx, double beta, double lambda, double eps, int r, const double *rf, const double *it,
                    int n_blocks, const int *block_dims);

/* dyson_it_ppsc(beta, itops, g0) constructor for every block at once (dlr_dyson_ppsc.hpp:91-116; one
 * object per block in python/triqs_xca/block_sparse_solver.py:136): uploads G0 (host packed complex
 * slab, real data) and its DLR coefficients. */
int xca_dyson_setup(xca_ctx *ctx, const double *G0);

/* dyson_it_ppsc::solve(sig, eta) for every block (dlr_dyson_ppsc.hpp:135-168): G solving
 * (I - G0 * (Sigma + eta)) G = G0 with the time-ordered DLR convolution.  hermitize != 0 adds the
 * step of solve_dyson (python/triqs_xca/block_sparse_solver.py:582-586), G(t) <- (G(t) + G(t)^T) / 2.
 * Host packed complex slabs in and out.  A singular system matrix gives XCA_ERR_RUNTIME. */
int xca_dyson_solve(xca_ctx *ctx, const double *Sigma, double eta, int hermitize, double *G_out);

/* dyson_it_ppsc::solve_with_op(sig, eta, op) (dlr_dyson_ppsc.hpp:188-216): the same solve with G0(t) op added to
 * the source term, (I - G0 * (Sigma + eta + op)) G = G0 in the reference's operation order (convolution, + eta
 * G0, + G0(t) op, negation).  op: one d_b x d_b complex matrix per block, packed in block order (real data). */
int xca_dyson_solve_with_op(xca_ctx *ctx, const double *Sigma, double eta, const double *op, int hermitize, double *G_out);

/* Same on device-resident real slabs, asynchronous on the context's stream; a singular system is
 * reported by the next xca_normalize_device or xca_dyson_solve. */
int xca_dyson_solve_device(xca_ctx *ctx, const double *Sigma_dev, double eta, int hermitize, double *G_dev);

/* trace(G) = sum_b Tr G_b(beta) by DLR evaluation at tau = beta (c++/triqs_xca/block_sparse.cpp:852-861);
 * tr_out = (re, im).  Host packed complex slab or device real slab. */
int xca_trace(xca_ctx *ctx, const double *G, double *tr_out);
int xca_trace_device(xca_ctx *ctx, const double *G_dev, double *tr_out);

/* normalize_pseudo_particle_gf (python/triqs_xca/block_sparse_solver.py:427-449) on a device slab:
 * Z = -Re trace(G), deta = log|Z| / beta, G(tau) <- G(tau) exp(-tau deta); returns Z and deta (the
 * caller adds deta to eta). */
int xca_normalize_device(xca_ctx *ctx, double *G_dev, double *Z, double *deta);

/* max_abs_diff_BlockGf (python/triqs_xca/block_sparse_solver.py:1379-1380) of two device slabs. */
int xca_max_abs_diff_device(xca_ctx *ctx, const double *a_dev, const double *b_dev, double *out);

/* y <- alpha x + beta y on device slabs: the mixing step G = mix G_new + (1 - mix) G of
 * python/triqs_xca/block_sparse_solver.py:346. */
int xca_axpby_device(xca_ctx *ctx, double alpha, const double *x_dev, double beta, double *y_dev);

/* DiagramEvaluator::get_num_self_energy_backbones, c++/triqs_xca/block_sparse_backbone.cpp:721-724. */
int xca_num_self_energy_backbones(xca_ctx *ctx, int m, const int *topology, long *out);

/* DiagramEvaluator::get_num_single_ptcle_gf_backbones, c++/triqs_xca/block_sparse_backbone.cpp:733-736. */
int xca_num_single_ptcle_gf_backbones(xca_ctx *ctx, int m, const int *topology, long *out);

/* DiagramEvaluator::compute_self_energy(G, topology[, f_ix_vec]),
 * c++/triqs_xca/block_sparse_backbone.cpp:369-459.  topology is m x 2 int.  f_ix == NULL evaluates
 * every flat index; otherwise the n_fix listed ones (out of range: XCA_ERR_RUNTIME as :319).
 * G and Sigma_out are host packed complex slabs; blocks that receive nothing come back as zeros. */
int xca_compute_self_energy(xca_ctx *ctx, const double *G, int m, const int *topology, const long *f_ix, long n_fix,
                            double *Sigma_out);

/* Same evaluation on device-resident real FP64 slabs (G_dev, Sigma_dev are device pointers of the
 * packed real layout), accumulating into Sigma_dev with weight `scale` (Sigma_dev += scale * Sigma).
 * This is the call the solve loop and the benchmark use with data resident in HBM. */
int xca_compute_self_energy_device(xca_ctx *ctx, const double *G_dev, int m, const int *topology, double scale,
                                   double *Sigma_dev);

/* Job-batched compute_self_energy_device (no counterpart in the reference, whose evaluator serves one solve
 * per process): job j adds scales[j] * Sigma(topology j, order orders[j]) of the evaluator ctxs[j] on its
 * device G_devs[j] into Sigma_devs[j].  The jobs' panel work units run in ONE persistent launch on ctxs[0]'s
 * stream, so the iterations of many small solves share the device without a launch each; chains too wide
 * for a panel follow on their own context's stream.  topologies is n_jobs x 6 ints (the first 2 m of each
 * used).  Every context must be set up on the same device with the same padded DLR rank and the
 * XCA_PREC_FP64 mode (else XCA_ERR_INVALID / XCA_ERR_UNSUPPORTED); the jobs of one context share one G.
 * Each context's stream is ordered after the batch; the call does not wait for the device. */
int xca_compute_self_energy_device_batch(int n_jobs, xca_ctx *const *ctxs, const double *const *G_devs, const int *orders,
                                         const int *topologies, const double *scales, double *const *Sigma_devs);

/* One shard of compute_self_energy_device: the work units u of the topology with u % n_shards == shard
 * (units are runs of pole tuples of one path class).  Summing the shards of every rank (an all-reduce)
 * gives the full result; replaces the flat-index scatter of python/triqs_xca/block_sparse_solver.py:29-33
 * and 629-640 whose partial results are then all-reduced (:638). */
int xca_compute_self_energy_device_shard(xca_ctx *ctx, const double *G_dev, int m, const int *topology, double scale,
                                         double *Sigma_dev, int shard, int n_shards);

/* Allocation-free variant of xca_compute_self_energy_device, for callers that must not allocate device
 * memory while they run: code that works inside a pre-sized memory pool or arena (a serving process that
 * reserved its HBM up front, a solver embedded in a framework that owns the device allocator), where a
 * cudaMalloc would fail, stall the device or break the owner's accounting.  No counterpart in the
 * reference.  Same arguments and result as xca_compute_self_energy_device; the per-call scratch (edge
 * tables, work list, block norms, unit counter) lives in one fixed 64 MiB array compiled into the
 * library, which every device that loads the library holds until the process exits.  The call itself
 * makes no cudaMalloc/cudaFree; the evaluator's set-up (xca_evaluator_setup) still allocates its tables
 * once beforehand.  Sizes whose scratch exceeds 64 MiB are rejected with XCA_ERR_INVALID (for example
 * third-order topologies on large bases: the edge tables grow as p^2): the edge tables' size is checked
 * before any launch, the work list's after the block-norm kernel, which has by then written the block
 * norms into the array.  Block chains wider than the panel kernel's panel give XCA_ERR_UNSUPPORTED.  The
 * call reads the block norms back, so it waits for the context's stream.  The first call on a device
 * looks up the array's device address (once per device, with that device current); make that first call
 * before any stream capture.  All calls on a device share the array: calls that overlap on the GPU (other
 * contexts or threads on the same device) race and must be serialised. */
int xca_compute_self_energy_device_noalloc(xca_ctx *ctx, const double *G_dev, int m, const int *topology, double scale,
                                           double *Sigma_dev);

/* DiagramEvaluator::compute_single_ptcle_gf(G, topology[, f_ix_vec])
 * (c++/triqs_xca/block_sparse_backbone.cpp:779-821, eval_correlator :528-706): the single-particle
 * correlator g(tau)[mu][ka] of one topology over every flat index (f_ix == NULL) or the n_fix listed
 * ones (out of range: XCA_ERR_RUNTIME).  G is a host packed complex slab; g_out is r x n x n complex. */
int xca_compute_single_ptcle_gf(xca_ctx *ctx, const double *G, int m, const int *topology, const long *f_ix, long n_fix,
                                double *g_out);

/* Same on device-resident real data, accumulating g_dev (r x n x n real) += scale * g. */
int xca_compute_single_ptcle_gf_device(xca_ctx *ctx, const double *G_dev, int m, const int *topology, double scale,
                                       double *g_dev);

/* DiagramEvaluator::compute_one_time_correlator(G, ops_tau, ops_0, ad, topology, f_ix_vec)
 * (c++/triqs_xca/block_sparse_backbone.cpp:843-866; Python eval_one_time_correlator,
 * python/triqs_xca/block_sparse_solver.py:701-741): the correlator C(tau)[mu][ka] of one topology,
 * eval_correlator (block_sparse_backbone.cpp:528-706) with the n_tau operators O_mu at tau and the n_0
 * operators O'_ka at 0 in place of F_mu and F^dag_ka.  Each operator is given in block form, as
 * setup_ops_from_triqs_2nd_quant_ops builds it (block_sparse_backbone.cpp:810-840): tau_index[mu * n_blocks
 * + b] is the block O_mu maps block b to (-1: none) and tau_data packs, in (mu, b) order over present
 * columns, the (d_target x d_b) complex block in the eigenbasis; zero_index / zero_data likewise.
 * f_ix == NULL evaluates every flat index; corr_out is r x n_tau x n_0 complex. */
int xca_compute_one_time_correlator(xca_ctx *ctx, const double *G, int n_tau, const int *tau_index, const double *tau_data, int n_0,
                                    const int *zero_index, const double *zero_data, int m, const int *topology, const long *f_ix,
                                    long n_fix, double *corr_out);

/* convolve_ppsc(G1, G2) (c++/triqs_xca/block_sparse.cpp:832-850): per block the time-ordered DLR
 * convolution (G1_b * G2_b)(tau) on the nodes.  Host packed complex slabs, or device real slabs. */
int xca_convolve_ppsc(xca_ctx *ctx, const double *G1, const double *G2, double *H_out);
int xca_convolve_ppsc_device(xca_ctx *ctx, const double *G1_dev, const double *G2_dev, double *H_dev);

/* expectation_value(op, ad, G) (c++/triqs_xca/block_sparse.cpp:797-818): -sum_b Tr[O_b G_b(beta)] for a
 * block-diagonal operator in the eigenbasis (ad.get_op_mat then U O U^dag): op_index[b] is b or -1 (no
 * block; any other value gives XCA_ERR_INVALID, the reference asserts connection[b] == b) and op_data packs
 * the (d_b x d_b) complex blocks of the present ones in block order.  out = (re, im). */
int xca_expectation_value(xca_ctx *ctx, const double *G, const int *op_index, const double *op_data, double *out);

/* Zero n_doubles of device memory on the context's stream. */
int xca_zero_device(xca_ctx *ctx, double *dev, long n_doubles);

/* Number of valid (flat index, block, symmetry set) items of find_path_self_energy
 * (c++/triqs_xca/block_sparse_backbone.cpp:229-314) for this G and topology, and optionally the rows
 * (f_ix, b_ix, p_kap, ind_path[0..2m-2]) of the first max_rows of them in flat-index order. */
int xca_self_energy_items(xca_ctx *ctx, const double *G, int m, const int *topology, long *rows, long max_rows,
                          long *n_items);

/* Algorithmic real-FP64 flop count and number of items of compute_self_energy(G, topology) over every
 * flat index, from the fixed per-item cost model (vertex 2 r d' d c [+ r d' c with a K factor]; edge
 * r d^2 #K + 2 r^2 (d^2 + d c) + 2 [r^2 (d^2 + 2 d c) + 3 r d^2 c]; zero vertex
 * |S| 2 r d_v d_1 d_0 + |S|^2 2 r d_v d_0 + |S| 2 r d_v+1 d_v d_0; accumulation r d_out d_0).
 * No counterpart in the reference (measurement support). */
int xca_self_energy_flops(xca_ctx *ctx, const double *G, int m, const int *topology, double *alg_flops, long *n_items);

/* Measurement support (no counterpart in the reference): enable/disable CUDA-event timing of every
 * Sigma kernel launch; returns (and resets) the summed device time and launch count recorded so far. */
int xca_profile(xca_ctx *ctx, int enable, double *sigma_ms, long *sigma_launches);

/* Measurement support: record CUDA event `slot` (0..7) on the context's stream; elapsed ms between two. */
int xca_event_record(xca_ctx *ctx, int slot);
int xca_event_elapsed(xca_ctx *ctx, int slot_a, int slot_b, double *ms);

/* Measurement support: overwrite `bytes` of scratch device memory on the context's stream (L2 flush). */
int xca_flush_l2(xca_ctx *ctx, long bytes);

/* Measurement support: FP64 fused-multiply-add throughput of this device in TFLOP/s (2 flops per FMA). */
int xca_fp64_fma_probe(xca_ctx *ctx, double *tflops);

/* Measurement support (no counterpart in the reference): FP64 tensor-core (mma.sync m8n8k4 f64)
 * throughput of this device in TFLOP/s (2 flops per multiply-add). */
int xca_fp64_mma_probe(xca_ctx *ctx, double *tflops);

/* Validation support (no counterpart in the reference): the panel kernels' products run on the FP64
 * tensor cores and rely on one MMA computing each element as four correctly rounded fused multiply-adds
 * in ascending k.  This checks that on the device over n_tiles random 8 x 8 x 4 tiles (every fourth one
 * cancelling) and returns the number of elements whose bits differ from the scalar chain (expected 0). */
int xca_fp64_mma_selftest(xca_ctx *ctx, long n_tiles, unsigned long long seed, long *mismatches);

/* Size in bytes of the packed real slab of the evaluator's blocks, and its rank r. */
int xca_slab_info(xca_ctx *ctx, long *n_doubles, int *r);

/* Device pointer to `bytes` of context-owned device memory (reused across calls; grown as needed). */
int xca_device_buffer(xca_ctx *ctx, int slot, long bytes, double **dev_ptr);

/* Copies between host and device slabs on the context's stream (synchronous). */
int xca_copy_to_device(xca_ctx *ctx, double *dev, const double *host, long n_doubles);
int xca_copy_to_host(xca_ctx *ctx, double *host, const double *dev, long n_doubles);

/* Wait for the context's stream. */
int xca_synchronize(xca_ctx *ctx);

/* Precision / summation mode of the context's Sigma evaluations (the reference has one mode, FP64 with
 * the sum order of its flat-index loop, c++/triqs_xca/block_sparse_backbone.cpp:407-435; this argument
 * takes the place of the precision_mode of the evaluation call).  XCA_PREC_FP64 (default): items reach
 * Sigma through atomic adds.  XCA_PREC_FP64_ORDERED: the same items summed in a fixed order — per output
 * block, path classes in enumeration order (directions, orbital tuple, symmetry set), within a class runs
 * of XCA_ORDERED_UNIT_TUPLES pole tuples in order, within a run the items in order, each partial sum
 * starting from zero; for a flat-index list (xca_compute_self_energy with f_ix) the items in list order.
 * XCA_PREC_FP32: the bulk arithmetic of the mixed-precision form — path classes that fit a shared-memory
 * panel evaluate their block products and DLR steps in FP32 (prefactors and the accumulation into Sigma
 * stay FP64); wider chains stay FP64.  Accurate to FP32 rounding for NCA topologies only: the DLR
 * convolution of every edge (K^-1 with cond ~ 1/eps, cancelling Hilbert-type sums) loses all FP32 digits,
 * so a mixed solve uses it for NCA warm-up iterations and runs the full order in FP64.
 * Applies to xca_compute_self_energy, xca_compute_self_energy_device and the single-shard
 * xca_compute_self_energy_device_shard (n_shards > 1 gives XCA_ERR_UNSUPPORTED in XCA_PREC_FP64_ORDERED); the
 * allocation-free variant always uses XCA_PREC_FP64.  Unknown modes give XCA_ERR_UNSUPPORTED. */
int xca_set_precision_mode(xca_ctx *ctx, int mode);
int xca_get_precision_mode(xca_ctx *ctx, int *mode);

/* Launch-shape parameters of the Sigma kernels, set per context (no counterpart in the reference; chosen by
 * the autotuner, xca_b200/autotune.py).  XCA_TUNE_UNIT_BATCHES: panel batches per work unit of the panel
 * kernel (1..64, default 4); XCA_TUNE_WIDE_UNIT_TUPLES: pole tuples per work unit of the wide-chain kernel
 * (1..1024, default 4); XCA_TUNE_WIDE_CTAS_PER_SM: resident CTAs per SM of the wide-chain kernel (1..8,
 * default 2); XCA_TUNE_DYSON_BLOCKED_MIN_N: the Dyson solve factorises every block with the multi-CTA blocked
 * LU when the largest system N = r d_b exceeds it, else with one CTA per block (0..2^30; the results are
 * identical bit for bit either way).  The Sigma results do not depend on them in XCA_PREC_FP64_ORDERED; in
 * XCA_PREC_FP64 they change only the order of the atomic additions.  Out-of-range values give
 * XCA_ERR_INVALID. */
#define XCA_TUNE_UNIT_BATCHES 0
#define XCA_TUNE_WIDE_UNIT_TUPLES 1
#define XCA_TUNE_WIDE_CTAS_PER_SM 2
#define XCA_TUNE_DYSON_BLOCKED_MIN_N 3
int xca_set_tuning(xca_ctx *ctx, int param, int value);
int xca_get_tuning(xca_ctx *ctx, int param, int *value);

/* Number of device allocations (cudaMalloc) the library's own buffers have made in this process since it was
 * loaded, over every context (no counterpart in the reference; lets a caller check that a call allocated
 * nothing). */
int xca_device_allocations(long *out);

/* Number of kernels this library launched on the context since creation. */
int xca_kernel_launches(xca_ctx *ctx, long *out);

#ifdef __cplusplus
}
#endif

#endif /* XCA_B200_H */
