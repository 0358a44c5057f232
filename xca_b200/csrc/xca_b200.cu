// xca_b200: B200-native (sm_100a) pseudo-particle strong-coupling hot path behind a C-ABI.
//
// Device data layout (HBM): every block Green's function is one packed slab of real FP64, block b an
// (r, d_b, d_b) array at offset goff[b]; the field operators of every symmetry set are packed slabs
// (q_s, d_target, d_b) per present block column, and the barred operators (q_s, p, d_target, d_b).
// The DLR basis matrices (LU of K(t_i, om_l), the Hilbert weights W, K(t_i, om_l)) live in global
// memory and are staged into shared memory by every block of the Sigma kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/xca_b200.h"
#include "dlr_host.hpp"
#include "launch.hpp"

namespace xca {

thread_local std::string g_err;

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define CUDA_CHECK(x)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (x);                                                                          \
    if (e_ != cudaSuccess) throw Error(XCA_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
  } while (0)

// Device allocations made by the library's own buffers since load (xca_device_allocations).
static std::atomic<long> g_device_allocations{0};

template <class T>
struct DevBuf {
  T *ptr = nullptr;
  size_t n = 0;
  void resize(size_t count) {
    if (count <= n && ptr) return;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    n = 0;
    if (count == 0) return;
    CUDA_CHECK(cudaMalloc(&ptr, count * sizeof(T)));
    g_device_allocations.fetch_add(1, std::memory_order_relaxed);
    n = count;
  }
  void upload(const std::vector<T> &v, cudaStream_t s) {
    resize(std::max<size_t>(v.size(), 1));
    if (!v.empty()) CUDA_CHECK(cudaMemcpyAsync(ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  ~DevBuf() {
    if (ptr) cudaFree(ptr);
  }
};

// Host-to-device copies of per-call descriptor lists through pinned staging memory: two areas used in turn,
// each refilled only after its previous copy completed, so a copy never waits for the work queued on the
// stream before it (a copy from pageable memory may).  An unchanged list is not copied again.
struct StagedUpload {
  void *host[2] = {nullptr, nullptr};
  size_t cap[2] = {0, 0};
  cudaEvent_t done[2] = {nullptr, nullptr};
  int next = 0;
  std::vector<unsigned char> last;  // the bytes of the last copy
  const void *last_dst = nullptr;
  void copy(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return;
    if (dst == last_dst && last.size() == bytes && std::memcmp(last.data(), src, bytes) == 0) return;
    const int k = next;
    next ^= 1;
    if (done[k]) CUDA_CHECK(cudaEventSynchronize(done[k]));
    else CUDA_CHECK(cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming));
    if (cap[k] < bytes) {
      if (host[k]) cudaFreeHost(host[k]);
      host[k] = nullptr;
      cap[k] = 0;
      CUDA_CHECK(cudaMallocHost(&host[k], bytes + bytes / 2));
      cap[k] = bytes + bytes / 2;
    }
    std::memcpy(host[k], src, bytes);
    CUDA_CHECK(cudaMemcpyAsync(dst, host[k], bytes, cudaMemcpyHostToDevice, s));
    CUDA_CHECK(cudaEventRecord(done[k], s));
    last.assign(static_cast<const unsigned char *>(src), static_cast<const unsigned char *>(src) + bytes);
    last_dst = dst;
  }
  ~StagedUpload() {
    for (int k = 0; k < 2; ++k) {
      if (done[k]) {
        cudaEventSynchronize(done[k]);
        cudaEventDestroy(done[k]);
      }
      if (host[k]) cudaFreeHost(host[k]);
    }
  }
};

// -------------------------------------------------------------------------------- small kernels
__global__ void block_maxabs_kernel(const double *G, const long *goff, const int *dims, int r, int nb, double *out) {
  int b = blockIdx.x;
  if (b >= nb) return;
  long n = (long)r * dims[b] * dims[b];
  double mx = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) mx = fmax(mx, fabs(G[goff[b] + i]));
  __shared__ double red[256];
  red[threadIdx.x] = mx;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[b] = red[0];
}

// FP64 fused multiply-add throughput probe (measurement support): 8 independent chains per thread.
__global__ void fp64_fma_probe_kernel(double *out, int iters, double x, double y) {
  double a0 = threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
  for (int i = 0; i < iters; ++i) {
    a0 = fma(a0, x, y); a1 = fma(a1, x, y); a2 = fma(a2, x, y); a3 = fma(a3, x, y);
    a4 = fma(a4, x, y); a5 = fma(a5, x, y); a6 = fma(a6, x, y); a7 = fma(a7, x, y);
  }
  double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 1.2345678e300) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// FP64 MMA throughput probe (measurement support): 8 independent 8 x 8 x 4 accumulations per warp.
__global__ void fp64_mma_probe_kernel(double *out, int iters, double x, double y) {
  const double a = x + 1e-3 * (threadIdx.x & 31), b = y;
  double c[8][2];
#pragma unroll
  for (int j = 0; j < 8; ++j) c[j][0] = c[j][1] = 0.0;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) dmma(c[j][0], c[j][1], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += c[j][0] + c[j][1];
  if (s == 1.2345678e300) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Deterministic test value of (tile, array, index): a splitmix64 hash mapped to +-[0, 1) * 2^[-7, 8].
__device__ __forceinline__ double selftest_value(unsigned long long seed, long tile, int arr, int idx) {
  unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(tile * 4 + arr + 1) + 0xD1B54A32D192ED03ull * (unsigned long long)(idx + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  const double u = (double)(z >> 11) * 0x1.0p-53 * 2.0 - 1.0;
  return scalbn(u, (int)((z >> 3) & 15) - 7);
}

// Check that one FP64 MMA computes every element as four fused multiply-adds in ascending k, each
// correctly rounded (the operation order the panel kernels rely on): per 8 x 8 x 4 tile, random A, B, C
// (every fourth tile with C cancelling A B), mma.sync against the scalar chain, mismatching bit patterns
// counted.
__global__ void fp64_mma_selftest_kernel(long n_tiles, unsigned long long seed, unsigned long long *mismatches) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = ((long)gridDim.x * blockDim.x) >> 5;
  unsigned long long bad = 0;
  for (long tile = warp; tile < n_tiles; tile += nwarps) {
    double c[2];
    for (int e = 0; e < 2; ++e) {
      const int j = 2 * q + e;
      if ((tile & 3) == 0) {
        double sp = 0.0;
        for (int k = 0; k < 4; ++k)
          sp = __dadd_rn(sp, __dmul_rn(selftest_value(seed, tile, 0, g * 4 + k), selftest_value(seed, tile, 1, k * 8 + j)));
        c[e] = -sp * (1.0 + 1e-9 * selftest_value(seed, tile, 2, g * 8 + j));
      } else {
        c[e] = (g + j) % 3 == 0 ? 0.0 : selftest_value(seed, tile, 2, g * 8 + j);
      }
    }
    double d0 = c[0], d1 = c[1];
    dmma(d0, d1, selftest_value(seed, tile, 0, g * 4 + q), selftest_value(seed, tile, 1, q * 8 + g));
    const double d[2] = {d0, d1};
    for (int e = 0; e < 2; ++e) {
      const int j = 2 * q + e;
      double ref = c[e];
      for (int k = 0; k < 4; ++k) ref = __fma_rn(selftest_value(seed, tile, 0, g * 4 + k), selftest_value(seed, tile, 1, k * 8 + j), ref);
      if (__double_as_longlong(ref) != __double_as_longlong(d[e])) ++bad;
    }
  }
  if (bad) atomicAdd(mismatches, bad);
}

__global__ void zero_kernel(double *x, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) x[i] = 0.0;
}

// -------------------------------------------------------------------------------- host context
struct Topology {
  int m;
  int t[MAXM][2];
};

// Fixed summation order of the ordered mode.  Work unit u writes the running sum of its items (pole tuples
// ascending) to slot_off[u]; groups are runs of consecutive units, listed block by block; block b's sum
// is S_b = (((0 + g_0) + g_1) + ...) over its groups in list order, each group's value
// (((0 + u_0) + u_1) + ...) over its units.  For a whole topology a group is one path class (its units
// are runs of XCA_ORDERED_UNIT_TUPLES pole tuples) and the groups of a block follow the class order
// (directions, orbital tuple, symmetry set); for a list of flat indices every (flat index, class) item is
// its own unit and group, in list order.
struct OrderedPlan {
  std::vector<WorkUnit> units;  // the panel kernel's units [0, n_panel), then the wide kernel's
  int n_panel = 0;
  std::vector<long> slot_off;
  long slot_doubles = 0;
  std::vector<int2> groups;
  std::vector<int> blk_group0;  // nb + 1
  int max_block_elems = 0;
  DevBuf<WorkUnit> d_units;
  DevBuf<long> d_slot_off;
  DevBuf<int2> d_groups;
  DevBuf<int> d_blk_group0;
};

struct ClassSet {
  std::vector<ClassRec> classes;
  std::vector<WorkUnit> units;
  DevBuf<ClassRec> d_classes;
  DevBuf<WorkUnit> d_units;
  // item order for the reference's flat-index walk: per (fb_ix, o_ix) the classes in (b, pk) order
  std::vector<std::vector<int>> by_fbo;
  long long n_items = 0;
  std::map<std::pair<int, int>, std::unique_ptr<ClassSet>> shards;
  std::unique_ptr<OrderedPlan> ordered;
  // classes too wide for a panel: their units (runs of Ctx::wide_unit_tuples pole tuples) and the per-CTA slab
  std::vector<WorkUnit> wide_units;
  DevBuf<WorkUnit> d_wide_units;
  long wide_slab = 0;  // r x widest state over the wide classes
};


struct CorrSet {
  std::vector<CorrClass> classes;
  std::vector<CorrChain> chains;
  std::vector<CorrTerm> terms;
  std::vector<WorkUnit> units;
  std::vector<int> cls_of_fbo;  // (fb * n^(m-1) + o) -> class, -1 when nothing closes a trace
  DevBuf<CorrClass> d_classes;
  DevBuf<CorrChain> d_chains;
  DevBuf<CorrTerm> d_terms;
  DevBuf<WorkUnit> d_units;
};

// External operators of a correlator: O_mu at tau (mu < nmu) and O'_ka at 0 (ka < nka), each a block
// operator (target block per block column, -1: none; a (d_target x d_b) slab per present column).  For
// the single-particle Green's function they are F_o and F^dag_o of every orbital.
struct ExtOps {
  int nmu = 0, nka = 0;
  std::vector<int> mu_idx, ka_idx;  // [op * nb + b]
  const double *d_ops = nullptr;
  const long *d_mu_off = nullptr, *d_ka_off = nullptr;
  std::string key;                  // block structure, part of the work-list cache key
};

struct Ctx {
  int device = 0;
  int nsm = 148;  // streaming multiprocessors of the device
  cudaStream_t stream = nullptr;
  long launches = 0;
  bool ready = false;
  // model
  int r = 0, p = 0, n = 0, nb = 0, nq = 0, nmax = 0;
  double beta = 0, lam = 0, eps = 0;
  std::vector<double> rf, it, tabs, k0, polesb;
  std::vector<int> dims;
  std::vector<long> goff;
  long slab = 0;
  std::vector<long> labels, sinds, ssizes;
  std::vector<int> set_to_orb;
  std::vector<int> F_idx, Fd_idx;
  std::vector<long> F_off, Fd_off, Fb_off, Fdb_off;
  std::vector<double> ops;
  std::vector<double> hval, hrefl, kitp, kitm, k0p, k0m, kpow;
  std::vector<double> LU, W, Kit, Kdinv;     // Kdinv: 1 / U_kk of K's LU factors
  std::vector<int> piv;
  int RP = 0;                                   // padded rank of the register-resident columns
  std::vector<double> LUp, Wp, BKp;             // RP x RP padded matrices
  std::vector<int> perm;                        // RP
  std::vector<long> tab_off;                    // per block offset into the edge tables (all signatures)
  long nsig_alloc = 0;
  long tab_doubles_full = 0, tab_doubles_small = 0;
  DevBuf<long> d_tab_off_small;                 // per block offsets of the 1 + 2p signature layout (orders <= 2)
  // device copies
  DevBuf<double> d_tabs, d_k0, d_kitp, d_kitm, d_kpow, d_polesb, d_hval, d_hrefl, d_ops;
  DevBuf<int> d_dims, d_set_to_orb, d_perm, d_pinv;
  DevBuf<double> d_LUp, d_Wp, d_BKp, d_tab;
  DevBuf<double> d_convw;  // RP^3: divided weights of the Dyson convolution-matrix rows
  DevBuf<double> d_op;     // per-block operator of xca_dyson_solve_with_op
  DevBuf<long> d_tab_off;
  DevBuf<long> d_goff, d_F_off, d_Fd_off, d_Fb_off, d_Fdb_off;
  DevBuf<int> d_counter;
  DevBuf<double> d_G, d_Sig, d_maxabs;
  std::vector<std::unique_ptr<DevBuf<double>>> user_bufs;
  std::map<std::string, std::unique_ptr<ClassSet>> class_cache;
  std::map<std::string, std::unique_ptr<struct CorrSet>> corr_cache;  // correlator work lists
  std::vector<double> RFp;                // RP x RP column-major: K(t_i, -om_l)
  DevBuf<double> d_RFp, d_corr_scratch;
  DevBuf<long> d_mu_off, d_ka_off;
  ExtOps spgf_ops;                        // F_o / F^dag_o of every orbital
  DevBuf<double> d_xops;                  // one-time correlator: uploaded operator slabs
  DevBuf<long> d_xmu_off, d_xka_off;
  std::map<std::string, std::unique_ptr<ClassSet>> noalloc_classes;  // host-only work lists of the allocation-free call
  const double *gmax_filter = nullptr;  // set while a device-resident call filters zero blocks in the kernels
  // job-batched Sigma launches led by this context: descriptors and units (host copies outlive the uploads)
  std::vector<SigmaJob> h_batch_jobs;
  std::vector<WorkUnit> h_batch_units;
  DevBuf<SigmaJob> d_batch_jobs;
  DevBuf<WorkUnit> d_batch_units;
  StagedUpload stage_jobs, stage_units;
  DevBuf<int> d_batch_counter;
  cudaEvent_t ev_batch = nullptr;  // orders this context's stream against a batch led by another context
  int unit_batches = 4;      // panel batches per work unit (tunable, XCA_TUNE_UNIT_BATCHES)
  int dyson_blocked_min_n = DYSON_BLOCKED_MIN_N;  // blocked Dyson LU above this N (XCA_TUNE_DYSON_BLOCKED_MIN_N)
  int wide_unit_tuples = 4;  // pole tuples per work unit of the wide kernel (XCA_TUNE_WIDE_UNIT_TUPLES)
  int wide_ctas_per_sm = 2;  // CTAs of the wide kernel per SM (XCA_TUNE_WIDE_CTAS_PER_SM)
  int precision = XCA_PREC_FP64;
  DevBuf<double> d_slots;  // ordered mode: per-unit partial sums
  DevBuf<double> d_wide_scratch;  // wide kernel: three slabs per CTA
  DevBuf<int> d_wide_counter;
  std::map<int, std::pair<int, std::unique_ptr<DevBuf<int2>>>> chunk_bufs;  // edge-table panel chunks per signature count
  // profiling: CUDA events around every Sigma launch (enabled on request), user events, L2 flush buffer
  bool profile = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;
  cudaEvent_t user_events[8] = {nullptr};
  DevBuf<double> d_flush;
  // Dyson solve state (basis-only contexts and evaluators alike)
  bool basis_ready = false, dyson_ready = false;
  std::vector<double> k1;                 // K(1, om_l)
  std::vector<long> woff, moff;           // per-block work and system-matrix offsets
  long n_conv_rows = 0;                   // largest r d_b^2 (rows of the convolution-matrix kernel grid)
  DevBuf<double> d_k1, d_rf, d_g0, d_g0c, d_g0t, d_dwork, d_mats, d_rhs, d_red, d_efac;
  DevBuf<double> d_bwork, d_ba, d_bb, d_bc, d_xop;  // convolve_ppsc / expectation_value scratch and operands
  DevBuf<long> d_bwoff, d_xop_off;
  DevBuf<long> d_woff, d_moff;
  DevBuf<int> d_status;

  DevBasis basis(int nsig) const {
    DevBasis B;
    std::memset(&B, 0, sizeof B);  // padding too: job descriptors are compared byte for byte
    B.r = r; B.p = p; B.n = n; B.nb = nb; B.nq = nq; B.beta = beta;
    B.LUp = d_LUp.ptr; B.perm = d_perm.ptr; B.pinv = d_pinv.ptr; B.Wp = d_Wp.ptr; B.BKp = d_BKp.ptr; B.tabs = d_tabs.ptr; B.k0 = d_k0.ptr;
    B.tab = d_tab.ptr; B.tab_off = nsig == nsig_alloc ? d_tab_off.ptr : d_tab_off_small.ptr; B.nsig = nsig;
    B.kitp = d_kitp.ptr; B.kitm = d_kitm.ptr; B.kpow = d_kpow.ptr; B.polesb = d_polesb.ptr;
    B.hval = d_hval.ptr; B.hrefl = d_hrefl.ptr; B.goff = d_goff.ptr; B.dims = d_dims.ptr; B.ops = d_ops.ptr;
    B.F_off = d_F_off.ptr; B.Fd_off = d_Fd_off.ptr; B.Fb_off = d_Fb_off.ptr; B.Fdb_off = d_Fdb_off.ptr;
    B.set_to_orb = d_set_to_orb.ptr;
    B.gmax = gmax_filter;
    return B;
  }
};

static void set_device(Ctx *c) { CUDA_CHECK(cudaSetDevice(c->device)); }

static Topology parse_topology(int m, const int *topo) {
  if (m < 1 || m > MAXM) throw Error(XCA_ERR_UNSUPPORTED, "topology order " + std::to_string(m) + " not supported (1..3)");
  Topology T;
  T.m = m;
  for (int i = 0; i < m; ++i) {
    T.t[i][0] = topo[2 * i];
    T.t[i][1] = topo[2 * i + 1];
    if (T.t[i][0] >= T.t[i][1]) throw Error(XCA_ERR_INVALID, "first row of topology must contain smaller-numbered vertices");
    if (T.t[i][1] >= 2 * m || T.t[i][0] < 0) throw Error(XCA_ERR_INVALID, "topology vertex out of range");
  }
  if (T.t[0][0] != 0) throw Error(XCA_ERR_INVALID, "topology(0,0) must be 0");
  return T;
}

// DLR basis of a context: block structure, K(t_i, om_l) and its LU factors, the Hilbert weights W, and
// the padded column-major copies the register-column kernels stage (imtime_ops, cppdlr; call sites
// block_sparse_backbone.cpp:68-70, dlr_dyson_ppsc.hpp:57-76).  Uploads them to the device.
static void setup_basis(Ctx *c, double beta, double lambda, double eps, int r, const double *rf, const double *it, int n_blocks,
                        const int *block_dims) {
  if (r <= 0 || n_blocks <= 0) throw Error(XCA_ERR_INVALID, "empty DLR basis or block structure");
  if (r > 64) throw Error(XCA_ERR_UNSUPPORTED, "DLR rank " + std::to_string(r) + " above 64 is not supported by the device kernels");
  c->basis_ready = false;
  c->dyson_ready = false;
  c->chunk_bufs.clear();
  c->r = r; c->nb = n_blocks; c->beta = beta; c->lam = lambda; c->eps = eps;
  c->rf.assign(rf, rf + r);
  c->it.assign(it, it + r);
  c->dims.assign(block_dims, block_dims + n_blocks);
  c->nmax = 1;
  for (int b = 0; b < n_blocks; ++b) {
    if (block_dims[b] <= 0) throw Error(XCA_ERR_INVALID, "block dimension must be positive");
    c->nmax = std::max(c->nmax, block_dims[b]);
  }
  c->goff.resize(n_blocks);
  long off = 0;
  for (int b = 0; b < n_blocks; ++b) { c->goff[b] = off; off += (long)r * block_dims[b] * block_dims[b]; }
  c->slab = off;
  c->tabs.resize(r); c->k0.resize(r); c->k1.resize(r);
  for (int i = 0; i < r; ++i) c->tabs[i] = it[i] < 0 ? 1.0 + it[i] : it[i];
  for (int l = 0; l < r; ++l) { c->k0[l] = k_abs(0.0, rf[l]); c->k1[l] = k_abs(1.0, rf[l]); }
  c->Kit.resize((size_t)r * r); c->W.assign((size_t)r * r, 0.0);
  for (int i = 0; i < r; ++i)
    for (int l = 0; l < r; ++l) c->Kit[(size_t)i * r + l] = k_it(it[i], rf[l]);
  for (int l = 0; l < r; ++l)
    for (int k = 0; k < r; ++k)
      if (k != l) c->W[(size_t)l * r + k] = c->k0[k] / (rf[k] - rf[l]);
  c->LU = c->Kit;
  lu_factor(c->LU, r, c->piv);
  c->Kdinv = lu_diag_reciprocals(c->LU, r);
  c->RP = r <= 32 ? 32 : (r <= 48 ? 48 : 64);
  const int RP = c->RP;
  c->LUp.assign((size_t)RP * RP + RP, 0.0); c->Wp.assign((size_t)RP * RP, 0.0); c->BKp.assign((size_t)RP * RP, 0.0);
  for (int k = 0; k < RP; ++k) c->LUp[(size_t)RP * RP + k] = k < r ? c->Kdinv[k] : 1.0;
  for (int i = 0; i < RP; ++i)
    for (int k = 0; k < RP; ++k) {
      // column-major: element (row i, column k) at k * RP + i
      if (i < r && k < r) {
        c->LUp[(size_t)k * RP + i] = c->LU[(size_t)i * r + k];
        c->Wp[(size_t)k * RP + i] = c->W[(size_t)i * r + k];
        c->BKp[(size_t)k * RP + i] = beta * c->Kit[(size_t)i * r + k];
      } else if (i == k) {
        c->LUp[(size_t)k * RP + i] = 1.0;
      }
    }
  c->perm.assign(RP, -1);
  {
    std::vector<int> idx(r);
    for (int i = 0; i < r; ++i) idx[i] = i;
    for (int k = 0; k < r; ++k) std::swap(idx[k], idx[c->piv[k]]);
    for (int i = 0; i < r; ++i) c->perm[i] = idx[i];
  }
  std::vector<int> pinv(RP, -1);
  for (int i = 0; i < r; ++i) pinv[c->perm[i]] = i;
  c->RFp.assign((size_t)RP * RP, 0.0);
  for (int i = 0; i < r; ++i)
    for (int l = 0; l < r; ++l) c->RFp[(size_t)l * RP + i] = k_it(it[i], -rf[l]);
  cudaStream_t s = c->stream;
  c->d_LUp.upload(c->LUp, s); c->d_Wp.upload(c->Wp, s); c->d_BKp.upload(c->BKp, s); c->d_perm.upload(c->perm, s);
  c->d_RFp.upload(c->RFp, s);
  c->d_pinv.upload(pinv, s);
  c->corr_cache.clear();
  c->d_tabs.upload(c->tabs, s); c->d_k0.upload(c->k0, s); c->d_k1.upload(c->k1, s); c->d_rf.upload(c->rf, s);
  c->d_dims.upload(c->dims, s); c->d_goff.upload(c->goff, s);
  // divided weights of the Dyson convolution-matrix rows, w(k, l, i) = ((beta K_il) K_k(0)) / (om_k - om_l) for
  // l != k (the kernel's terms, each operation correctly rounded as there), formed once per basis
  std::vector<double> convw((size_t)RP * RP * RP, 0.0);
  for (int k = 0; k < r; ++k)
    for (int l = 0; l < r; ++l) {
      if (l == k) continue;
      const double den = c->rf[k] - c->rf[l];
      for (int i = 0; i < r; ++i) convw[((size_t)k * RP + l) * RP + i] = (c->BKp[(size_t)l * RP + i] * c->k0[k]) / den;
    }
  c->d_convw.upload(convw, s);
  c->basis_ready = true;
}

static long ipow(long a, int e) {
  long r = 1;
  for (int i = 0; i < e; ++i) r *= a;
  return r;
}

// K0 work-list builder: path classes of find_path_self_energy (block_sparse_backbone.cpp:229-314).
// Validity of a block path depends on the directions, the orbital tuple, the output block, the
// symmetry set and the zero-block flags of G, never on the pole tuple, so it is enumerated once per
// (topology, zero pattern) and every valid path class stands for p^(m-1) items.

static int panel_nc_host(int RP) { return RP == 32 ? panel_width<32>() : (RP == 48 ? panel_width<48>() : panel_width<64>()); }

// (block, first column) chunks of the edge-table panels for `nsig` signatures per block.
static std::vector<int2> table_chunks(const Ctx *c, int nsig) {
  const int nc = panel_nc_host(c->RP);
  std::vector<int2> ch;
  for (int b = 0; b < c->nb; ++b) {
    const long total = (long)nsig * c->dims[b] * c->dims[b];
    for (long q = 0; q < total; q += nc) ch.push_back(make_int2(b, (int)q));
  }
  return ch;
}

static std::string class_key(const Topology &T, const std::vector<int> &zero) {
  std::ostringstream key;
  key << T.m;
  for (int i = 0; i < T.m; ++i) key << ":" << T.t[i][0] << "," << T.t[i][1];
  key << "|";
  for (int z : zero) key << (z ? '0' : '1');
  return key.str();
}

// Host side of the work list: the path classes and their work units (no device memory touched).
static std::unique_ptr<ClassSet> build_classes(Ctx *c, const Topology &T, const std::vector<int> &zero) {
  auto cs = std::make_unique<ClassSet>();
  const int m = T.m, nv = 2 * m, vct0 = T.t[0][1];
  const long fbmax = 1L << m, omax = ipow(c->n, m - 1);
  const long npt = ipow(c->p, m - 1);
  if (npt > INT32_MAX) throw Error(XCA_ERR_UNSUPPORTED, "too many pole tuples");
  cs->by_fbo.resize(fbmax * omax);
  for (long fb = 0; fb < fbmax; ++fb)
    for (long o = 0; o < omax; ++o) {
      int fbv[MAXM];
      long q = fb;
      for (int i = 0; i < m; ++i) { fbv[i] = q % 2; q /= 2; }
      int dag[MAXV] = {0}, bar[MAXV] = {0}, orb[MAXV], vline[MAXV];
      for (int v = 0; v < nv; ++v) { orb[v] = -1; vline[v] = 0; }
      // set_directions (backbone.cpp:35-76)
      if (fbv[0] == 1) { dag[0] = 0; dag[T.t[0][1]] = 1; } else { dag[0] = 1; dag[T.t[0][1]] = 0; }
      for (int i = 1; i < m; ++i) {
        bar[T.t[i][0]] = 0; bar[T.t[i][1]] = 1;
        if (fbv[i] == 1) { dag[T.t[i][0]] = 0; dag[T.t[i][1]] = 1; } else { dag[T.t[i][0]] = 1; dag[T.t[i][1]] = 0; }
        vline[T.t[i][0]] = i; vline[T.t[i][1]] = i;
      }
      // set_orb_inds (backbone.cpp:165-186)
      long oq = o;
      for (int i = 1; i < m; ++i) {
        int ov = (int)(oq % c->n);
        oq /= c->n;
        orb[T.t[i][0]] = ov;
        orb[T.t[i][1]] = ov;
      }
      auto idx_of = [&](int v, int set, int b) -> int {
        return dag[v] ? c->Fd_idx[set * c->nb + b] : c->F_idx[set * c->nb + b];
      };
      for (int b = 0; b < c->nb; ++b)
        for (int pk = 0; pk < c->nq; ++pk) {
          int path[2 * MAXM], bd[2 * MAXM + 1];
          bool bad = false;
          int ip = -1;
          for (int v = 0; v < vct0; ++v) {
            int set = (v == 0) ? pk : (int)c->labels[orb[v]];
            ip = idx_of(v, set, v == 0 ? b : ip);
            bad = (ip == -1) || (v < nv - 1 && zero[ip]);
            if (bad) break;
            path[v] = ip;
          }
          if (bad) continue;
          bd[0] = c->dims[b];
          bd[1] = c->dims[idx_of(0, pk, b)];
          for (int v = 0; v < vct0 - 1; ++v) bd[v + 2] = c->dims[idx_of(v + 1, (int)c->labels[orb[v + 1]], path[v])];
          ip = path[vct0 - 1];
          for (int v = vct0; v < nv; ++v) {
            int set = (v == vct0) ? pk : (int)c->labels[orb[v]];
            ip = idx_of(v, set, ip);
            bad = (ip == -1) || (v < nv - 1 && zero[ip]);
            if (bad) break;
            if (v < nv - 1) path[v] = ip;
          }
          if (bad) continue;
          bd[vct0 + 1] = c->dims[idx_of(vct0, pk, path[vct0 - 1])];
          for (int v = vct0; v < nv - 1; ++v) bd[v + 2] = c->dims[idx_of(v + 1, (int)c->labels[orb[v + 1]], path[v])];
          if (bd[nv] != c->dims[b] || bd[0] != c->dims[b])
            throw Error(XCA_ERR_INVALID, "BlockDiagOpFun::add_block: contribution shape does not match block " + std::to_string(b));
          ClassRec R;
          std::memset(&R, 0, sizeof(R));
          R.m = m; R.vct0 = vct0; R.b_out = b; R.pk = pk; R.npt = (int)npt;
          R.fbmask = 0;
          for (int i = 0; i < m; ++i) R.fbmask |= fbv[i] << i;
          for (int i = 0; i < m; ++i) { R.la[i] = T.t[i][0]; R.lb[i] = T.t[i][1]; }
          for (int i = 0; i < nv - 1; ++i) R.ind_path[i] = path[i];
          for (int i = 0; i <= nv; ++i) R.bdims[i] = bd[i];
          {
            // widest panel state along the chain: blocks up to the zero vertex carry d1 columns per
            // entry, the zero vertex's intermediate and everything after it d0
            int w = 0;
            for (int i = 1; i <= vct0; ++i) w = std::max(w, bd[i] * bd[1]);
            for (int i = vct0; i <= nv; ++i) w = std::max(w, bd[i] * bd[0]);
            R.dcmax = w;
            const int nc = panel_nc_host(c->RP);
            R.wide = R.dcmax > nc ? 1 : 0;
            R.batch = R.wide ? 1 : std::min(PANEL_BMAX, nc / R.dcmax);
          }
          for (int v = 0; v < nv; ++v) {
            R.vline[v] = vline[v];
            if (v == 0 || v == vct0) { R.vkind[v] = 0; R.vset[v] = pk; R.vqo[v] = 0; continue; }
            R.vkind[v] = bar[v] ? (dag[v] ? 3 : 2) : (dag[v] ? 1 : 0);
            R.vset[v] = (int)c->labels[orb[v]];
            R.vqo[v] = (int)c->sinds[orb[v]];
          }
          cs->by_fbo[fb * omax + o].push_back((int)cs->classes.size());
          cs->classes.push_back(R);
        }
    }
  for (size_t k = 0; k < cs->classes.size(); ++k) {
    const ClassRec &R = cs->classes[k];
    const long usz = R.wide ? c->wide_unit_tuples : (long)R.batch * c->unit_batches;
    for (long s = 0; s < npt; s += usz) {
      WorkUnit u;
      u.cls = (int)k;
      u.first = (int)s;
      u.count = (int)std::min<long>(usz, npt - s);
      (R.wide ? cs->wide_units : cs->units).push_back(u);
    }
    if (R.wide) cs->wide_slab = std::max(cs->wide_slab, (long)c->r * R.dcmax);
  }
  cs->n_items = (long long)cs->classes.size() * npt;
  return cs;
}

static ClassSet *get_classes(Ctx *c, const Topology &T, const std::vector<int> &zero) {
  const std::string key = class_key(T, zero);
  auto itc = c->class_cache.find(key);
  if (itc != c->class_cache.end()) return itc->second.get();
  auto cs = build_classes(c, T, zero);
  cs->d_classes.upload(cs->classes, c->stream);
  cs->d_units.upload(cs->units, c->stream);
  cs->d_wide_units.upload(cs->wide_units, c->stream);
  ClassSet *ret = cs.get();
  c->class_cache[key] = std::move(cs);
  return ret;
}

static void launch_tables(Ctx *c, const double *G_dev, int nsig, const int2 *d_chunks, int n_chunks, const DevBasis &B) {
  (void)nsig;
  switch (c->RP) {
    case 32: c->launches += launch_edge_tables<32>(c->stream, c->nsm, B, G_dev, d_chunks, n_chunks); break;
    case 48: c->launches += launch_edge_tables<48>(c->stream, c->nsm, B, G_dev, d_chunks, n_chunks); break;
    default: c->launches += launch_edge_tables<64>(c->stream, c->nsm, B, G_dev, d_chunks, n_chunks); break;
  }
}

// Edge tables of the current G for every signature an order-m topology can use.
static int prepare_tables(Ctx *c, const double *G_dev, int m) {
  const int nsig = (m >= 3) ? (int)c->nsig_alloc : 1 + 2 * c->p;
  const long need = (m >= 3) ? c->tab_doubles_full : c->tab_doubles_small;
  if ((size_t)need > c->d_tab.n) {
    size_t free_b = 0, total_b = 0;
    CUDA_CHECK(cudaMemGetInfo(&free_b, &total_b));
    if ((double)need * 8.0 > 0.85 * (double)(free_b + c->d_tab.n * 8))
      throw Error(XCA_ERR_UNSUPPORTED, "edge tables of order " + std::to_string(m) + " need " + std::to_string(need * 8) +
                                           " bytes of device memory, more than is free");
    c->d_tab.resize(need);
  }
  auto it = c->chunk_bufs.find(nsig);
  if (it == c->chunk_bufs.end()) {
    const auto ch = table_chunks(c, nsig);
    auto buf = std::make_unique<DevBuf<int2>>();
    buf->upload(ch, c->stream);
    it = c->chunk_bufs.emplace(nsig, std::make_pair((int)ch.size(), std::move(buf))).first;
  }
  launch_tables(c, G_dev, nsig, it->second.second->ptr, it->second.first, c->basis(nsig));
  return nsig;
}

static void launch_sigma_units(Ctx *c, const DevBasis &B, const ClassRec *d_classes, const WorkUnit *d_units, int n_units, int *counter,
                               const double *G_dev, const SigmaOut &out) {
  switch (c->RP) {
    case 32: c->launches += launch_sigma_panel<32>(c->stream, c->nsm, B, d_classes, d_units, n_units, counter, G_dev, out); break;
    case 48: c->launches += launch_sigma_panel<48>(c->stream, c->nsm, B, d_classes, d_units, n_units, counter, G_dev, out); break;
    default: c->launches += launch_sigma_panel<64>(c->stream, c->nsm, B, d_classes, d_units, n_units, counter, G_dev, out); break;
  }
}

static SigmaOut atomic_out(double *Sig_dev, double scale) {
  SigmaOut o;
  o.Sigma = Sig_dev;
  o.scale = scale;
  o.slots = nullptr;
  o.slot_off = nullptr;
  return o;
}

// Per-block max |G_b| of a device G into d_maxabs, left on the device: the Sigma kernels drop the paths
// through zero blocks themselves, so a device-resident call needs no host round trip.  The work list is
// the one of the all-nonzero pattern.
static const double *block_max_async(Ctx *c, const double *G_dev) {
  c->d_maxabs.resize(c->nb);
  block_maxabs_kernel<<<c->nb, 256, 0, c->stream>>>(G_dev, c->d_goff.ptr, c->d_dims.ptr, c->r, c->nb, c->d_maxabs.ptr);
  c->launches++;
  CUDA_CHECK(cudaGetLastError());
  return c->d_maxabs.ptr;
}

// Clears the context's zero-block filter when a device-resident call leaves (also on errors).
struct GmaxFilter {
  Ctx *c;
  GmaxFilter(Ctx *ctx, const double *gmax) : c(ctx) { c->gmax_filter = gmax; }
  ~GmaxFilter() { c->gmax_filter = nullptr; }
};

static std::vector<int> zero_flags_device(Ctx *c, const double *G_dev) {
  c->d_maxabs.resize(c->nb);
  block_maxabs_kernel<<<c->nb, 256, 0, c->stream>>>(G_dev, c->d_goff.ptr, c->d_dims.ptr, c->r, c->nb, c->d_maxabs.ptr);
  c->launches++;
  CUDA_CHECK(cudaGetLastError());
  std::vector<double> mx(c->nb);
  CUDA_CHECK(cudaMemcpyAsync(mx.data(), c->d_maxabs.ptr, c->nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  std::vector<int> z(c->nb);
  for (int b = 0; b < c->nb; ++b) z[b] = mx[b] < 1e-16 ? 1 : 0;
  return z;
}

// Ordered-mode plan of a unit list: slot offsets and per-block groups.  `group_of_unit[u]` numbers the
// group of unit u (groups are listed in increasing number within a block); the units of a group belong to
// one class.  The panel kernel's units are placed first, then the wide kernel's.
static std::unique_ptr<OrderedPlan> make_plan(const Ctx *c, const std::vector<ClassRec> &classes, const std::vector<WorkUnit> &units,
                                              const std::vector<int> &group_of_unit) {
  auto P = std::make_unique<OrderedPlan>();
  const size_t nu = units.size();
  std::vector<int> grp;
  for (int pass = 0; pass < 2; ++pass)
    for (size_t u = 0; u < nu; ++u)
      if (classes[units[u].cls].wide == pass) {
        P->units.push_back(units[u]);
        grp.push_back(group_of_unit[u]);
      }
  P->n_panel = 0;
  for (const WorkUnit &w : P->units) P->n_panel += classes[w.cls].wide ? 0 : 1;
  P->slot_off.resize(nu);
  long off = 0;
  for (size_t u = 0; u < nu; ++u) {
    const ClassRec &R = classes[P->units[u].cls];
    P->slot_off[u] = off;
    off += (long)c->r * R.bdims[2 * R.m] * R.bdims[0];
  }
  P->slot_doubles = off;
  // groups: consecutive units of equal group number, then per block in increasing group number
  std::vector<std::vector<std::pair<int, int2>>> per_block(c->nb);
  for (size_t u = 0; u < nu;) {
    size_t v = u + 1;
    while (v < nu && grp[v] == grp[u]) ++v;
    per_block[classes[P->units[u].cls].b_out].push_back({grp[u], make_int2((int)u, (int)v)});
    u = v;
  }
  P->blk_group0.assign(c->nb + 1, 0);
  for (int b = 0; b < c->nb; ++b) {
    auto &lst = per_block[b];
    std::stable_sort(lst.begin(), lst.end(), [](const std::pair<int, int2> &a, const std::pair<int, int2> &x) { return a.first < x.first; });
    P->blk_group0[b + 1] = P->blk_group0[b] + (int)lst.size();
    for (const auto &g : lst) P->groups.push_back(g.second);
    P->max_block_elems = std::max(P->max_block_elems, c->r * c->dims[b] * c->dims[b]);
  }
  P->d_units.upload(P->units, c->stream);
  P->d_slot_off.upload(P->slot_off, c->stream);
  P->d_groups.upload(P->groups, c->stream);
  P->d_blk_group0.upload(P->blk_group0, c->stream);
  return P;
}

// Plan of a whole topology: per class (class order) runs of XCA_ORDERED_UNIT_TUPLES pole tuples.
static OrderedPlan *ordered_plan(Ctx *c, ClassSet *cs) {
  if (cs->ordered) return cs->ordered.get();
  std::vector<WorkUnit> units;
  std::vector<int> grp;
  for (size_t k = 0; k < cs->classes.size(); ++k) {
    const int npt = cs->classes[k].npt;
    for (int s = 0; s < npt; s += XCA_ORDERED_UNIT_TUPLES) {
      units.push_back(WorkUnit{(int)k, s, std::min(XCA_ORDERED_UNIT_TUPLES, npt - s)});
      grp.push_back((int)k);
    }
  }
  cs->ordered = make_plan(c, cs->classes, units, grp);
  return cs->ordered.get();
}

// Sum of the unit slots in the plan's fixed order, Sigma_b += scale * S_b (ordered mode, second step).
__global__ void sigma_ordered_reduce_kernel(const double *__restrict__ slots, const long *__restrict__ slot_off,
                                            const int2 *__restrict__ groups, const int *__restrict__ blk_group0,
                                            const long *__restrict__ goff, const int *__restrict__ dims, int r, double scale,
                                            double *__restrict__ Sigma) {
  const int b = blockIdx.y;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= r * dims[b] * dims[b]) return;
  double S = 0.0;
  for (int g = blk_group0[b]; g < blk_group0[b + 1]; ++g) {
    const int2 gr = groups[g];
    double cp = 0.0;
    for (int u = gr.x; u < gr.y; ++u) cp = __dadd_rn(cp, slots[slot_off[u] + x]);
    S = __dadd_rn(S, cp);
  }
  double *dst = Sigma + goff[b] + x;
  *dst = __dadd_rn(*dst, __dmul_rn(scale, S));
}

// The wide kernel over n_units units (per-CTA slabs of `slab` doubles, three each).
static void launch_wide_units(Ctx *c, const DevBasis &B, const ClassRec *d_classes, const WorkUnit *d_units, int n_units, long slab,
                              const double *G_dev, const SigmaOut &out) {
  if (n_units == 0) return;
  const int grid = std::max(1, std::min(c->wide_ctas_per_sm * c->nsm, n_units));
  long qmax = 1;
  for (long q : c->ssizes) qmax = std::max(qmax, q);
  const long cta_doubles = (3 + qmax) * std::max(slab, 1L);
  c->d_wide_scratch.resize((size_t)grid * cta_doubles);
  c->d_wide_counter.resize(1);
  switch (c->RP) {
    case 32: c->launches += launch_sigma_wide<32>(c->stream, grid, B, d_classes, d_units, n_units, c->d_wide_counter.ptr, G_dev, out, c->d_wide_scratch.ptr, slab, cta_doubles); break;
    case 48: c->launches += launch_sigma_wide<48>(c->stream, grid, B, d_classes, d_units, n_units, c->d_wide_counter.ptr, G_dev, out, c->d_wide_scratch.ptr, slab, cta_doubles); break;
    default: c->launches += launch_sigma_wide<64>(c->stream, grid, B, d_classes, d_units, n_units, c->d_wide_counter.ptr, G_dev, out, c->d_wide_scratch.ptr, slab, cta_doubles); break;
  }
}

static long plan_wide_slab(const Ctx *c, const std::vector<ClassRec> &classes, const OrderedPlan *P) {
  long slab = 0;
  for (size_t u = P->n_panel; u < P->units.size(); ++u) slab = std::max(slab, (long)c->r * classes[P->units[u].cls].dcmax);
  return slab;
}

static void launch_sigma_plan(Ctx *c, const std::vector<ClassRec> &classes, const ClassRec *d_classes, OrderedPlan *P,
                              const double *G_dev, double *Sig_dev, double scale, int nsig) {
  if (P->units.empty()) return;
  c->d_slots.resize(std::max<long>(P->slot_doubles, 1));
  SigmaOut o;
  o.Sigma = nullptr;
  o.scale = 1.0;
  o.slots = c->d_slots.ptr;
  o.slot_off = P->d_slot_off.ptr;
  const DevBasis B = c->basis(nsig);
  c->d_counter.resize(1);
  if (P->n_panel > 0) launch_sigma_units(c, B, d_classes, P->d_units.ptr, P->n_panel, c->d_counter.ptr, G_dev, o);
  const int n_wide = (int)P->units.size() - P->n_panel;
  if (n_wide > 0) {
    SigmaOut ow = o;
    ow.slot_off = P->d_slot_off.ptr + P->n_panel;
    launch_wide_units(c, B, d_classes, P->d_units.ptr + P->n_panel, n_wide, plan_wide_slab(c, classes, P), G_dev, ow);
  }
  dim3 grid((unsigned)((P->max_block_elems + 127) / 128), (unsigned)c->nb);
  sigma_ordered_reduce_kernel<<<grid, 128, 0, c->stream>>>(c->d_slots.ptr, P->d_slot_off.ptr, P->d_groups.ptr, P->d_blk_group0.ptr,
                                                           c->d_goff.ptr, c->d_dims.ptr, c->r, scale, Sig_dev);
  c->launches++;
  CUDA_CHECK(cudaGetLastError());
}

static void launch_sigma(Ctx *c, ClassSet *cs, const double *G_dev, double *Sig_dev, double scale, int nsig) {
  if (cs->units.empty() && cs->wide_units.empty()) return;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (c->profile) {
    CUDA_CHECK(cudaEventCreate(&e0));
    CUDA_CHECK(cudaEventCreate(&e1));
    CUDA_CHECK(cudaEventRecord(e0, c->stream));
  }
  if (c->precision == XCA_PREC_FP64_ORDERED) {
    launch_sigma_plan(c, cs->classes, cs->d_classes.ptr, ordered_plan(c, cs), G_dev, Sig_dev, scale, nsig);
  } else {
    c->d_counter.resize(1);
    if (!cs->units.empty() && c->precision == XCA_PREC_FP32) {
      const DevBasis B = c->basis(nsig);
      const int nu = (int)cs->units.size();
      const SigmaOut o = atomic_out(Sig_dev, scale);
      switch (c->RP) {
        case 32: c->launches += launch_sigma_f32<32>(c->stream, c->nsm, B, cs->d_classes.ptr, cs->d_units.ptr, nu, c->d_counter.ptr, G_dev, o); break;
        case 48: c->launches += launch_sigma_f32<48>(c->stream, c->nsm, B, cs->d_classes.ptr, cs->d_units.ptr, nu, c->d_counter.ptr, G_dev, o); break;
        default: c->launches += launch_sigma_f32<64>(c->stream, c->nsm, B, cs->d_classes.ptr, cs->d_units.ptr, nu, c->d_counter.ptr, G_dev, o); break;
      }
    } else if (!cs->units.empty()) {
      launch_sigma_units(c, c->basis(nsig), cs->d_classes.ptr, cs->d_units.ptr, (int)cs->units.size(), c->d_counter.ptr, G_dev,
                         atomic_out(Sig_dev, scale));
    }
    launch_wide_units(c, c->basis(nsig), cs->d_classes.ptr, cs->d_wide_units.ptr, (int)cs->wide_units.size(), cs->wide_slab, G_dev,
                      atomic_out(Sig_dev, scale));
  }
  if (c->profile) {
    CUDA_CHECK(cudaEventRecord(e1, c->stream));
    c->prof_events.emplace_back(e0, e1);
  }
}

// Algorithmic real-FP64 flop count of one item (vertex / edge / zero-vertex / accumulate terms of the
// fixed per-item cost model), for one case pattern of its lines.
static double item_flops(const Ctx *c, const ClassRec &R, const int *caseA) {
  const double r = c->r;
  const int m = R.m, vct0 = R.vct0;
  double f = 0;
  auto vertex = [&](int v, int ncol) {
    double dv = R.bdims[v], dvp = R.bdims[v + 1];
    f += 2 * r * dvp * dv * ncol;
    int line = R.vline[v];
    if (line > 0 && caseA[line]) f += r * dvp * ncol;
  };
  auto edge = [&](int e, int ncol) {
    double d = R.bdims[e + 1];
    int nk = 0;
    for (int i = 1; i < m; ++i)
      if (!caseA[i] && e >= R.la[i] && e < R.lb[i]) nk++;
    f += r * d * d * nk + 2 * r * r * (d * d + d * ncol) + 2 * (r * r * (d * d + 2 * d * ncol) + 3 * r * d * d * ncol);
  };
  for (int v = 1; v < vct0; ++v) { vertex(v, R.bdims[1]); edge(v, R.bdims[1]); }
  {
    double S = c->ssizes[R.pk], dv = R.bdims[vct0], d1 = R.bdims[1], d0 = R.bdims[0], dvp = R.bdims[vct0 + 1];
    f += S * 2 * r * dv * d1 * d0 + S * S * 2 * r * dv * d0 + S * 2 * r * dvp * dv * d0;
  }
  for (int v = vct0 + 1; v < 2 * m; ++v) { edge(v - 1, R.bdims[0]); vertex(v, R.bdims[0]); }
  f += r * R.bdims[2 * m] * R.bdims[0];
  return f;
}

// real part of a host complex slab, rejecting non-zero imaginary parts
static void real_part(const double *cplx, long n, std::vector<double> &out, const char *what) {
  out.resize(n);
  for (long i = 0; i < n; ++i) {
    if (cplx[2 * i + 1] != 0.0)
      throw Error(XCA_ERR_UNSUPPORTED, std::string(what) + " has a non-zero imaginary part; the device path computes in real FP64");
    out[i] = cplx[2 * i];
  }
}


// -------------------------------------------------------------------------------- single-particle correlator
// Work list of compute_single_ptcle_gf for one topology and zero pattern of G: per (directions, orbital
// tuple) the right chains (set_directions / eval_correlator's walk over vertices 1 .. vct0-1,
// block_sparse_backbone.cpp:540-566), the left chains (vertices vct0+1 .. 2m-1, :567-600) and the
// (mu, b, ka) terms of the trace contraction (:602-706) that close; classes without a term are dropped.
static CorrSet *get_corr(Ctx *c, const Topology &T, const std::vector<int> &zero, const ExtOps &X) {
  const std::string key = class_key(T, zero) + "|" + X.key;
  auto itc = c->corr_cache.find(key);
  if (itc != c->corr_cache.end()) return itc->second.get();
  auto cs = std::make_unique<CorrSet>();
  const int m = T.m, nv = 2 * m, vct0 = T.t[0][1], nb = c->nb, n = c->n;
  const long fbmax = 1L << (m - 1), omax = ipow(n, m - 1), npt = ipow(c->p, m - 1);
  if (npt > INT32_MAX) throw Error(XCA_ERR_UNSUPPORTED, "too many pole tuples");
  cs->cls_of_fbo.assign(fbmax * omax, -1);
  auto incomplete = [&](int ip) { return ip < 0 || zero[ip]; };
  for (long fb = 0; fb < fbmax; ++fb)
    for (long o = 0; o < omax; ++o) {
      int fbv[MAXM] = {0}, dag[MAXV] = {0}, bar[MAXV] = {0}, orb[MAXV], vline[MAXV];
      for (int v = 0; v < nv; ++v) { orb[v] = -1; vline[v] = 0; }
      for (int i = 1; i < m; ++i) fbv[i] = (int)((fb >> (i - 1)) & 1);
      // CorrelatorBackbone::set_directions (backbone.cpp:241-274)
      dag[0] = 1; dag[vct0] = 0;
      for (int i = 1; i < m; ++i) {
        bar[T.t[i][0]] = 0; bar[T.t[i][1]] = 1;
        if (fbv[i] == 1) { dag[T.t[i][0]] = 0; dag[T.t[i][1]] = 1; } else { dag[T.t[i][0]] = 1; dag[T.t[i][1]] = 0; }
        vline[T.t[i][0]] = i; vline[T.t[i][1]] = i;
      }
      long oq = o;
      for (int i = 1; i < m; ++i) {
        const int ov = (int)(oq % n);
        oq /= n;
        orb[T.t[i][0]] = ov;
        orb[T.t[i][1]] = ov;
      }
      auto idx_of = [&](int v, int col) -> int {
        const int set = (int)c->labels[orb[v]];
        return dag[v] ? c->Fd_idx[set * nb + col] : c->F_idx[set * nb + col];
      };
      CorrClass R;
      std::memset(&R, 0, sizeof(R));
      R.m = m; R.vct0 = vct0;
      for (int i = 1; i < m; ++i) R.fbmask |= fbv[i] << i;
      for (int i = 0; i < m; ++i) { R.la[i] = T.t[i][0]; R.lb[i] = T.t[i][1]; }
      for (int v = 0; v < nv; ++v) {
        R.vline[v] = vline[v];
        if (v == 0 || v == vct0) continue;
        R.vkind[v] = bar[v] ? (dag[v] ? 3 : 2) : (dag[v] ? 1 : 0);
        R.vset[v] = (int)c->labels[orb[v]];
        R.vqo[v] = (int)c->sinds[orb[v]];
      }
      // right chains from every start block
      std::vector<CorrChain> rch(nb), lch(nb);
      std::vector<int> rend(nb, -1), lend(nb, -1);
      for (int b = 0; b < nb; ++b) {
        CorrChain H;
        std::memset(&H, 0, sizeof(H));
        for (int v = 0; v < MAXV; ++v) H.path[v] = -1;
        H.start = b; H.gblock = b;
        H.path[0] = b;
        H.bd[1] = c->dims[b];
        bool bad = false;
        int ip = b;
        for (int v = 1; v < vct0; ++v) {
          ip = idx_of(v, ip);
          if (incomplete(ip)) { bad = true; break; }
          H.path[v] = ip;
          H.bd[v + 1] = c->dims[ip];
        }
        if (bad) continue;
        H.rows = H.bd[vct0];
        H.cols = H.bd[1];
        rch[b] = H;
        rend[b] = H.path[vct0 - 1];
      }
      // left chains from every start block
      for (int b = 0; b < nb; ++b) {
        CorrChain H;
        std::memset(&H, 0, sizeof(H));
        for (int v = 0; v < MAXV; ++v) H.path[v] = -1;
        H.start = b;
        H.path[vct0] = b;
        H.bd[vct0 + 1] = c->dims[b];
        bool bad = false;
        int ip = b;
        for (int v = vct0 + 1; v < nv; ++v) {
          ip = idx_of(v, ip);
          if (incomplete(ip)) { bad = true; break; }
          H.path[v] = ip;
          H.bd[v + 1] = c->dims[ip];
        }
        if (bad) continue;
        H.gblock = H.path[nv - 1];
        H.rows = H.bd[nv];
        H.cols = H.bd[vct0 + 1];
        lch[b] = H;
        lend[b] = H.path[nv - 1];
      }
      // closing terms
      std::vector<CorrTerm> terms;
      std::vector<int> rused(nb, -1), lused(nb, -1);
      std::vector<int> rlist, llist;
      for (int mu = 0; mu < X.nmu; ++mu)
        for (int b = 0; b < nb; ++b) {
          const int e0 = rend[b];
          if (incomplete(e0)) continue;
          const int e1 = X.mu_idx[mu * nb + e0];
          if (incomplete(e1)) continue;
          const int e2 = lend[e1];
          if (incomplete(e2)) continue;
          for (int ka = 0; ka < X.nka; ++ka) {
            if (X.ka_idx[ka * nb + e2] != b) continue;
            if (rused[b] < 0) { rused[b] = (int)rlist.size(); rlist.push_back(b); }
            if (lused[e1] < 0) { lused[e1] = (int)llist.size(); llist.push_back(e1); }
            CorrTerm P;
            P.mu = mu; P.ka = ka; P.rchain = rused[b]; P.lchain = lused[e1]; P.e0 = e0; P.e2 = e2;
            P.c0 = c->dims[b]; P.c1 = rch[b].rows; P.c2 = c->dims[e1]; P.c3 = lch[e1].rows;
            terms.push_back(P);
          }
        }
      if (terms.empty()) continue;
      R.chain0 = (int)cs->chains.size();
      R.n_right = (int)rlist.size();
      R.n_left = (int)llist.size();
      for (int b : rlist) cs->chains.push_back(rch[b]);
      for (int b : llist) cs->chains.push_back(lch[b]);
      R.term0 = (int)cs->terms.size();
      R.n_terms = (int)terms.size();
      cs->terms.insert(cs->terms.end(), terms.begin(), terms.end());
      cs->cls_of_fbo[fb * omax + o] = (int)cs->classes.size();
      cs->classes.push_back(R);
    }
  const int usz = 4;
  for (size_t k = 0; k < cs->classes.size(); ++k)
    for (long q = 0; q < npt; q += usz) cs->units.push_back(WorkUnit{(int)k, (int)q, (int)std::min<long>(usz, npt - q)});
  cs->d_classes.upload(cs->classes, c->stream);
  cs->d_chains.upload(cs->chains, c->stream);
  cs->d_terms.upload(cs->terms, c->stream);
  cs->d_units.upload(cs->units, c->stream);
  CorrSet *ret = cs.get();
  c->corr_cache[key] = std::move(cs);
  return ret;
}

static void launch_corr(Ctx *c, CorrSet *cs, const ExtOps &X, const WorkUnit *d_units, int n_units, const double *G_dev, double *g_dev,
                        double scale, int nsig) {
  if (n_units == 0) return;
  const int warps_per_cta = 4;
  const int grid = std::max(1, std::min(2 * c->nsm, (n_units + warps_per_cta - 1) / warps_per_cta));
  const long slab = (long)c->r * c->nmax * c->nmax;
  const long warp_doubles = (3 + 2L * c->nb) * slab + (long)c->r * X.nmu * X.nka;
  c->d_corr_scratch.resize((size_t)grid * warps_per_cta * warp_doubles);
  c->d_counter.resize(1);
  CUDA_CHECK(cudaMemsetAsync(c->d_counter.ptr, 0, sizeof(int), c->stream));
  CorrBasis CB;
  CB.RFp = c->d_RFp.ptr;
  CB.ops = X.d_ops;
  CB.mu_off = X.d_mu_off;
  CB.ka_off = X.d_ka_off;
  CB.nmu = X.nmu;
  CB.nka = X.nka;
  const DevBasis B = c->basis(nsig);
  switch (c->RP) {
#define XCA_CORR(RPV)                                                                                                          \
  case RPV:                                                                                                                    \
    c->launches += launch_correlator<RPV>(c->stream, grid, warps_per_cta, B, CB, cs->d_classes.ptr, cs->d_chains.ptr, cs->d_terms.ptr, \
                                          d_units, n_units, c->d_counter.ptr, G_dev, g_dev, scale, c->nmax, c->d_corr_scratch.ptr,  \
                                          warp_doubles);                                                                       \
    break;
    XCA_CORR(32)
    XCA_CORR(48)
    XCA_CORR(64)
#undef XCA_CORR
  }
}

// -------------------------------------------------------------------------------- Dyson, trace, normalisation
static DysonBasis dyson_basis(Ctx *c) {
  DysonBasis B;
  B.r = c->r; B.nb = c->nb; B.beta = c->beta;
  B.LUp = c->d_LUp.ptr; B.Wp = c->d_Wp.ptr; B.BKp = c->d_BKp.ptr; B.perm = c->d_perm.ptr;
  B.tabs = c->d_tabs.ptr; B.k0 = c->d_k0.ptr; B.k1 = c->d_k1.ptr; B.rf = c->d_rf.ptr;
  B.goff = c->d_goff.ptr; B.dims = c->d_dims.ptr; B.woff = c->d_woff.ptr; B.moff = c->d_moff.ptr;
  B.g0 = c->d_g0.ptr; B.g0c = c->d_g0c.ptr; B.g0t = c->d_g0t.ptr;
  B.work = c->d_dwork.ptr; B.mats = c->d_mats.ptr; B.convw = c->d_convw.ptr;
  return B;
}

static void require_basis(const Ctx *c) {
  if (!c->basis_ready) throw Error(XCA_ERR_INVALID, "no DLR basis set up on this context");
}

static void require_dyson(const Ctx *c) {
  require_basis(c);
  if (!c->dyson_ready) throw Error(XCA_ERR_INVALID, "Dyson solver not set up (xca_dyson_setup)");
}

static void launch_dyson(Ctx *c, const double *Sig_dev, double eta, int hermitize, double *G_dev, const double *op_dev = nullptr) {
  CUDA_CHECK(cudaMemsetAsync(c->d_status.ptr, 0, sizeof(int), c->stream));
  const DysonBasis B = dyson_basis(c);
  const int n_max = c->r * c->nmax, d_max = c->nmax;
  switch (c->RP) {
    case 32: c->launches += launch_dyson<32>(c->stream, B, c->n_conv_rows, Sig_dev, eta, hermitize, c->d_rhs.ptr, G_dev, c->d_status.ptr, n_max, d_max,
                                                        c->dyson_blocked_min_n, op_dev); break;
    case 48: c->launches += launch_dyson<48>(c->stream, B, c->n_conv_rows, Sig_dev, eta, hermitize, c->d_rhs.ptr, G_dev, c->d_status.ptr, n_max, d_max,
                                                        c->dyson_blocked_min_n, op_dev); break;
    default: c->launches += launch_dyson<64>(c->stream, B, c->n_conv_rows, Sig_dev, eta, hermitize, c->d_rhs.ptr, G_dev, c->d_status.ptr, n_max, d_max,
                                                        c->dyson_blocked_min_n, op_dev); break;
  }
}

// DysonBasis whose work area is the per-block scratch of the block-wise DLR operations (6 r d_b^2
// doubles per block), for calls that need no Dyson set-up.
static DysonBasis block_op_basis(Ctx *c) {
  if (!c->d_bwoff.ptr || c->d_bwork.n < (size_t)(6 * c->slab)) {
    std::vector<long> off(c->nb);
    long o = 0;
    for (int b = 0; b < c->nb; ++b) { off[b] = o; o += 6L * c->r * c->dims[b] * c->dims[b]; }
    c->d_bwoff.upload(off, c->stream);
    c->d_bwork.resize(std::max(o, 1L));
  }
  DysonBasis B = dyson_basis(c);
  B.work = c->d_bwork.ptr;
  B.woff = c->d_bwoff.ptr;
  return B;
}

static void launch_convolve_blocks(Ctx *c, const double *G1_dev, const double *G2_dev, double *H_dev) {
  const DysonBasis B = block_op_basis(c);
  switch (c->RP) {
    case 32: c->launches += launch_convolve_ppsc<32>(c->stream, B, G1_dev, G2_dev, H_dev); break;
    case 48: c->launches += launch_convolve_ppsc<48>(c->stream, B, G1_dev, G2_dev, H_dev); break;
    default: c->launches += launch_convolve_ppsc<64>(c->stream, B, G1_dev, G2_dev, H_dev); break;
  }
}

// Raise if a Dyson solve since the last check met a singular system matrix (call after a synchronize).
static void check_dyson_status(Ctx *c) {
  if (!c->d_status.ptr) return;
  int st = 0;
  CUDA_CHECK(cudaMemcpyAsync(&st, c->d_status.ptr, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  if (st) {
    CUDA_CHECK(cudaMemsetAsync(c->d_status.ptr, 0, sizeof(int), c->stream));
    throw Error(XCA_ERR_RUNTIME, "Dyson solve: singular system matrix (getrf info > 0)");
  }
}

// sum_b Tr G_b(beta) (trace, block_sparse.cpp:852-861): per-block partial traces on the device, summed on
// the host in block order.
static double trace_beta(Ctx *c, const double *G_dev) {
  const DysonBasis B = dyson_basis(c);
  c->d_red.resize(std::max(c->nb, 256));
  switch (c->RP) {
    case 32: c->launches += launch_trace_beta<32>(c->stream, B, G_dev, c->d_red.ptr); break;
    case 48: c->launches += launch_trace_beta<48>(c->stream, B, G_dev, c->d_red.ptr); break;
    default: c->launches += launch_trace_beta<64>(c->stream, B, G_dev, c->d_red.ptr); break;
  }
  std::vector<double> part(c->nb);
  CUDA_CHECK(cudaMemcpyAsync(part.data(), c->d_red.ptr, c->nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  double s = 0;
  for (double x : part) s += x;
  return s;
}

// -------------------------------------------------------------------------------- allocation-free Sigma
// xca_compute_self_energy_device_noalloc keeps everything it needs beyond its inputs, its output and the
// evaluator's set-up tables in this fixed array of the library's device image, so the call itself never
// allocates device memory.  Every device that loads the library holds the array until the process exits.
constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(64) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mu;
static std::map<int, unsigned char *> g_noalloc_base;  // device ordinal -> device address of the array

// Device address of the scratch array on `device`, which must be current.  In host code the array's name
// is only a host-side stand-in, so its address is looked up once per device and cached.
static unsigned char *noalloc_scratch(int device) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  auto it = g_noalloc_base.find(device);
  if (it != g_noalloc_base.end()) return it->second;
  void *ptr = nullptr;
  CUDA_CHECK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
  auto *base = static_cast<unsigned char *>(ptr);
  g_noalloc_base[device] = base;
  return base;
}

static size_t align256(size_t x) { return (x + 255) / 256 * 256; }

static void noalloc_fits(size_t need, const char *what) {
  if (need > NOALLOC_SCRATCH_BYTES)
    throw Error(XCA_ERR_INVALID, std::string("xca_compute_self_energy_device_noalloc: ") + what + " need " +
                                     std::to_string(need) + " bytes of scratch, the fixed scratch array holds " +
                                     std::to_string(NOALLOC_SCRATCH_BYTES) + "; use xca_compute_self_energy_device");
}

// Host entry of a correlator over the external operators X (compute_single_ptcle_gf and
// compute_one_time_correlator): every flat index (f_ix == NULL) or the listed ones.
static void correlator_host(Ctx *c, const double *G, int m, const int *topology, const long *f_ix, long n_fix, const ExtOps &X,
                            double *g_out, const char *who) {
  Topology T = parse_topology(m, topology);
  const long omax = ipow(c->n, m - 1), npt = ipow(c->p, m - 1);
  const long nmaxb = (1L << (m - 1)) * omax * npt;
  std::vector<double> g;
  real_part(G, c->slab, g, "G");
  const long nout = (long)c->r * X.nmu * X.nka;
  c->d_G.resize(c->slab);
  c->d_Sig.resize(std::max(c->slab, nout));
  CUDA_CHECK(cudaMemcpyAsync(c->d_G.ptr, g.data(), c->slab * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  zero_kernel<<<64, 256, 0, c->stream>>>(c->d_Sig.ptr, nout);
  c->launches++;
  auto zero = zero_flags_device(c, c->d_G.ptr);
  CorrSet *cs = get_corr(c, T, zero, X);
  int nsig = prepare_tables(c, c->d_G.ptr, m);
  if (f_ix == nullptr) {
    launch_corr(c, cs, X, cs->d_units.ptr, (int)cs->units.size(), c->d_G.ptr, c->d_Sig.ptr, 1.0, nsig);
  } else {
    std::vector<WorkUnit> units;
    for (long z = 0; z < n_fix; ++z) {
      const long f = f_ix[z];
      if (f < 0 || f >= nmaxb) throw Error(XCA_ERR_RUNTIME, std::string("DiagramEvaluator::") + who + ": f_ix out of range");
      const long o = f % omax, q = f / omax, pix = q % npt, fb = q / npt;
      const int k = cs->cls_of_fbo[fb * omax + o];
      if (k >= 0) units.push_back(WorkUnit{k, (int)pix, 1});
    }
    DevBuf<WorkUnit> du;
    du.upload(units, c->stream);
    launch_corr(c, cs, X, du.ptr, (int)units.size(), c->d_G.ptr, c->d_Sig.ptr, 1.0, nsig);
    CUDA_CHECK(cudaStreamSynchronize(c->stream));
  }
  std::vector<double> out(nout);
  CUDA_CHECK(cudaMemcpyAsync(out.data(), c->d_Sig.ptr, nout * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  for (long i = 0; i < nout; ++i) {
    g_out[2 * i] = out[i];
    g_out[2 * i + 1] = 0.0;
  }
}

}  // namespace xca

using namespace xca;

#define API_BEGIN try {
#define API_END                                     \
  return XCA_OK;                                    \
  }                                                 \
  catch (const Error &e) {                          \
    g_err = e.what();                               \
    return e.code;                                  \
  }                                                 \
  catch (const std::invalid_argument &e) {          \
    g_err = e.what();                               \
    return XCA_ERR_INVALID;                         \
  }                                                 \
  catch (const std::exception &e) {                 \
    g_err = e.what();                               \
    return XCA_ERR_RUNTIME;                         \
  }

extern "C" {

const char *xca_last_error(void) { return g_err.c_str(); }

int xca_abi_version(void) { return 1; }

int xca_dlr_build_rf(double lambda, double eps, double *rf_out, int max_r, int *r_out) {
  API_BEGIN
  if (!(lambda > 0) || !(eps > 0)) throw Error(XCA_ERR_INVALID, "Lambda and eps must be positive");
  auto rf = build_dlr_rf(lambda, eps);
  *r_out = (int)rf.size();
  if ((int)rf.size() > max_r) throw Error(XCA_ERR_INVALID, "rf_out too small: rank " + std::to_string(rf.size()));
  std::copy(rf.begin(), rf.end(), rf_out);
  API_END
}

int xca_dlr_build_it(double lambda, const double *rf, int r, double *it_out) {
  API_BEGIN
  std::vector<double> v(rf, rf + r);
  auto it = build_dlr_it(lambda, v);
  std::copy(it.begin(), it.end(), it_out);
  API_END
}

int xca_ctx_create(int device, xca_ctx **out) {
  API_BEGIN
  auto *c = new Ctx();
  c->device = device;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    delete c;
    throw Error(XCA_ERR_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(e));
  }
  set_device(c);
  CUDA_CHECK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device));
  CUDA_CHECK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  *out = reinterpret_cast<xca_ctx *>(c);
  API_END
}

int xca_ctx_destroy(xca_ctx *ctx) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c) return XCA_OK;
  set_device(c);
  cudaStreamSynchronize(c->stream);
  for (auto &e : c->prof_events) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  for (auto &e : c->user_events)
    if (e) cudaEventDestroy(e);
  if (c->ev_batch) cudaEventDestroy(c->ev_batch);
  cudaStream_t s = c->stream;
  delete c;
  if (s) cudaStreamDestroy(s);
  API_END
}

int xca_evaluator_setup(xca_ctx *ctx, double beta, double lambda, double eps, int r, const double *rf, const double *it, int p,
                        const double *hyb_poles, const double *hyb_coeffs, int n, const long *labels, int n_blocks,
                        const int *block_dims, const int *F_index, const double *F_data, const int *Fd_index, const double *Fd_data) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  if (r <= 0 || p <= 0 || n <= 0 || n_blocks <= 0) throw Error(XCA_ERR_INVALID, "empty basis, hybridization or block structure");
  c->ready = false;
  setup_basis(c, beta, lambda, eps, r, rf, it, n_blocks, block_dims);
  c->p = p; c->n = n;
  c->labels.assign(labels, labels + n);
  long nq = 0;
  for (int i = 0; i < n; ++i) {
    if (labels[i] < 0) throw Error(XCA_ERR_INVALID, "negative symmetry-set label");
    nq = std::max(nq, labels[i] + 1);
  }
  c->nq = (int)nq;
  c->sinds.assign(n, 0); c->ssizes.assign(nq, 0); c->set_to_orb.assign((size_t)nq * n, -1);
  for (int i = 0; i < n; ++i) {
    c->sinds[i] = c->ssizes[labels[i]];
    c->set_to_orb[(size_t)labels[i] * n + c->sinds[i]] = i;
    c->ssizes[labels[i]]++;
  }
  for (long s = 0; s < nq; ++s)
    if (c->ssizes[s] == 0) throw Error(XCA_ERR_INVALID, "BlockOpSymQuartet: symmetry set " + std::to_string(s) + " has no orbital");
  // hybridization coefficients: real part, block-diagonality in the symmetry sets (block_sparse.cpp:443-492)
  std::vector<double> coef;
  real_part(hyb_coeffs, (long)p * n * n, coef, "hyb_coeffs");
  double mx = 0;
  for (double x : coef) mx = std::max(mx, std::fabs(x));
  if (!std::isfinite(mx)) throw Error(XCA_ERR_INVALID, "DiagramEvaluator: hyb_coeffs contains a non-finite entry");
  for (int l = 0; l < p; ++l)
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        if (labels[i] != labels[j] && std::fabs(coef[((size_t)l * n + i) * n + j]) > 1e-12 * mx)
          throw Error(XCA_ERR_INVALID, "DiagramEvaluator: hyb_coeffs couples different symmetry sets, which the symmetry-set storage cannot represent");
  // operators: F, F^dag slabs, then the barred operators (BlockOpSymQuartet, block_sparse.cpp:555-576)
  c->F_idx.assign(F_index, F_index + nq * n_blocks);
  c->Fd_idx.assign(Fd_index, Fd_index + nq * n_blocks);
  c->ops.clear();
  c->F_off.assign(nq * n_blocks, -1); c->Fd_off.assign(nq * n_blocks, -1);
  c->Fb_off.assign(nq * n_blocks, -1); c->Fdb_off.assign(nq * n_blocks, -1);
  auto load = [&](const std::vector<int> &idx, const double *data, std::vector<long> &offs, const char *what) {
    long pos = 0;
    for (long s = 0; s < nq; ++s)
      for (int b = 0; b < n_blocks; ++b) {
        int tg = idx[s * n_blocks + b];
        if (tg < -1 || tg >= n_blocks) throw Error(XCA_ERR_INVALID, std::string(what) + ": block index out of range");
        if (tg < 0) continue;
        long sz = c->ssizes[s] * block_dims[tg] * block_dims[b];
        offs[s * n_blocks + b] = (long)c->ops.size();
        std::vector<double> re;
        real_part(data + 2 * pos, sz, re, what);
        c->ops.insert(c->ops.end(), re.begin(), re.end());
        pos += sz;
      }
  };
  load(c->F_idx, F_data, c->F_off, "F");
  load(c->Fd_idx, Fd_data, c->Fd_off, "F_dag");
  for (long s = 0; s < nq; ++s) {
    long q = c->ssizes[s];
    for (int b = 0; b < n_blocks; ++b) {
      if (c->Fd_idx[s * n_blocks + b] >= 0) {
        long bs = (long)block_dims[c->Fd_idx[s * n_blocks + b]] * block_dims[b];
        c->Fdb_off[s * n_blocks + b] = (long)c->ops.size();
        c->ops.resize(c->ops.size() + q * p * bs, 0.0);
      }
      if (c->F_idx[s * n_blocks + b] >= 0) {
        long bs = (long)block_dims[c->F_idx[s * n_blocks + b]] * block_dims[b];
        c->Fb_off[s * n_blocks + b] = (long)c->ops.size();
        c->ops.resize(c->ops.size() + q * p * bs, 0.0);
      }
    }
    for (int l = 0; l < p; ++l)
      for (long lam = 0; lam < q; ++lam)
        for (long nu = 0; nu < q; ++nu) {
          int lo = c->set_to_orb[s * n + lam], no = c->set_to_orb[s * n + nu];
          double cf = coef[((size_t)l * n + no) * n + lo];
          if (cf == 0.0) continue;
          for (int b = 0; b < n_blocks; ++b) {
            if (c->Fd_idx[s * n_blocks + b] >= 0) {
              long bs = (long)block_dims[c->Fd_idx[s * n_blocks + b]] * block_dims[b];
              double *dst = c->ops.data() + c->Fdb_off[s * n_blocks + b] + ((size_t)lam * p + l) * bs;
              const double *src = c->ops.data() + c->Fd_off[s * n_blocks + b] + (size_t)nu * bs;
              for (long x = 0; x < bs; ++x) dst[x] += cf * src[x];
            }
            if (c->F_idx[s * n_blocks + b] >= 0) {
              long bs = (long)block_dims[c->F_idx[s * n_blocks + b]] * block_dims[b];
              double *dst = c->ops.data() + c->Fb_off[s * n_blocks + b] + ((size_t)nu * p + l) * bs;
              const double *src = c->ops.data() + c->F_off[s * n_blocks + b] + (size_t)lam * bs;
              for (long x = 0; x < bs; ++x) dst[x] += -cf * src[x];
            }
          }
        }
  }
  // hybridization tables (Hybridization ctor, hyb.cpp:15-44)
  c->polesb.resize(p); c->kitp.resize((size_t)r * p); c->kitm.resize((size_t)r * p); c->k0p.resize(p); c->k0m.resize(p);
  for (int l = 0; l < p; ++l) {
    c->polesb[l] = hyb_poles[l] * beta;
    c->k0p[l] = k_it(0.0, c->polesb[l]);
    c->k0m[l] = k_it(0.0, -c->polesb[l]);
    for (int t = 0; t < r; ++t) {
      c->kitp[(size_t)t * p + l] = k_it(it[t], c->polesb[l]);
      c->kitm[(size_t)t * p + l] = k_it(it[t], -c->polesb[l]);
    }
  }
  c->kpow.assign((size_t)2 * p * (MAXE + 1), 1.0);
  for (int row = 0; row < 2; ++row)
    for (int l = 0; l < p; ++l)
      for (int e = 1; e <= MAXE; ++e) c->kpow[((size_t)row * p + l) * (MAXE + 1) + e] = std::pow(row == 0 ? c->k0p[l] : c->k0m[l], -e);
  c->hval.assign((size_t)r * n * n, 0.0);
  for (int t = 0; t < r; ++t)
    for (int l = 0; l < p; ++l) {
      double k = c->kitp[(size_t)t * p + l];
      for (int z = 0; z < n * n; ++z) c->hval[(size_t)t * n * n + z] += k * coef[(size_t)l * n * n + z];
    }
  // values_reflect = reflect(values) through the DLR basis (hyb.cpp:84)
  {
    std::vector<double> cfs = c->hval;
    long nc = (long)n * n;
    lu_solve_recip(c->LU, c->Kdinv, r, c->piv, cfs.data(), nc);
    c->hrefl.assign((size_t)r * nc, 0.0);
    for (int i = 0; i < r; ++i)
      for (int l = 0; l < r; ++l) {
        double k = k_it(it[i], -rf[l]);
        for (long j = 0; j < nc; ++j) c->hrefl[(size_t)i * nc + j] = std::fma(k, cfs[(size_t)l * nc + j], c->hrefl[(size_t)i * nc + j]);
      }
  }
  // edge tables: per block, 1 + 2p (orders <= 2) or 1 + 2p + 4p^2 (order 3) signatures of [fc | W fc]
  // (r d^2 each), allocated on first use by prepare_tables
  c->nsig_alloc = 1 + 2L * p + 4L * p * p;
  c->tab_off.assign(n_blocks, 0);
  std::vector<long> small_off(n_blocks, 0);
  long toff = 0, soff = 0;
  for (int b = 0; b < n_blocks; ++b) {
    c->tab_off[b] = toff;
    small_off[b] = soff;
    toff += c->nsig_alloc * 2L * r * block_dims[b] * block_dims[b];
    soff += (1 + 2L * p) * 2L * r * block_dims[b] * block_dims[b];
  }
  c->tab_doubles_full = toff;
  c->tab_doubles_small = soff;
  // upload
  cudaStream_t s = c->stream;
  c->d_tab_off.upload(c->tab_off, s);
  c->d_tab_off_small.upload(small_off, s);
  c->d_kitp.upload(c->kitp, s); c->d_kitm.upload(c->kitm, s);
  c->d_kpow.upload(c->kpow, s); c->d_polesb.upload(c->polesb, s);
  c->d_hval.upload(c->hval, s); c->d_hrefl.upload(c->hrefl, s); c->d_ops.upload(c->ops, s);
  c->d_set_to_orb.upload(c->set_to_orb, s);
  c->d_F_off.upload(c->F_off, s); c->d_Fd_off.upload(c->Fd_off, s); c->d_Fb_off.upload(c->Fb_off, s); c->d_Fdb_off.upload(c->Fdb_off, s);
  c->class_cache.clear();
  c->noalloc_classes.clear();
  c->corr_cache.clear();
  {
    // per-orbital F and F^dag slabs (the external operators of the single-particle correlator)
    std::vector<long> mo((size_t)n * n_blocks, -1), ko((size_t)n * n_blocks, -1);
    for (int o = 0; o < n; ++o) {
      const long sset = labels[o], qo = c->sinds[o];
      for (int b = 0; b < n_blocks; ++b) {
        const int tf = c->F_idx[sset * n_blocks + b], td = c->Fd_idx[sset * n_blocks + b];
        if (tf >= 0) mo[(size_t)o * n_blocks + b] = c->F_off[sset * n_blocks + b] + qo * block_dims[tf] * block_dims[b];
        if (td >= 0) ko[(size_t)o * n_blocks + b] = c->Fd_off[sset * n_blocks + b] + qo * block_dims[td] * block_dims[b];
      }
    }
    c->d_mu_off.upload(mo, s);
    c->d_ka_off.upload(ko, s);
    ExtOps &X = c->spgf_ops;
    X.nmu = X.nka = n;
    X.mu_idx.assign((size_t)n * n_blocks, -1);
    X.ka_idx.assign((size_t)n * n_blocks, -1);
    for (int o = 0; o < n; ++o)
      for (int b = 0; b < n_blocks; ++b) {
        X.mu_idx[(size_t)o * n_blocks + b] = c->F_idx[labels[o] * n_blocks + b];
        X.ka_idx[(size_t)o * n_blocks + b] = c->Fd_idx[labels[o] * n_blocks + b];
      }
    X.d_ops = c->d_ops.ptr;
    X.d_mu_off = c->d_mu_off.ptr;
    X.d_ka_off = c->d_ka_off.ptr;
    X.key = "spgf";
  }
  CUDA_CHECK(cudaStreamSynchronize(s));
  c->ready = true;
  API_END
}

int xca_num_self_energy_backbones(xca_ctx *ctx, int m, const int *topology, long *out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  parse_topology(m, topology);
  *out = (1L << m) * ipow(c->n, m - 1) * ipow(c->p, m - 1);
  API_END
}

int xca_num_single_ptcle_gf_backbones(xca_ctx *ctx, int m, const int *topology, long *out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  parse_topology(m, topology);
  *out = (1L << (m - 1)) * ipow(c->n, m - 1) * ipow(c->p, m - 1);
  API_END
}

int xca_compute_self_energy_device(xca_ctx *ctx, const double *G_dev, int m, const int *topology, double scale, double *Sigma_dev) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  set_device(c);
  Topology T = parse_topology(m, topology);
  GmaxFilter filter(c, block_max_async(c, G_dev));
  ClassSet *cs = get_classes(c, T, std::vector<int>(c->nb, 0));
  int nsig = prepare_tables(c, G_dev, m);
  launch_sigma(c, cs, G_dev, Sigma_dev, scale, nsig);
  API_END
}

int xca_compute_self_energy_device_batch(int n_jobs, xca_ctx *const *ctxs, const double *const *G_devs, const int *orders,
                                         const int *topologies, const double *scales, double *const *Sigma_devs) {
  API_BEGIN
  if (n_jobs < 1) throw Error(XCA_ERR_INVALID, "compute_self_energy_device_batch: no jobs");
  auto *c0 = reinterpret_cast<Ctx *>(ctxs[0]);
  for (int j = 0; j < n_jobs; ++j) {
    auto *c = reinterpret_cast<Ctx *>(ctxs[j]);
    if (!c || !c->ready) throw Error(XCA_ERR_INVALID, "compute_self_energy_device_batch: evaluator not set up");
    if (c->device != c0->device || c->RP != c0->RP)
      throw Error(XCA_ERR_INVALID, "compute_self_energy_device_batch: the jobs' contexts must share the device and the padded DLR rank");
    if (c->precision != XCA_PREC_FP64)
      throw Error(XCA_ERR_UNSUPPORTED, "compute_self_energy_device_batch: the batched launch sums with atomics (XCA_PREC_FP64)");
  }
  set_device(c0);
  // one preparation per context: its G's block norms (left on the device) and its edge tables in the layout
  // of the highest order among its jobs
  struct Prep {
    Ctx *c;
    const double *G;
    int maxm;
    int nsig;
    const double *gmax;
  };
  std::vector<Prep> preps;
  std::vector<int> prep_of(n_jobs);
  std::vector<ClassSet *> sets(n_jobs);
  for (int j = 0; j < n_jobs; ++j) {
    auto *c = reinterpret_cast<Ctx *>(ctxs[j]);
    size_t k = 0;
    while (k < preps.size() && preps[k].c != c) ++k;
    if (k == preps.size()) preps.push_back(Prep{c, G_devs[j], orders[j], 0, nullptr});
    if (preps[k].G != G_devs[j])
      throw Error(XCA_ERR_INVALID, "compute_self_energy_device_batch: the jobs of one context must share its G");
    preps[k].maxm = std::max(preps[k].maxm, orders[j]);
    prep_of[j] = (int)k;
    set_device(c);
    sets[j] = get_classes(c, parse_topology(orders[j], topologies + 6 * j), std::vector<int>(c->nb, 0));
  }
  for (Prep &pr : preps) {
    Ctx *c = pr.c;
    pr.gmax = block_max_async(c, pr.G);
    pr.nsig = prepare_tables(c, pr.G, pr.maxm);
    if (c != c0) {
      if (!c->ev_batch) CUDA_CHECK(cudaEventCreateWithFlags(&c->ev_batch, cudaEventDisableTiming));
      CUDA_CHECK(cudaEventRecord(c->ev_batch, c->stream));
      CUDA_CHECK(cudaStreamWaitEvent(c0->stream, c->ev_batch, 0));
    }
  }
  // the jobs' descriptors and their panel units, job by job, in one launch on the leading context's stream
  c0->h_batch_jobs.resize(n_jobs);
  c0->h_batch_units.clear();
  for (int j = 0; j < n_jobs; ++j) {
    const Prep &pr = preps[prep_of[j]];
    SigmaJob &J = c0->h_batch_jobs[j];
    std::memset(&J, 0, sizeof J);
    J.B = pr.c->basis(pr.nsig);
    J.B.gmax = pr.gmax;
    J.classes = sets[j]->d_classes.ptr;
    J.G = pr.G;
    J.out = atomic_out(Sigma_devs[j], scales[j]);
    for (WorkUnit w : sets[j]->units) {
      w.job = j;
      c0->h_batch_units.push_back(w);
    }
  }
  if (!c0->h_batch_units.empty()) {
    // device lists with headroom, so that a stream of slightly growing batches does not reallocate each time
    const size_t nj = c0->h_batch_jobs.size(), nu_ = c0->h_batch_units.size();
    if (nj > c0->d_batch_jobs.n) c0->d_batch_jobs.resize(nj + nj / 2);
    if (nu_ > c0->d_batch_units.n) c0->d_batch_units.resize(nu_ + nu_ / 2);
    c0->stage_jobs.copy(c0->d_batch_jobs.ptr, c0->h_batch_jobs.data(), nj * sizeof(SigmaJob), c0->stream);
    c0->stage_units.copy(c0->d_batch_units.ptr, c0->h_batch_units.data(), nu_ * sizeof(WorkUnit), c0->stream);
    c0->d_batch_counter.resize(1);
    const int nu = (int)c0->h_batch_units.size();
    switch (c0->RP) {
      case 32: c0->launches += launch_sigma_panel_batch<32>(c0->stream, c0->nsm, c0->d_batch_jobs.ptr, c0->d_batch_units.ptr, nu, c0->d_batch_counter.ptr); break;
      case 48: c0->launches += launch_sigma_panel_batch<48>(c0->stream, c0->nsm, c0->d_batch_jobs.ptr, c0->d_batch_units.ptr, nu, c0->d_batch_counter.ptr); break;
      default: c0->launches += launch_sigma_panel_batch<64>(c0->stream, c0->nsm, c0->d_batch_jobs.ptr, c0->d_batch_units.ptr, nu, c0->d_batch_counter.ptr); break;
    }
  }
  // chains too wide for a panel: the wide kernel of the job's context, after the batch
  if (!c0->ev_batch) CUDA_CHECK(cudaEventCreateWithFlags(&c0->ev_batch, cudaEventDisableTiming));
  CUDA_CHECK(cudaEventRecord(c0->ev_batch, c0->stream));
  for (const Prep &pr : preps)
    if (pr.c != c0) CUDA_CHECK(cudaStreamWaitEvent(pr.c->stream, c0->ev_batch, 0));
  for (int j = 0; j < n_jobs; ++j) {
    ClassSet *cs = sets[j];
    if (cs->wide_units.empty()) continue;
    const Prep &pr = preps[prep_of[j]];
    set_device(pr.c);
    GmaxFilter filter(pr.c, pr.gmax);
    launch_wide_units(pr.c, pr.c->basis(pr.nsig), cs->d_classes.ptr, cs->d_wide_units.ptr, (int)cs->wide_units.size(), cs->wide_slab,
                      pr.G, atomic_out(Sigma_devs[j], scales[j]));
  }
  API_END
}

int xca_compute_self_energy_device_shard(xca_ctx *ctx, const double *G_dev, int m, const int *topology, double scale,
                                         double *Sigma_dev, int shard, int n_shards) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  if (n_shards < 1 || shard < 0 || shard >= n_shards) throw Error(XCA_ERR_INVALID, "shard out of range");
  if (n_shards > 1 && c->precision == XCA_PREC_FP64_ORDERED)
    throw Error(XCA_ERR_UNSUPPORTED, "the ordered summation mode evaluates whole topologies on one device (n_shards must be 1)");
  set_device(c);
  Topology T = parse_topology(m, topology);
  GmaxFilter filter(c, block_max_async(c, G_dev));
  ClassSet *cs = get_classes(c, T, std::vector<int>(c->nb, 0));
  int nsig = prepare_tables(c, G_dev, m);
  if (n_shards == 1) {
    launch_sigma(c, cs, G_dev, Sigma_dev, scale, nsig);
  } else {
    auto key = std::make_pair(shard, n_shards);
    auto it = cs->shards.find(key);
    if (it == cs->shards.end()) {
      auto sub = std::make_unique<ClassSet>();
      sub->classes = cs->classes;
      for (size_t u = shard; u < cs->units.size(); u += n_shards) sub->units.push_back(cs->units[u]);
      for (size_t u = shard; u < cs->wide_units.size(); u += n_shards) sub->wide_units.push_back(cs->wide_units[u]);
      sub->wide_slab = cs->wide_slab;
      sub->d_classes.upload(sub->classes, c->stream);
      sub->d_units.upload(sub->units, c->stream);
      sub->d_wide_units.upload(sub->wide_units, c->stream);
      it = cs->shards.emplace(key, std::move(sub)).first;
    }
    launch_sigma(c, it->second.get(), G_dev, Sigma_dev, scale, nsig);
  }
  API_END
}

int xca_basis_setup(xca_ctx *ctx, double beta, double lambda, double eps, int r, const double *rf, const double *it,
                    int n_blocks, const int *block_dims) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  c->ready = false;
  setup_basis(c, beta, lambda, eps, r, rf, it, n_blocks, block_dims);
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  API_END
}

int xca_dyson_setup(xca_ctx *ctx, const double *G0) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  require_basis(c);
  set_device(c);
  c->dyson_ready = false;
  std::vector<double> g0;
  real_part(G0, c->slab, g0, "G0");
  // DLR coefficients of G0 (vals2coefs, dlr_dyson_ppsc.hpp:106) and their Hilbert transform W g0c
  std::vector<double> g0c = g0, g0t(c->slab, 0.0);
  const int r = c->r;
  c->woff.assign(c->nb, 0);
  c->moff.assign(c->nb, 0);
  long wo = 0, mo = 0;
  c->n_conv_rows = 0;
  for (int b = 0; b < c->nb; ++b) {
    const long dd = (long)c->dims[b] * c->dims[b];
    double *gc = g0c.data() + c->goff[b];
    lu_solve_recip(c->LU, c->Kdinv, r, c->piv, gc, dd);
    double *gt = g0t.data() + c->goff[b];
    for (int l = 0; l < r; ++l)
      for (int k = 0; k < r; ++k) {
        const double w = c->W[(size_t)l * r + k];
        for (long x = 0; x < dd; ++x) gt[l * dd + x] = std::fma(w, gc[k * dd + x], gt[l * dd + x]);
      }
    c->woff[b] = wo;
    wo += 6L * r * dd;
    c->moff[b] = mo;
    mo += (long)r * c->dims[b] * (long)r * c->dims[b];
    c->n_conv_rows = std::max(c->n_conv_rows, (long)r * dd);
  }
  cudaStream_t s = c->stream;
  c->d_g0.upload(g0, s); c->d_g0c.upload(g0c, s); c->d_g0t.upload(g0t, s);
  c->d_woff.upload(c->woff, s); c->d_moff.upload(c->moff, s);
  c->d_dwork.resize(std::max(wo, 1L));
  c->d_mats.resize(std::max(mo, 1L));
  c->d_rhs.resize(std::max(c->slab, 1L));
  c->d_red.resize(std::max(c->nb, 256));
  c->d_status.resize(1);
  CUDA_CHECK(cudaMemsetAsync(c->d_status.ptr, 0, sizeof(int), s));
  CUDA_CHECK(cudaStreamSynchronize(s));
  c->dyson_ready = true;
  API_END
}

int xca_dyson_solve(xca_ctx *ctx, const double *Sigma, double eta, int hermitize, double *G_out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  require_dyson(c);
  set_device(c);
  std::vector<double> sg;
  real_part(Sigma, c->slab, sg, "Sigma");
  c->d_Sig.resize(c->slab);
  c->d_G.resize(c->slab);
  CUDA_CHECK(cudaMemcpyAsync(c->d_Sig.ptr, sg.data(), c->slab * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  launch_dyson(c, c->d_Sig.ptr, eta, hermitize, c->d_G.ptr);
  std::vector<double> g(c->slab);
  CUDA_CHECK(cudaMemcpyAsync(g.data(), c->d_G.ptr, c->slab * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  check_dyson_status(c);
  for (long i = 0; i < c->slab; ++i) { G_out[2 * i] = g[i]; G_out[2 * i + 1] = 0.0; }
  API_END
}

int xca_dyson_solve_with_op(xca_ctx *ctx, const double *Sigma, double eta, const double *op, int hermitize, double *G_out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  require_dyson(c);
  set_device(c);
  long nop = 0;
  for (int b = 0; b < c->nb; ++b) nop += (long)c->dims[b] * c->dims[b];
  std::vector<double> sg, o;
  real_part(Sigma, c->slab, sg, "Sigma");
  real_part(op, nop, o, "op");
  c->d_Sig.resize(c->slab);
  c->d_G.resize(c->slab);
  c->d_op.resize(std::max(nop, 1L));
  CUDA_CHECK(cudaMemcpyAsync(c->d_Sig.ptr, sg.data(), c->slab * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CUDA_CHECK(cudaMemcpyAsync(c->d_op.ptr, o.data(), nop * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  launch_dyson(c, c->d_Sig.ptr, eta, hermitize, c->d_G.ptr, c->d_op.ptr);
  std::vector<double> g(c->slab);
  CUDA_CHECK(cudaMemcpyAsync(g.data(), c->d_G.ptr, c->slab * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  check_dyson_status(c);
  for (long i = 0; i < c->slab; ++i) { G_out[2 * i] = g[i]; G_out[2 * i + 1] = 0.0; }
  API_END
}

int xca_dyson_solve_device(xca_ctx *ctx, const double *Sigma_dev, double eta, int hermitize, double *G_dev) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  require_dyson(c);
  set_device(c);
  launch_dyson(c, Sigma_dev, eta, hermitize, G_dev);
  API_END
}

int xca_trace(xca_ctx *ctx, const double *G, double *tr_out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  require_basis(c);
  set_device(c);
  std::vector<double> g;
  real_part(G, c->slab, g, "G");
  c->d_G.resize(c->slab);
  CUDA_CHECK(cudaMemcpyAsync(c->d_G.ptr, g.data(), c->slab * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  tr_out[0] = trace_beta(c, c->d_G.ptr);
  tr_out[1] = 0.0;
  API_END
}

int xca_trace_device(xca_ctx *ctx, const double *G_dev, double *tr_out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  require_basis(c);
  set_device(c);
  tr_out[0] = trace_beta(c, G_dev);
  tr_out[1] = 0.0;
  API_END
}

int xca_normalize_device(xca_ctx *ctx, double *G_dev, double *Z, double *deta) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  require_basis(c);
  set_device(c);
  check_dyson_status(c);
  const double z = -trace_beta(c, G_dev);
  const double de = std::log(std::fabs(z)) / c->beta;
  // exp(-tau_t deta) per node on the host (libm, as the normalisation step's own arithmetic), then scaled
  std::vector<double> fac(c->r);
  for (int t = 0; t < c->r; ++t) fac[t] = std::exp(-((c->beta * c->tabs[t]) * de));
  c->d_efac.resize(c->r);
  CUDA_CHECK(cudaMemcpyAsync(c->d_efac.ptr, fac.data(), c->r * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  c->launches += launch_energy_shift(c->stream, dyson_basis(c), G_dev, c->d_efac.ptr);
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  *Z = z;
  *deta = de;
  API_END
}

int xca_max_abs_diff_device(xca_ctx *ctx, const double *a_dev, const double *b_dev, double *out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  require_basis(c);
  set_device(c);
  const int blocks = 256;
  c->d_red.resize(std::max(c->nb, blocks));
  c->launches += launch_max_abs_diff(c->stream, blocks, a_dev, b_dev, c->slab, c->d_red.ptr);
  std::vector<double> part(blocks);
  CUDA_CHECK(cudaMemcpyAsync(part.data(), c->d_red.ptr, blocks * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  double m = 0.0;
  for (double x : part) m = std::max(m, x);
  *out = m;
  API_END
}

int xca_axpby_device(xca_ctx *ctx, double alpha, const double *x_dev, double beta, double *y_dev) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  require_basis(c);
  set_device(c);
  const long n = c->slab;
  c->launches += launch_axpby(c->stream, alpha, x_dev, beta, y_dev, n);
  API_END
}

int xca_compute_single_ptcle_gf_device(xca_ctx *ctx, const double *G_dev, int m, const int *topology, double scale, double *g_dev) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  set_device(c);
  Topology T = parse_topology(m, topology);
  auto zero = zero_flags_device(c, G_dev);
  CorrSet *cs = get_corr(c, T, zero, c->spgf_ops);
  int nsig = prepare_tables(c, G_dev, m);
  launch_corr(c, cs, c->spgf_ops, cs->d_units.ptr, (int)cs->units.size(), G_dev, g_dev, scale, nsig);
  API_END
}

int xca_compute_single_ptcle_gf(xca_ctx *ctx, const double *G, int m, const int *topology, const long *f_ix, long n_fix, double *g_out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  set_device(c);
  correlator_host(c, G, m, topology, f_ix, n_fix, c->spgf_ops, g_out, "compute_single_ptcle_gf");
  API_END
}

int xca_convolve_ppsc(xca_ctx *ctx, const double *G1, const double *G2, double *H_out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  require_basis(c);
  set_device(c);
  std::vector<double> a, b;
  real_part(G1, c->slab, a, "G1");
  real_part(G2, c->slab, b, "G2");
  c->d_ba.resize(c->slab);
  c->d_bb.resize(c->slab);
  c->d_bc.resize(c->slab);
  CUDA_CHECK(cudaMemcpyAsync(c->d_ba.ptr, a.data(), c->slab * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CUDA_CHECK(cudaMemcpyAsync(c->d_bb.ptr, b.data(), c->slab * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  launch_convolve_blocks(c, c->d_ba.ptr, c->d_bb.ptr, c->d_bc.ptr);
  std::vector<double> h(c->slab);
  CUDA_CHECK(cudaMemcpyAsync(h.data(), c->d_bc.ptr, c->slab * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  for (long i = 0; i < c->slab; ++i) { H_out[2 * i] = h[i]; H_out[2 * i + 1] = 0.0; }
  API_END
}

int xca_convolve_ppsc_device(xca_ctx *ctx, const double *G1_dev, const double *G2_dev, double *H_dev) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  require_basis(c);
  set_device(c);
  launch_convolve_blocks(c, G1_dev, G2_dev, H_dev);
  API_END
}

int xca_expectation_value(xca_ctx *ctx, const double *G, const int *op_index, const double *op_data, double *out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  require_basis(c);
  set_device(c);
  std::vector<long> off(c->nb, -1);
  long pos = 0;
  for (int b = 0; b < c->nb; ++b) {
    const int t = op_index[b];
    if (t == -1) continue;
    if (t != b) throw Error(XCA_ERR_INVALID, "expectation_value: the operator must be block diagonal (connection[b] == b)");
    off[b] = pos;
    pos += (long)c->dims[b] * c->dims[b];
  }
  std::vector<double> ops;
  real_part(op_data, pos, ops, "operator");
  std::vector<double> g;
  real_part(G, c->slab, g, "G");
  c->d_ba.resize(c->slab);
  c->d_xop.resize(std::max(pos, 1L));
  c->d_xop_off.upload(off, c->stream);
  c->d_red.resize(std::max(c->nb, 256));
  CUDA_CHECK(cudaMemcpyAsync(c->d_ba.ptr, g.data(), c->slab * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (pos) CUDA_CHECK(cudaMemcpyAsync(c->d_xop.ptr, ops.data(), pos * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  const DysonBasis B = block_op_basis(c);
  switch (c->RP) {
    case 32: c->launches += launch_expectation_beta<32>(c->stream, B, c->d_ba.ptr, c->d_xop.ptr, c->d_xop_off.ptr, c->d_red.ptr); break;
    case 48: c->launches += launch_expectation_beta<48>(c->stream, B, c->d_ba.ptr, c->d_xop.ptr, c->d_xop_off.ptr, c->d_red.ptr); break;
    default: c->launches += launch_expectation_beta<64>(c->stream, B, c->d_ba.ptr, c->d_xop.ptr, c->d_xop_off.ptr, c->d_red.ptr); break;
  }
  std::vector<double> part(c->nb);
  CUDA_CHECK(cudaMemcpyAsync(part.data(), c->d_red.ptr, c->nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  // sum += -trace(O_b G_b(beta)) block after block (block_sparse.cpp:805-813)
  double sum = 0.0;
  for (int b = 0; b < c->nb; ++b)
    if (off[b] >= 0) sum += -part[b];
  out[0] = sum;
  out[1] = 0.0;
  API_END
}

int xca_compute_one_time_correlator(xca_ctx *ctx, const double *G, int n_tau, const int *tau_index, const double *tau_data, int n_0,
                                    const int *zero_index, const double *zero_data, int m, const int *topology, const long *f_ix,
                                    long n_fix, double *corr_out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  if (n_tau < 1 || n_0 < 1) throw Error(XCA_ERR_INVALID, "compute_one_time_correlator: empty operator list");
  set_device(c);
  const int nb = c->nb;
  ExtOps X;
  X.nmu = n_tau;
  X.nka = n_0;
  X.mu_idx.assign(tau_index, tau_index + (size_t)n_tau * nb);
  X.ka_idx.assign(zero_index, zero_index + (size_t)n_0 * nb);
  // operator slabs: the ops at tau, then the ops at 0, each a (d_target x d_b) block per present column
  std::vector<long> mo((size_t)n_tau * nb, -1), ko((size_t)n_0 * nb, -1);
  std::vector<double> data;
  std::ostringstream key;
  key << "ot" << n_tau << ":" << n_0;
  auto load = [&](int nops, const std::vector<int> &idx, const double *src, std::vector<long> &offs, const char *what) {
    long pos = 0;
    for (int o = 0; o < nops; ++o)
      for (int b = 0; b < nb; ++b) {
        const int t = idx[(size_t)o * nb + b];
        key << "," << t;
        if (t == -1) continue;
        if (t < -1 || t >= nb) throw Error(XCA_ERR_INVALID, std::string(what) + ": block index out of range");
        const long sz = (long)c->dims[t] * c->dims[b];
        offs[(size_t)o * nb + b] = (long)data.size();
        std::vector<double> re;
        real_part(src + 2 * pos, sz, re, what);
        data.insert(data.end(), re.begin(), re.end());
        pos += sz;
      }
  };
  load(n_tau, X.mu_idx, tau_data, mo, "ops_tau");
  load(n_0, X.ka_idx, zero_data, ko, "ops_0");
  X.key = key.str();
  c->d_xops.upload(data, c->stream);
  c->d_xmu_off.upload(mo, c->stream);
  c->d_xka_off.upload(ko, c->stream);
  X.d_ops = c->d_xops.ptr;
  X.d_mu_off = c->d_xmu_off.ptr;
  X.d_ka_off = c->d_xka_off.ptr;
  correlator_host(c, G, m, topology, f_ix, n_fix, X, corr_out, "compute_one_time_correlator");
  API_END
}

int xca_zero_device(xca_ctx *ctx, double *dev, long n) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  zero_kernel<<<std::max<long>(1, std::min<long>(1184, (n + 255) / 256)), 256, 0, c->stream>>>(dev, n);
  c->launches++;
  CUDA_CHECK(cudaGetLastError());
  API_END
}

int xca_compute_self_energy(xca_ctx *ctx, const double *G, int m, const int *topology, const long *f_ix, long n_fix, double *Sigma_out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  set_device(c);
  Topology T = parse_topology(m, topology);
  long nmaxb = (1L << m) * ipow(c->n, m - 1) * ipow(c->p, m - 1);
  std::vector<double> g;
  real_part(G, c->slab, g, "G");
  c->d_G.resize(c->slab);
  c->d_Sig.resize(c->slab);
  CUDA_CHECK(cudaMemcpyAsync(c->d_G.ptr, g.data(), c->slab * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  zero_kernel<<<64, 256, 0, c->stream>>>(c->d_Sig.ptr, c->slab);
  c->launches++;
  auto zero = zero_flags_device(c, c->d_G.ptr);
  ClassSet *cs = get_classes(c, T, zero);
  int nsig = prepare_tables(c, c->d_G.ptr, m);
  if (f_ix == nullptr) {
    launch_sigma(c, cs, c->d_G.ptr, c->d_Sig.ptr, 1.0, nsig);
  } else {
    // subset of flat indices: build a dedicated unit list (one unit per listed f_ix and valid class)
    const long omax = ipow(c->n, m - 1), npt = ipow(c->p, m - 1);
    std::vector<WorkUnit> units;
    for (long z = 0; z < n_fix; ++z) {
      long f = f_ix[z];
      if (f < 0 || f >= nmaxb) throw Error(XCA_ERR_RUNTIME, "DiagramEvaluator::eval_self_energy: f_ix out of range");
      long o = f % omax, q = f / omax;
      long pix = q % npt, fb = q / npt;
      for (int k : cs->by_fbo[fb * omax + o]) units.push_back(WorkUnit{k, (int)pix, 1});
    }
    if (!units.empty() && c->precision == XCA_PREC_FP64_ORDERED) {
      // every (flat index, class) item its own group, in list order: the sequential order of the list
      std::vector<int> grp(units.size());
      for (size_t u = 0; u < units.size(); ++u) grp[u] = (int)u;
      auto P = make_plan(c, cs->classes, units, grp);
      launch_sigma_plan(c, cs->classes, cs->d_classes.ptr, P.get(), c->d_G.ptr, c->d_Sig.ptr, 1.0, nsig);
      CUDA_CHECK(cudaStreamSynchronize(c->stream));
    } else if (!units.empty()) {
      ClassSet tmp;
      tmp.classes = cs->classes;
      for (const WorkUnit &w : units) {
        const ClassRec &R = cs->classes[w.cls];
        (R.wide ? tmp.wide_units : tmp.units).push_back(w);
        if (R.wide) tmp.wide_slab = std::max(tmp.wide_slab, (long)c->r * R.dcmax);
      }
      tmp.d_classes.upload(tmp.classes, c->stream);
      tmp.d_units.upload(tmp.units, c->stream);
      tmp.d_wide_units.upload(tmp.wide_units, c->stream);
      launch_sigma(c, &tmp, c->d_G.ptr, c->d_Sig.ptr, 1.0, nsig);
      CUDA_CHECK(cudaStreamSynchronize(c->stream));
    }
  }
  std::vector<double> out(c->slab);
  CUDA_CHECK(cudaMemcpyAsync(out.data(), c->d_Sig.ptr, c->slab * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  // blocks that end below 1e-16 come back as exact zeros (set_zero_block_indices, bsb.cpp:386-395)
  for (int b = 0; b < c->nb; ++b) {
    long o = c->goff[b], sz = (long)c->r * c->dims[b] * c->dims[b];
    double mx = 0;
    for (long i = 0; i < sz; ++i) mx = std::max(mx, std::fabs(out[o + i]));
    if (mx < 1e-16)
      for (long i = 0; i < sz; ++i) out[o + i] = 0.0;
  }
  for (long i = 0; i < c->slab; ++i) {
    Sigma_out[2 * i] = out[i];
    Sigma_out[2 * i + 1] = 0.0;
  }
  API_END
}

int xca_self_energy_items(xca_ctx *ctx, const double *G, int m, const int *topology, long *rows, long max_rows, long *n_items) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  Topology T = parse_topology(m, topology);
  std::vector<double> g;
  real_part(G, c->slab, g, "G");
  std::vector<int> zero(c->nb);
  for (int b = 0; b < c->nb; ++b) {
    long o = c->goff[b], sz = (long)c->r * c->dims[b] * c->dims[b];
    double mx = 0;
    for (long i = 0; i < sz; ++i) mx = std::max(mx, std::fabs(g[o + i]));
    zero[b] = mx < 1e-16;
  }
  set_device(c);
  ClassSet *cs = get_classes(c, T, zero);
  const long omax = ipow(c->n, m - 1), npt = ipow(c->p, m - 1), fbmax = 1L << m;
  const int width = 3 + 2 * m - 1;
  long count = 0;
  for (long fb = 0; fb < fbmax; ++fb)
    for (long pix = 0; pix < npt; ++pix)
      for (long o = 0; o < omax; ++o) {
        const auto &lst = cs->by_fbo[fb * omax + o];
        if (!rows || count >= max_rows) {
          count += (long)lst.size();
          continue;
        }
        long f = o + omax * (pix + npt * fb);
        for (int k : lst) {
          if (count < max_rows) {
            long *rw = rows + count * width;
            const ClassRec &R = cs->classes[k];
            rw[0] = f; rw[1] = R.b_out; rw[2] = R.pk;
            for (int i = 0; i < 2 * m - 1; ++i) rw[3 + i] = R.ind_path[i];
          }
          count++;
        }
      }
  *n_items = count;
  API_END
}

int xca_self_energy_flops(xca_ctx *ctx, const double *G, int m, const int *topology, double *alg_flops, long *n_items) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  Topology T = parse_topology(m, topology);
  std::vector<double> g;
  real_part(G, c->slab, g, "G");
  std::vector<int> zero(c->nb);
  for (int b = 0; b < c->nb; ++b) {
    long o = c->goff[b], sz = (long)c->r * c->dims[b] * c->dims[b];
    double mx = 0;
    for (long i = 0; i < sz; ++i) mx = std::max(mx, std::fabs(g[o + i]));
    zero[b] = mx < 1e-16;
  }
  set_device(c);
  ClassSet *cs = get_classes(c, T, zero);
  // count pole tuples per case pattern: a line's case depends on its direction and its pole's sign
  const int p = c->p;
  long nA[2] = {0, 0};
  for (int l = 0; l < p; ++l) {
    if (c->polesb[l] <= 0.0) nA[1]++;  // forward line, case A
    if (c->polesb[l] >= 0.0) nA[0]++;  // backward line, case A
  }
  double tot = 0;
  for (const ClassRec &R : cs->classes) {
    int nl = m - 1;
    for (int mask = 0; mask < (1 << nl); ++mask) {
      int caseA[MAXM] = {0, 0, 0};
      double count = 1;
      for (int i = 1; i < m; ++i) {
        int fwd = (R.fbmask >> i) & 1;
        caseA[i] = (mask >> (i - 1)) & 1;
        long a = nA[fwd];
        count *= caseA[i] ? a : (p - a);
      }
      if (count > 0) tot += count * item_flops(c, R, caseA);
    }
  }
  *alg_flops = tot;
  *n_items = (long)cs->n_items;
  API_END
}

int xca_profile(xca_ctx *ctx, int enable, double *sigma_ms, long *sigma_launches) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  double ms = 0;
  long n = 0;
  if (!c->prof_events.empty()) {
    CUDA_CHECK(cudaStreamSynchronize(c->stream));
    for (auto &e : c->prof_events) {
      float x = 0;
      CUDA_CHECK(cudaEventElapsedTime(&x, e.first, e.second));
      ms += x;
      n++;
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
    c->prof_events.clear();
  }
  c->profile = enable != 0;
  if (sigma_ms) *sigma_ms = ms;
  if (sigma_launches) *sigma_launches = n;
  API_END
}

int xca_event_record(xca_ctx *ctx, int slot) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  if (slot < 0 || slot >= 8) throw Error(XCA_ERR_INVALID, "event slot out of range");
  if (!c->user_events[slot]) CUDA_CHECK(cudaEventCreate(&c->user_events[slot]));
  CUDA_CHECK(cudaEventRecord(c->user_events[slot], c->stream));
  API_END
}

int xca_event_elapsed(xca_ctx *ctx, int slot_a, int slot_b, double *ms) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  if (slot_a < 0 || slot_a >= 8 || slot_b < 0 || slot_b >= 8 || !c->user_events[slot_a] || !c->user_events[slot_b])
    throw Error(XCA_ERR_INVALID, "event slot not recorded");
  CUDA_CHECK(cudaEventSynchronize(c->user_events[slot_b]));
  float x = 0;
  CUDA_CHECK(cudaEventElapsedTime(&x, c->user_events[slot_a], c->user_events[slot_b]));
  *ms = x;
  API_END
}

int xca_flush_l2(xca_ctx *ctx, long bytes) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  long n = (bytes + 7) / 8;
  c->d_flush.resize(n);
  zero_kernel<<<1184, 256, 0, c->stream>>>(c->d_flush.ptr, n);
  CUDA_CHECK(cudaGetLastError());
  API_END
}

int xca_fp64_fma_probe(xca_ctx *ctx, double *tflops) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  const int blocks = nsm * 8, threads = 256, iters = 8192;
  c->d_flush.resize((size_t)blocks * threads);
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  fp64_fma_probe_kernel<<<blocks, threads, 0, c->stream>>>(c->d_flush.ptr, iters, 0.999999, 1e-7);
  CUDA_CHECK(cudaEventRecord(e0, c->stream));
  for (int rep = 0; rep < 5; ++rep) fp64_fma_probe_kernel<<<blocks, threads, 0, c->stream>>>(c->d_flush.ptr, iters, 0.999999, 1e-7);
  CUDA_CHECK(cudaEventRecord(e1, c->stream));
  CUDA_CHECK(cudaEventSynchronize(e1));
  float ms = 0;
  CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *tflops = 5.0 * 2.0 * 8.0 * iters * (double)blocks * threads / (ms * 1e-3) / 1e12;
  API_END
}

int xca_fp64_mma_probe(xca_ctx *ctx, double *tflops) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  const int blocks = nsm * 4, threads = 256, iters = 4096;
  c->d_flush.resize((size_t)blocks * threads);
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  fp64_mma_probe_kernel<<<blocks, threads, 0, c->stream>>>(c->d_flush.ptr, iters, 0.999999, 1e-7);
  CUDA_CHECK(cudaEventRecord(e0, c->stream));
  for (int rep = 0; rep < 5; ++rep) fp64_mma_probe_kernel<<<blocks, threads, 0, c->stream>>>(c->d_flush.ptr, iters, 0.999999, 1e-7);
  CUDA_CHECK(cudaEventRecord(e1, c->stream));
  CUDA_CHECK(cudaEventSynchronize(e1));
  float ms = 0;
  CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // 8 MMAs of 8 x 8 x 4 (512 flops) per warp and iteration
  *tflops = 5.0 * 8.0 * 512.0 * iters * ((double)blocks * threads / 32) / (ms * 1e-3) / 1e12;
  API_END
}

int xca_fp64_mma_selftest(xca_ctx *ctx, long n_tiles, unsigned long long seed, long *mismatches) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  if (n_tiles < 1) throw Error(XCA_ERR_INVALID, "n_tiles must be positive");
  DevBuf<unsigned long long> cnt;
  cnt.resize(1);
  CUDA_CHECK(cudaMemsetAsync(cnt.ptr, 0, sizeof(unsigned long long), c->stream));
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  fp64_mma_selftest_kernel<<<nsm * 4, 256, 0, c->stream>>>(n_tiles, seed, cnt.ptr);
  c->launches++;
  CUDA_CHECK(cudaGetLastError());
  unsigned long long h = 0;
  CUDA_CHECK(cudaMemcpyAsync(&h, cnt.ptr, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  *mismatches = (long)h;
  API_END
}

int xca_slab_info(xca_ctx *ctx, long *n_doubles, int *r) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  *n_doubles = c->slab;
  *r = c->r;
  API_END
}

int xca_device_buffer(xca_ctx *ctx, int slot, long bytes, double **dev_ptr) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  if (slot < 0 || slot > 63) throw Error(XCA_ERR_INVALID, "buffer slot out of range");
  while ((int)c->user_bufs.size() <= slot) c->user_bufs.emplace_back(new DevBuf<double>());
  c->user_bufs[slot]->resize((bytes + 7) / 8);
  *dev_ptr = c->user_bufs[slot]->ptr;
  API_END
}

int xca_copy_to_device(xca_ctx *ctx, double *dev, const double *host, long n) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  CUDA_CHECK(cudaMemcpyAsync(dev, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  API_END
}

int xca_copy_to_host(xca_ctx *ctx, double *host, const double *dev, long n) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  CUDA_CHECK(cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  API_END
}

int xca_synchronize(xca_ctx *ctx) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  API_END
}

int xca_set_precision_mode(xca_ctx *ctx, int mode) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (mode != XCA_PREC_FP64 && mode != XCA_PREC_FP64_ORDERED && mode != XCA_PREC_FP32)
    throw Error(XCA_ERR_UNSUPPORTED, "precision mode " + std::to_string(mode) + " is not available");
  c->precision = mode;
  API_END
}

int xca_set_tuning(xca_ctx *ctx, int param, int value) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  int *slot = nullptr;
  int lo = 1, hi = 1;
  switch (param) {
    case XCA_TUNE_UNIT_BATCHES: slot = &c->unit_batches; hi = 64; break;
    case XCA_TUNE_WIDE_UNIT_TUPLES: slot = &c->wide_unit_tuples; hi = 1024; break;
    case XCA_TUNE_WIDE_CTAS_PER_SM: slot = &c->wide_ctas_per_sm; hi = 8; break;
    case XCA_TUNE_DYSON_BLOCKED_MIN_N: slot = &c->dyson_blocked_min_n; lo = 0; hi = 1 << 30; break;
    default: throw Error(XCA_ERR_INVALID, "unknown tuning parameter " + std::to_string(param));
  }
  if (value < lo || value > hi)
    throw Error(XCA_ERR_INVALID, "tuning value " + std::to_string(value) + " out of range [" + std::to_string(lo) + ", " +
                                     std::to_string(hi) + "]");
  if (*slot != value) {
    *slot = value;
    if (param != XCA_TUNE_DYSON_BLOCKED_MIN_N) {
      c->class_cache.clear();  // work lists are cut with these sizes
      c->noalloc_classes.clear();
    }
  }
  API_END
}

int xca_get_tuning(xca_ctx *ctx, int param, int *value) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  switch (param) {
    case XCA_TUNE_UNIT_BATCHES: *value = c->unit_batches; break;
    case XCA_TUNE_WIDE_UNIT_TUPLES: *value = c->wide_unit_tuples; break;
    case XCA_TUNE_WIDE_CTAS_PER_SM: *value = c->wide_ctas_per_sm; break;
    case XCA_TUNE_DYSON_BLOCKED_MIN_N: *value = c->dyson_blocked_min_n; break;
    default: throw Error(XCA_ERR_INVALID, "unknown tuning parameter " + std::to_string(param));
  }
  API_END
}

int xca_get_precision_mode(xca_ctx *ctx, int *mode) {
  API_BEGIN
  *mode = reinterpret_cast<Ctx *>(ctx)->precision;
  API_END
}

int xca_device_allocations(long *out) {
  API_BEGIN
  *out = g_device_allocations.load(std::memory_order_relaxed);
  API_END
}

int xca_kernel_launches(xca_ctx *ctx, long *out) {
  API_BEGIN
  *out = reinterpret_cast<Ctx *>(ctx)->launches;
  API_END
}

int xca_compute_self_energy_device_noalloc(xca_ctx *ctx, const double *G_dev, int m, const int *topology, double scale,
                                           double *Sigma_dev) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  set_device(c);
  Topology T = parse_topology(m, topology);
  unsigned char *base = noalloc_scratch(c->device);
  const int nb = c->nb, r = c->r;
  const int nsig = (m >= 3) ? (int)c->nsig_alloc : 1 + 2 * c->p;
  const std::vector<int2> chunks = table_chunks(c, nsig);
  // layout: unit counter | block max |G| | edge-table offsets | table chunks | edge tables | path classes | work units
  const size_t off_counter = 0;
  const size_t off_maxabs = 256;
  const size_t off_taboff = off_maxabs + align256((size_t)nb * sizeof(double));
  const size_t off_chunks = off_taboff + align256((size_t)nb * sizeof(long));
  const size_t off_tab = off_chunks + align256(chunks.size() * sizeof(int2));
  std::vector<long> tab_off(nb);
  long tab_doubles = 0;
  for (int b = 0; b < nb; ++b) {
    tab_off[b] = tab_doubles;
    tab_doubles += (long)nsig * 2L * r * c->dims[b] * c->dims[b];
  }
  const size_t off_classes = off_tab + align256((size_t)tab_doubles * sizeof(double));
  noalloc_fits(off_classes, "the edge tables of this topology order");
  // zero-block flags of G (max |G_b| < 1e-16: c++/triqs_xca/block_sparse.cpp:45-49, used at block_sparse_backbone.cpp:248)
  double *maxabs = reinterpret_cast<double *>(base + off_maxabs);
  block_maxabs_kernel<<<nb, 256, 0, c->stream>>>(G_dev, c->d_goff.ptr, c->d_dims.ptr, r, nb, maxabs);
  c->launches++;
  CUDA_CHECK(cudaGetLastError());
  std::vector<double> mx(nb);
  CUDA_CHECK(cudaMemcpyAsync(mx.data(), maxabs, nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  std::vector<int> zero(nb);
  for (int b = 0; b < nb; ++b) zero[b] = mx[b] < 1e-16 ? 1 : 0;
  // host work list, cached per (topology, zero pattern)
  const std::string key = class_key(T, zero);
  // the allocating path's cached work list when it has built one (its host vectors only), else a host-only one
  const ClassSet *cs = nullptr;
  auto itk = c->class_cache.find(key);
  if (itk != c->class_cache.end()) {
    cs = itk->second.get();
  } else {
    auto itc = c->noalloc_classes.find(key);
    if (itc == c->noalloc_classes.end()) itc = c->noalloc_classes.emplace(key, build_classes(c, T, zero)).first;
    cs = itc->second.get();
  }
  if (!cs->wide_units.empty())
    throw Error(XCA_ERR_UNSUPPORTED, "xca_compute_self_energy_device_noalloc: block chains wider than the panel kernel's panel are "
                                     "not supported; use xca_compute_self_energy_device");
  const size_t off_units = off_classes + align256(cs->classes.size() * sizeof(ClassRec));
  noalloc_fits(off_units + cs->units.size() * sizeof(WorkUnit), "the edge tables and work list of this topology");
  // contents: everything is rewritten before use except the unit counter, which must start at zero
  auto *d_tab_off = reinterpret_cast<long *>(base + off_taboff);
  auto *d_chunks = reinterpret_cast<int2 *>(base + off_chunks);
  auto *d_classes = reinterpret_cast<ClassRec *>(base + off_classes);
  auto *d_units = reinterpret_cast<WorkUnit *>(base + off_units);
  auto *counter = reinterpret_cast<int *>(base + off_counter);
  CUDA_CHECK(cudaMemcpyAsync(d_tab_off, tab_off.data(), nb * sizeof(long), cudaMemcpyHostToDevice, c->stream));
  CUDA_CHECK(cudaMemcpyAsync(d_chunks, chunks.data(), chunks.size() * sizeof(int2), cudaMemcpyHostToDevice, c->stream));
  if (!cs->classes.empty())
    CUDA_CHECK(cudaMemcpyAsync(d_classes, cs->classes.data(), cs->classes.size() * sizeof(ClassRec), cudaMemcpyHostToDevice,
                               c->stream));
  if (!cs->units.empty())
    CUDA_CHECK(cudaMemcpyAsync(d_units, cs->units.data(), cs->units.size() * sizeof(WorkUnit), cudaMemcpyHostToDevice,
                               c->stream));
  DevBasis B = c->basis(nsig);
  B.tab = reinterpret_cast<const double *>(base + off_tab);
  B.tab_off = d_tab_off;
  launch_tables(c, G_dev, nsig, d_chunks, (int)chunks.size(), B);
  if (!cs->units.empty())
    launch_sigma_units(c, B, d_classes, d_units, (int)cs->units.size(), counter, G_dev, atomic_out(Sigma_dev, scale));
  API_END
}

}  // extern "C"
