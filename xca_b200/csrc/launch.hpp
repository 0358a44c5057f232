// Host-side launchers of the device kernels, one translation unit per kernel family and padded rank
// (sigma_rp.cu and spgf_rp.cu are compiled once per RP in {32, 48, 64}; dyson.cu holds every rank).
// The context code in xca_b200.cu calls these; each returns the number of kernels it launched.
#pragma once
#include <cuda_runtime.h>

#include "sigma_kernel.cuh"
#include "spgf_kernel.cuh"

namespace xca {

template <int RP>
int launch_edge_tables(cudaStream_t s, int nsm, const DevBasis &B, const double *G, const int2 *chunks, int n_chunks);

template <int RP>
int launch_sigma_panel(cudaStream_t s, int nsm, const DevBasis &B, const ClassRec *classes, const WorkUnit *units, int n_units,
                       int *counter, const double *G, const SigmaOut &out);

// Job-batched panel kernel: units of several jobs (SigmaJob) in one persistent launch.
template <int RP>
int launch_sigma_panel_batch(cudaStream_t s, int nsm, const SigmaJob *jobs, const WorkUnit *units, int n_units, int *counter);

// FP32 Sigma kernel (sigma_f32.cuh) over the panel classes' units: fast (atomic) output into FP64 Sigma.
template <int RP>
int launch_sigma_f32(cudaStream_t s, int nsm, const DevBasis &B, const ClassRec *classes, const WorkUnit *units, int n_units, int *counter,
                     const double *G, const SigmaOut &out);

// Wide-chain Sigma kernel (sigma_wide.cuh) over n_units units with `grid` CTAs; each CTA's region of scratch
// is cta_doubles long and holds 3 + (largest symmetry set) slabs of `slab` doubles.
template <int RP>
int launch_sigma_wide(cudaStream_t s, int grid, const DevBasis &B, const ClassRec *classes, const WorkUnit *units, int n_units,
                      int *counter, const double *G, const SigmaOut &out, double *scratch, long slab, long cta_doubles);

// Usable panel columns of the panel kernels of rank RP.
template <int RP>
int panel_width();

template <int RP>
int launch_correlator(cudaStream_t s, int grid, int warps_per_cta, const DevBasis &B, const CorrBasis &CB, const CorrClass *classes,
                      const CorrChain *chains, const CorrTerm *terms, const WorkUnit *units, int n_units, int *counter,
                      const double *G, double *g, double scale, int nmax, double *scratch, long warp_doubles);

// Default threshold: when the largest system (N = r d_b) exceeds blocked_min_n, every block is factorised by
// the blocked kernels, else by one CTA each (the results are the same bit for bit).
constexpr int DYSON_BLOCKED_MIN_N = 192;
// One-CTA systems whose matrix and right-hand sides fit these bounds are factorised in shared memory.
constexpr int DYSON_SMEM_MAX_N = 192;
constexpr size_t DYSON_SMEM_MAX_BYTES = 220 * 1024;

template <int RP>
int launch_dyson(cudaStream_t s, const DysonBasis &B, long n_conv_rows, const double *Sigma, double eta, int hermitize, double *rhs,
                 double *G, int *status, int n_max, int d_max, int blocked_min_n, const double *op = nullptr);

template <int RP>
int launch_trace_beta(cudaStream_t s, const DysonBasis &B, const double *G, double *out);

template <int RP>
int launch_convolve_ppsc(cudaStream_t s, const DysonBasis &B, const double *G1, const double *G2, double *H);

template <int RP>
int launch_expectation_beta(cudaStream_t s, const DysonBasis &B, const double *G, const double *ops, const long *op_off, double *out);

int launch_energy_shift(cudaStream_t s, const DysonBasis &B, double *G, const double *fac);
int launch_max_abs_diff(cudaStream_t s, int blocks, const double *a, const double *b, long n, double *out);
int launch_axpby(cudaStream_t s, double alpha, const double *x, double beta, double *y, long n);

}  // namespace xca
