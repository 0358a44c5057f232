// C++ face of libxca_b200 with the reference's class and method names, for C++ callers of TRIQS/xca's
// evaluator (c++/triqs_xca/block_sparse_backbone.hpp:23-165) and Dyson solver
// (c++/triqs_xca/dlr_dyson_ppsc.hpp:45-231).  Header only; link with -lxca_b200.
//
// TRIQS containers are not required: a block Green's function is a BlockGf, one std::vector of
// complex<double> per Fock-space block holding an (r, d_b, d_b) array (tau node slowest), and a topology
// is a list of vertex pairs.  Failing calls throw the reference's exception types: std::invalid_argument
// for XCA_ERR_INVALID (shape and symmetry-set violations) and std::runtime_error for everything else (an
// f_ix out of range, CUDA errors, unsupported sizes).
#pragma once

#include <array>
#include <complex>
#include <stdexcept>
#include <string>
#include <vector>

#include "xca_b200.h"

namespace xca_b200 {

using dcomplex = std::complex<double>;
using BlockGf = std::vector<std::vector<dcomplex>>;
using Topology = std::vector<std::array<int, 2>>;

inline void check(int status) {
  if (status == XCA_OK) return;
  const std::string msg = xca_last_error();
  if (status == XCA_ERR_INVALID) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

namespace detail {
inline std::vector<int> flat(const Topology &t) {
  std::vector<int> v;
  for (const auto &p : t) {
    v.push_back(p[0]);
    v.push_back(p[1]);
  }
  return v;
}
inline std::vector<dcomplex> pack(const BlockGf &G) {
  std::vector<dcomplex> v;
  for (const auto &b : G) v.insert(v.end(), b.begin(), b.end());
  return v;
}
inline const double *dp(const std::vector<dcomplex> &v) { return reinterpret_cast<const double *>(v.data()); }
inline double *dp(std::vector<dcomplex> &v) { return reinterpret_cast<double *>(v.data()); }
}  // namespace detail

namespace block_sparse {

// BlockOpSymQuartet's input (c++/triqs_xca/block_sparse.hpp:181-291): symmetry-set label per orbital, and
// for F and F^dag the target block of set s on block column b (index[s * n_blocks + b], -1: none) with the
// (q_s, d_target, d_b) slabs of the present columns packed in (s, b) order.
struct BlockOpSymQuartet {
  std::vector<long> sym_set_labels;
  std::vector<int> dims;
  std::vector<int> F_index, Fd_index;
  std::vector<dcomplex> F_data, Fd_data;
};

// A block operator (BlockOp): the block each column maps to (-1: none) and its (d_target x d_b) block.
struct BlockOp {
  std::vector<int> index;
  std::vector<std::vector<dcomplex>> blocks;
};

class DiagramEvaluator {
 public:
  // DiagramEvaluator(beta, Lambda, eps, hyb_poles, hyb_coeffs, Fq), block_sparse_backbone.hpp:158-162.
  // hyb_coeffs is p x n x n.
  DiagramEvaluator(double beta, double Lambda, double eps, const std::vector<double> &hyb_poles, const std::vector<dcomplex> &hyb_coeffs,
                   const BlockOpSymQuartet &Fq, int device = 0)
      : beta(beta), dims_(Fq.dims) {
    std::vector<double> rf(4096);
    int rank = 0;
    check(xca_dlr_build_rf(Lambda, eps, rf.data(), (int)rf.size(), &rank));
    rf.resize(rank);
    std::vector<double> it(rank);
    check(xca_dlr_build_it(Lambda, rf.data(), rank, it.data()));
    check(xca_ctx_create(device, &ctx_));
    n = (int)Fq.sym_set_labels.size();
    r = rank;
    q = 0;
    for (long l : Fq.sym_set_labels) q = std::max<int>(q, (int)l + 1);
    Nmax = 0;
    for (int d : dims_) Nmax = std::max(Nmax, d);
    if (hyb_coeffs.size() != hyb_poles.size() * (size_t)n * n)
      throw std::invalid_argument("DiagramEvaluator: hyb_coeffs must have p x n x n entries");
    const int status = xca_evaluator_setup(ctx_, beta, Lambda, eps, rank, rf.data(), it.data(), (int)hyb_poles.size(), hyb_poles.data(),
                                           detail::dp(hyb_coeffs), n, Fq.sym_set_labels.data(), (int)dims_.size(), dims_.data(),
                                           Fq.F_index.data(), detail::dp(Fq.F_data), Fq.Fd_index.data(), detail::dp(Fq.Fd_data));
    if (status != XCA_OK) {
      xca_ctx_destroy(ctx_);
      ctx_ = nullptr;
      check(status);
    }
  }
  DiagramEvaluator(const DiagramEvaluator &) = delete;
  DiagramEvaluator &operator=(const DiagramEvaluator &) = delete;
  ~DiagramEvaluator() {
    if (ctx_) xca_ctx_destroy(ctx_);
  }

  // get_num_self_energy_backbones, block_sparse_backbone.cpp:721-724
  long get_num_self_energy_backbones(const Topology &topology) const {
    long out = 0;
    const auto t = detail::flat(topology);
    check(xca_num_self_energy_backbones(ctx_, (int)topology.size(), t.data(), &out));
    return out;
  }
  long get_num_single_ptcle_gf_backbones(const Topology &topology) const {
    long out = 0;
    const auto t = detail::flat(topology);
    check(xca_num_single_ptcle_gf_backbones(ctx_, (int)topology.size(), t.data(), &out));
    return out;
  }

  // compute_self_energy(G, topology[, f_ix | f_ix_vec]), block_sparse_backbone.cpp:369-459
  BlockGf compute_self_energy(const BlockGf &G, const Topology &topology) { return sigma(G, topology, nullptr, 0); }
  BlockGf compute_self_energy(const BlockGf &G, const Topology &topology, long f_ix) { return sigma(G, topology, &f_ix, 1); }
  BlockGf compute_self_energy(const BlockGf &G, const Topology &topology, const std::vector<long> &f_ix_vec) {
    return sigma(G, topology, f_ix_vec.data(), (long)f_ix_vec.size());
  }

  // compute_single_ptcle_gf(G, topology[, f_ix | f_ix_vec]), block_sparse_backbone.cpp:779-821: r x n x n
  std::vector<dcomplex> compute_single_ptcle_gf(const BlockGf &G, const Topology &topology) { return spgf(G, topology, nullptr, 0); }
  std::vector<dcomplex> compute_single_ptcle_gf(const BlockGf &G, const Topology &topology, long f_ix) {
    return spgf(G, topology, &f_ix, 1);
  }
  std::vector<dcomplex> compute_single_ptcle_gf(const BlockGf &G, const Topology &topology, const std::vector<long> &f_ix_vec) {
    return spgf(G, topology, f_ix_vec.data(), (long)f_ix_vec.size());
  }

  // compute_one_time_correlator(G, ops_tau, ops_0, ad, topology, f_ix_vec), block_sparse_backbone.cpp:843-866,
  // with the operators already in block form: r x ops_tau.size() x ops_0.size()
  std::vector<dcomplex> compute_one_time_correlator(const BlockGf &G, const std::vector<BlockOp> &ops_tau, const std::vector<BlockOp> &ops_0,
                                                    const Topology &topology, const std::vector<long> &f_ix_vec) {
    std::vector<int> ti, zi;
    std::vector<dcomplex> td, zd;
    pack_ops(ops_tau, ti, td);
    pack_ops(ops_0, zi, zd);
    const auto g = detail::pack(G);
    const auto t = detail::flat(topology);
    std::vector<dcomplex> out((size_t)r * ops_tau.size() * ops_0.size());
    check(xca_compute_one_time_correlator(ctx_, detail::dp(g), (int)ops_tau.size(), ti.data(), detail::dp(td), (int)ops_0.size(), zi.data(),
                                          detail::dp(zd), (int)topology.size(), t.data(), f_ix_vec.data(), (long)f_ix_vec.size(),
                                          detail::dp(out)));
    return out;
  }

  // convolve_ppsc and trace of block_sparse.cpp:832-861 on this evaluator's basis and blocks
  BlockGf convolve_ppsc(const BlockGf &G1, const BlockGf &G2) {
    const auto a = detail::pack(G1), b = detail::pack(G2);
    std::vector<dcomplex> out(a.size());
    check(xca_convolve_ppsc(ctx_, detail::dp(a), detail::dp(b), detail::dp(out)));
    return unpack(out);
  }
  dcomplex trace(const BlockGf &G) {
    const auto g = detail::pack(G);
    double out[2];
    check(xca_trace(ctx_, detail::dp(g), out));
    return {out[0], out[1]};
  }
  // expectation_value(op, ad, G), block_sparse.cpp:797-818, with the operator already in block form
  dcomplex expectation_value(const BlockOp &op, const BlockGf &G) {
    std::vector<int> idx;
    std::vector<dcomplex> data;
    pack_ops({op}, idx, data);
    const auto g = detail::pack(G);
    double out[2];
    check(xca_expectation_value(ctx_, detail::dp(g), idx.data(), detail::dp(data), out));
    return {out[0], out[1]};
  }

  // XCA_PREC_FP64 or XCA_PREC_FP64_ORDERED
  void set_precision_mode(int mode) { check(xca_set_precision_mode(ctx_, mode)); }

  xca_ctx *context() const { return ctx_; }

  double beta;
  int r = 0, n = 0, q = 0, Nmax = 0;

 private:
  BlockGf sigma(const BlockGf &G, const Topology &topology, const long *f_ix, long n_fix) {
    const auto g = detail::pack(G);
    const auto t = detail::flat(topology);
    std::vector<dcomplex> out(g.size());
    check(xca_compute_self_energy(ctx_, detail::dp(g), (int)topology.size(), t.data(), f_ix, n_fix, detail::dp(out)));
    return unpack(out);
  }
  std::vector<dcomplex> spgf(const BlockGf &G, const Topology &topology, const long *f_ix, long n_fix) {
    const auto g = detail::pack(G);
    const auto t = detail::flat(topology);
    std::vector<dcomplex> out((size_t)r * n * n);
    check(xca_compute_single_ptcle_gf(ctx_, detail::dp(g), (int)topology.size(), t.data(), f_ix, n_fix, detail::dp(out)));
    return out;
  }
  BlockGf unpack(const std::vector<dcomplex> &flat) const {
    BlockGf out;
    size_t off = 0;
    for (int d : dims_) {
      out.emplace_back(flat.begin() + off, flat.begin() + off + (size_t)r * d * d);
      off += (size_t)r * d * d;
    }
    return out;
  }
  void pack_ops(const std::vector<BlockOp> &ops, std::vector<int> &idx, std::vector<dcomplex> &data) const {
    for (const auto &op : ops) {
      if (op.index.size() != dims_.size()) throw std::invalid_argument("BlockOp: one target index per block required");
      for (size_t b = 0; b < dims_.size(); ++b) {
        idx.push_back(op.index[b]);
        if (op.index[b] >= 0) data.insert(data.end(), op.blocks[b].begin(), op.blocks[b].end());
      }
    }
    if (data.empty()) data.resize(1);
  }

  std::vector<int> dims_;
  xca_ctx *ctx_ = nullptr;
};

}  // namespace block_sparse

namespace cppdlr {

// dyson_it_ppsc(beta, itops, g0) and solve(sig, eta), dlr_dyson_ppsc.hpp:91-168, for one block of
// dimension d on the DLR basis of (Lambda, eps); g0 and sig are (r, d, d).
class dyson_it_ppsc {
 public:
  dyson_it_ppsc(double beta, double Lambda, double eps, const std::vector<dcomplex> &g0, int d, int device = 0) : d_(d) {
    std::vector<double> rf(4096);
    int rank = 0;
    check(xca_dlr_build_rf(Lambda, eps, rf.data(), (int)rf.size(), &rank));
    rf.resize(rank);
    std::vector<double> it(rank);
    check(xca_dlr_build_it(Lambda, rf.data(), rank, it.data()));
    r_ = rank;
    if (g0.size() != (size_t)rank * d * d) throw std::invalid_argument("dyson_it_ppsc: g0 must be r x d x d");
    check(xca_ctx_create(device, &ctx_));
    int status = xca_basis_setup(ctx_, beta, Lambda, eps, rank, rf.data(), it.data(), 1, &d_);
    if (status == XCA_OK) status = xca_dyson_setup(ctx_, detail::dp(g0));
    if (status != XCA_OK) {
      xca_ctx_destroy(ctx_);
      ctx_ = nullptr;
      check(status);
    }
  }
  dyson_it_ppsc(const dyson_it_ppsc &) = delete;
  dyson_it_ppsc &operator=(const dyson_it_ppsc &) = delete;
  ~dyson_it_ppsc() {
    if (ctx_) xca_ctx_destroy(ctx_);
  }
  std::vector<dcomplex> solve(const std::vector<dcomplex> &sig, double eta) {
    if (sig.size() != (size_t)r_ * d_ * d_) throw std::invalid_argument("dyson_it_ppsc::solve: sig must be r x d x d");
    std::vector<dcomplex> out(sig.size());
    check(xca_dyson_solve(ctx_, detail::dp(sig), eta, 0, detail::dp(out)));
    return out;
  }
  // dlr_dyson_ppsc.hpp:188-216: the source term gains G0(t) op (op: d x d)
  std::vector<dcomplex> solve_with_op(const std::vector<dcomplex> &sig, double eta, const std::vector<dcomplex> &op) {
    if (sig.size() != (size_t)r_ * d_ * d_) throw std::invalid_argument("dyson_it_ppsc::solve_with_op: sig must be r x d x d");
    if (op.size() != (size_t)d_ * d_) throw std::invalid_argument("dyson_it_ppsc::solve_with_op: op must be d x d");
    std::vector<dcomplex> out(sig.size());
    check(xca_dyson_solve_with_op(ctx_, detail::dp(sig), eta, detail::dp(op), 0, detail::dp(out)));
    return out;
  }
  int rank() const { return r_; }

 private:
  int d_ = 0, r_ = 0;
  xca_ctx *ctx_ = nullptr;
};

}  // namespace cppdlr
}  // namespace xca_b200
