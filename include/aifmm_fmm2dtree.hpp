// aifmm_fmm2dtree.hpp -- header-only C++ surface of the reference solver over the C ABI.
//
// Mirrors the classes a reference driver uses (kernel.hpp userkernel,
// FMM2DTree_find_error.hpp FMM2DTree<userkernel>) so that
// testFMM2D_find_error.cpp-style code ports by changing includes.  All work is
// done by libaifmm_b200.so on the GPU; there is no CPU path.
#ifndef AIFMM_FMM2DTREE_HPP
#define AIFMM_FMM2DTREE_HPP

#include <cmath>
#include <complex>
#include <stdexcept>
#include <string>
#include <vector>

#include "aifmm_b200.h"

namespace aifmm {

using dtype = std::complex<double>;
struct pts2D { double x, y; };

inline void check(aifmm_status s, const aifmm_problem* p) {
  if (s != AIFMM_OK)
    throw std::runtime_error(std::string("aifmm: ") + aifmm_status_string(s) + (p ? std::string(": ") + aifmm_last_error(p) : ""));
}

// userkernel (kernel.hpp:90-193).  The reference reads kappa and Qchoice from
// globals set by main (LS/LS_Assembly.hpp:31,35) and TOL_POW from the tree's
// constructor; here they are constructor arguments.
class userkernel {
 public:
  int N = 0;
  int nLevelsResolve = 0;
  std::vector<pts2D> gridPoints;
  std::vector<dtype> rhs;

  userkernel(int nChebNodes, int /*treeAdaptivity*/, int degreeOfBases, double L, int nLevelsUniform,
             double kappa, int Qchoice, int TOL_POW, int device = 0, double q_amp = 1.5, double q_width = 32.0,
             double q_radius = 0.5) {
    aifmm_desc d{nChebNodes, kappa, degreeOfBases, L, nLevelsUniform, TOL_POW, Qchoice, q_amp, q_width, q_radius};
    check(aifmm_problem_create(&d, device, &p_), nullptr);
    check(aifmm_tables_compute(p_, 1), p_);  // evaluatePrecomputations + the 6-digit text round trip
    check(aifmm_num_points(p_, &N), p_);
    nLevelsResolve = nLevelsUniform;
    std::vector<double> xy(2 * (size_t)N);
    check(aifmm_grid_points(p_, xy.data()), p_);
    gridPoints.resize(N);
    for (int i = 0; i < N; ++i) gridPoints[i] = {xy[2 * i], xy[2 * i + 1]};
    const double th = 0.0;  // IncidenceFunction exp(i kappa x) (LS/LS_functions.hpp:113-116)
    rhs.resize(N);
    check(aifmm_rhs_plane_wave(p_, 1, &th, reinterpret_cast<double*>(rhs.data()), AIFMM_PTR_HOST), p_);
  }
  ~userkernel() { if (p_) aifmm_problem_destroy(p_); }
  userkernel(const userkernel&) = delete;
  userkernel& operator=(const userkernel&) = delete;

  dtype getMatrixEntry(unsigned i, unsigned j) {
    int I = (int)i, J = (int)j;
    dtype v;
    check(aifmm_entries(p_, 1, &I, &J, reinterpret_cast<double*>(&v), AIFMM_PTR_HOST), p_);
    return v;
  }
  std::vector<dtype> getMatrix(const std::vector<int>& rows, const std::vector<int>& cols) {  // column-major
    std::vector<dtype> out(rows.size() * cols.size());
    check(aifmm_get_matrix(p_, (int)rows.size(), rows.data(), (int)cols.size(), cols.data(),
                           reinterpret_cast<double*>(out.data()), AIFMM_PTR_HOST), p_);
    return out;
  }
  std::vector<dtype> getRow(int j, const std::vector<int>& cols) { return getMatrix({j}, cols); }
  std::vector<dtype> getCol(int k, const std::vector<int>& rows) { return getMatrix(rows, {k}); }
  aifmm_problem* handle() { return p_; }

 private:
  aifmm_problem* p_ = nullptr;
};

// FMM2DTree<userkernel> (FMM2DTree_find_error.hpp:76-2583).  The particles are the
// kernel's grid points in order (boxNumbers = iota, nChebNodes^2 per leaf), as
// in testFMM2D_find_error.cpp:119-127.
template <class K>
class FMM2DTree {
 public:
  FMM2DTree(K* k, int N, int nLevels, int /*TOL_POW: fixed by the kernel*/, const double* /*locations*/,
            const dtype* properties, int nrhs = 1)
      : K_(k), N_(N), nLevels_(nLevels), nrhs_(nrhs), b_(properties, properties + (size_t)N * nrhs),
        x_((size_t)N * nrhs) {}

  void createTree() { check(aifmm_build_tree(K_->handle()), K_->handle()); }
  void assign_Tree_Interactions() {}
  // assignLeafChargeLocations .. initialise_P2P_Leaf_Level (F:1072-1741) in one call
  void assemble() { check(aifmm_assemble(K_->handle()), K_->handle()); }
  void assignLeafChargeLocations() {}
  void assign_Leaf_rhs() {}
  void getNodes() { assemble(); }
  void assemble_M2L() {}
  void initialise_phase() {}
  void initialise_P2P_Leaf_Level() {}
  // eliminate_phase_efficient + back_substitution_phase with the right-hand sides carried
  void eliminate_phase_efficient() {
    check(aifmm_factorize_solve(K_->handle(), nrhs_, reinterpret_cast<const double*>(b_.data()),
                                reinterpret_cast<double*>(x_.data()), AIFMM_PTR_HOST), K_->handle());
  }
  void back_substitution_phase() {}
  const std::vector<dtype>& solution() const { return x_; }
  // error_check (F:2534-2581): relative forward error against x_true
  double error_check(const std::vector<dtype>& x_true) const {
    double e = 0.0, n = 0.0;
    for (size_t i = 0; i < x_.size(); ++i) { e += std::norm(x_[i] - x_true[i]); n += std::norm(x_true[i]); }
    return std::sqrt(e / n);
  }

 private:
  K* K_;
  int N_, nLevels_, nrhs_;
  std::vector<dtype> b_, x_;
};

}  // namespace aifmm
#endif
