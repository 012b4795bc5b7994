// aifmm_fmm2dtree.hpp -- header-only C++ surface of the reference solver over the C ABI.
//
// Mirrors the classes a reference driver uses (kernel.hpp userkernel,
// FMM2DTree_find_error.hpp FMM2DTree<userkernel>) so that
// testFMM2D_find_error.cpp-style code ports by changing includes.  All work is
// done by libaifmm_b200.so on the GPU; there is no CPU path.
#ifndef AIFMM_FMM2DTREE_HPP
#define AIFMM_FMM2DTREE_HPP

#include <algorithm>
#include <cmath>
#include <complex>
#include <fstream>
#include <iterator>
#include <sstream>
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

// A matrix file of the reference's precomputations/ directory (written with Eigen's
// operator<<, LS/LS_Assembly.hpp:1166-1184 and :1328-1420), read the way the
// reference reads it (ReadFromTextFile, :1187-1214): rows = newline count,
// columns = whitespace-separated tokens / rows, each token a "(re,im)" complex.
// Returns the entries column-major.
inline std::vector<dtype> read_eigen_text(const std::string& path, long& rows, long& cols) {
  std::ifstream in(path);
  if (!in.good()) throw std::runtime_error("aifmm: cannot open " + path);
  std::stringstream buf;
  buf << in.rdbuf();
  const std::string text = buf.str();
  rows = (long)std::count(text.begin(), text.end(), '\n');
  std::istringstream words(text);
  const long ntok = (long)std::distance(std::istream_iterator<std::string>(words), std::istream_iterator<std::string>());
  if (rows == 0 || ntok % rows != 0) throw std::runtime_error("aifmm: " + path + " cannot form a matrix");
  cols = ntok / rows;
  std::istringstream vals(text);
  std::vector<dtype> out((size_t)rows * cols);
  for (long i = 0; i < rows; ++i)
    for (long j = 0; j < cols; ++j)
      if (!(vals >> out[(size_t)i + (size_t)j * rows])) throw std::runtime_error("aifmm: bad entry in " + path);
  return out;
}

// The leaf-level tables a reference build wrote under root (M_<n>_<depth> and the
// nine colleagueNeighborInteraction_<depth>_<n> files) in the interleaved layout of
// aifmm_tables_set: M = 121 x nCheb^2, then nine nCheb^2 x nCheb^2 tables, all
// column-major.  With them the solver factorises exactly the reference's matrix.
inline void read_reference_tables(const std::string& root, int nChebNodes, double kappa, int degreeOfBases,
                                  int depth, std::vector<double>& M, std::vector<double>& near_tables) {
  const std::string tag = std::to_string(nChebNodes) + "_" + std::to_string(int(kappa)) + "_" +
                          std::to_string(degreeOfBases);
  const std::string pre = root + "/precomputations";
  const long rank = (long)nChebNodes * nChebNodes;
  long r = 0, c = 0;
  auto m = read_eigen_text(pre + "/M/M_" + tag + "/M_" + std::to_string(nChebNodes) + "_" + std::to_string(depth), r, c);
  if (r != 121 || c != rank) throw std::runtime_error("aifmm: M table has the wrong shape");
  M.assign(reinterpret_cast<const double*>(m.data()), reinterpret_cast<const double*>(m.data()) + 2 * m.size());
  near_tables.clear();
  for (int n = 0; n < 9; ++n) {
    auto t = read_eigen_text(pre + "/Neighbor/Neighbor_" + tag + "/colleagueNeighborInteraction_" +
                             std::to_string(depth) + "_" + std::to_string(n), r, c);
    if (r != rank || c != rank) throw std::runtime_error("aifmm: colleague table has the wrong shape");
    near_tables.insert(near_tables.end(), reinterpret_cast<const double*>(t.data()),
                       reinterpret_cast<const double*>(t.data()) + 2 * t.size());
  }
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
  // readMFromFile + readNeighborInteractions (LS/LS_Assembly.hpp:1216-1228, 1423-1459):
  // replace the computed tables by the leaf-level files a reference build wrote
  void readTables(const std::string& root, int nChebNodes, double kappa, int degreeOfBases) {
    std::vector<double> M, near_tables;
    read_reference_tables(root, nChebNodes, kappa, degreeOfBases, nLevelsResolve, M, near_tables);
    check(aifmm_tables_set(p_, M.data(), near_tables.data()), p_);
  }
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
  // eliminate_phase_efficient (F:2407-2451) with the base-level factorisation; the
  // reference carries the right-hand side through it, here the factors are kept and
  // the right-hand side goes through back_substitution_phase
  // precision AIFMM_PRECISION_C64: the mixed form (complex64 factors; refine() recovers
  // FP64 accuracy and needs keep_assembly)
  void eliminate_phase_efficient(int precision = AIFMM_PRECISION_FP64, bool keep_assembly = false) {
    check(aifmm_factorize(K_->handle(), precision, keep_assembly ? AIFMM_KEEP_ASSEMBLY : 0), K_->handle());
  }
  // the right-hand-side updates of the elimination, the base-level solve and the
  // back substitution (F:1968-2001, 2252-2293, 2453-2532) with the kept factors
  void back_substitution_phase() {
    check(aifmm_solve(K_->handle(), nrhs_, reinterpret_cast<const double*>(b_.data()), N_,
                      reinterpret_cast<double*>(x_.data()), N_, nullptr, AIFMM_PTR_HOST), K_->handle());
  }
  // no counterpart in the reference: GMRES refinement of the solution against the
  // compressed operator to relative residual rtol, with the kept factors as the
  // preconditioner (eliminate_phase_efficient(..., true) first); returns the
  // iterations, *relres the worst column's final relative residual
  int refine(double rtol, int maxit = 90, double* relres = nullptr) {
    int it = 0;
    check(aifmm_solve_refined(K_->handle(), nrhs_, reinterpret_cast<const double*>(b_.data()), N_,
                              reinterpret_cast<double*>(x_.data()), N_, rtol, maxit, &it, relres, AIFMM_PTR_HOST),
          K_->handle());
    return it;
  }
  // another right-hand side against the same factors
  void set_rhs(const dtype* properties) { b_.assign(properties, properties + (size_t)N_ * nrhs_); }
  const std::vector<dtype>& solution() const { return x_; }
  // error_check (F:2534-2581): relative forward error against x_true
  double error_check(const std::vector<dtype>& x_true) const {
    double rel = 0.0;
    check(aifmm_find_error(K_->handle(), nrhs_, reinterpret_cast<const double*>(x_.data()), N_,
                           reinterpret_cast<const double*>(x_true.data()), N_, &rel, AIFMM_PTR_HOST), K_->handle());
    return rel;
  }

 private:
  K* K_;
  int N_, nLevels_, nrhs_;
  std::vector<dtype> b_, x_;
};

}  // namespace aifmm
#endif
