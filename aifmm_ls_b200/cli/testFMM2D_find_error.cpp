// testFMM2D_find_error -- the reference driver's command line on the B200 solver.
//
//   testFMM2D_find_error nChebNodes kappa degreeOfBases L Qchoice TOL_POW nLevelsUniform
//
// (argv order of testFMM2D_find_error.cpp:44-52).  The reference needs two
// binaries and files on disk for its find_error protocol (gen_rhs_x writes
// x and rhs = A x, find_error solves with rhs and compares); both passes run
// here in one process: solve the physical right-hand side for x_true, form
// rhs = A x_true with exact entries, solve again, print ||x - x_true|| / ||x_true||.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "aifmm_fmm2dtree.hpp"

using aifmm::dtype;

int main(int argc, char* argv[]) {
  if (argc < 8) {
    fprintf(stderr, "usage: %s nChebNodes kappa degreeOfBases L Qchoice TOL_POW nLevelsUniform\n", argv[0]);
    return 2;
  }
  const int nCheb = atoi(argv[1]);
  const double kappa = atof(argv[2]);
  const int degree = atoi(argv[3]);
  const double L = atof(argv[4]);
  const int Qchoice = atoi(argv[5]);
  const int TOL_POW = atoi(argv[6]);
  const int nLevels = atoi(argv[7]);
  printf("\n---------------problem parameters---------------\n");
  printf("kappa: %g\nnChebNodes: %d\nL: %g\nQchoice: %d\nTOL_POW: %d\nnLevelsUniform: %d\n", kappa, nCheb, L, Qchoice,
         TOL_POW, nLevels);
  printf("------------------------------------------------\n\n");
  try {
    auto now = [] { return std::chrono::steady_clock::now(); };
    auto secs = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
    aifmm::userkernel K(nCheb, 1, degree, L, nLevels, kappa, Qchoice, TOL_POW);
    const int N = K.N;
    printf("N: %d\n", N);
    // gen_rhs_x pass: x_true solves A x = b_physical
    aifmm::FMM2DTree<aifmm::userkernel> G(&K, N, nLevels, TOL_POW, nullptr, K.rhs.data());
    G.createTree();
    G.assemble();
    G.eliminate_phase_efficient();
    G.back_substitution_phase();
    std::vector<dtype> x_true = G.solution(), rhs(N);
    aifmm_status s = aifmm_dense_matvec(K.handle(), 1, reinterpret_cast<const double*>(x_true.data()),
                                        reinterpret_cast<double*>(rhs.data()), AIFMM_PTR_HOST);
    aifmm::check(s, K.handle());
    // find_error pass
    aifmm::FMM2DTree<aifmm::userkernel> A(&K, N, nLevels, TOL_POW, nullptr, rhs.data());
    auto t0 = now();
    A.createTree();
    A.assign_Tree_Interactions();
    auto t1 = now();
    printf("Number of Levels of tree: %d\n\nTime taken to create the tree is: %g\n", nLevels, secs(t0, t1));
    A.assemble();
    auto t2 = now();
    printf("\nTime taken to assemble is: %g\n", secs(t1, t2));
    A.eliminate_phase_efficient();
    auto t3 = now();
    printf("\nTime taken to factorize is: %g\n", secs(t2, t3));
    A.back_substitution_phase();
    auto t4 = now();
    printf("\nTime taken to solve is: %g\n", secs(t3, t4));
    printf("\nPerforming error calculation... \n");
    printf("\nerror: %g\n\n", A.error_check(x_true));
  } catch (const std::exception& e) {
    fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
