// Driver of the reference's own C++ sources (vaishna77/RCS src/*.cpp and
// include/AIFMMTree2D_3D_memory_optimized.hpp, compiled unmodified where they
// lie, against the project-written Eigen subset in include/aifmm/Eigen) that
// writes what the oracle's parity checks need.  Test infrastructure: it is
// built by oracle/ref.mk into oracle/_ref/ and run only by the fixture
// scripts under tests/golden/.
//
// It follows the reference's own driver, test/sphere.cpp: the kernel from a
// node/patch file pair (EFIEMatrix(inputsToKernelClass), sphere.cpp:97), the
// solver inputs from the RWG edge midpoints (sphere.cpp:139-170), the
// x-polarised plane-wave right-hand side (sphere.cpp:172-177), the dense LU
// solution (getCoefficients, sphere.cpp:181), the AIFMM constructor,
// factorize, backSubstitute1/2/3 and getPhi (sphere.cpp:203-262).  The
// frequency is the reference's compiled-in constant (includes.hpp: 10 MHz).
//
//   aifmm_ref EFIE <nodeList> <patchList> <leaf> <tol_pow> <fillin_tol> <out.bin> [dense 0|1] [threads]
//
// Output (little-endian): int32 magic 0x52454631, int32 N, int32 nLevels,
// int32 nPairs; N complex128 right-hand side; N complex128 dense LU solution
// (zeros when dense = 0); N complex128 AIFMM solution (getPhi order);
// nPairs x (int32 i, int32 j, complex128 getMatrixEntry(i, j)) for seeded
// pairs; per level j = 0..nLevels and box k: int32 rank after assembly
// (L2P columns), int32 rank after factorization; float64 seconds of assemble,
// factorize, solve; then two block tables, after assembly and after
// factorization: int64 count, count x 7 float64 rows (level, box, kind, key,
// rows, cols, Frobenius norm) with kind 0 L2P, 1 P2M, 2 M2L, 3 P2P, 4 M2P,
// 5 P2L, 6 L2P_f, 7 P2M_f, 8 M2M_f (key = the partner box), 9 L2M_f.
#include <omp.h>

#include <cstdint>
#include <cstdio>
#include <fstream>
#include <random>

#include "AIFMM.hpp"

static void put_i(std::ofstream& f, int32_t v) { f.write(reinterpret_cast<const char*>(&v), 4); }
static void put_d(std::ofstream& f, double v) { f.write(reinterpret_cast<const char*>(&v), 8); }
static void put_c(std::ofstream& f, const std::complex<double>& v) {
  put_d(f, v.real());
  put_d(f, v.imag());
}

// every block of every box: (level, box, kind, key, rows, cols, norm)
template <typename Tree>
static std::vector<double> block_table(Tree* t) {
  std::vector<double> out;
  for (int j = 0; j <= t->nLevels; ++j)
    for (size_t k = 0; k < t->tree->at(j).size(); ++k) {
      FMM2DBox& B = t->tree->at(j)[k];
      auto add = [&](int kind, int key, const Mat& m) {
        const double row[7] = {(double)j, (double)k, (double)kind, (double)key, (double)m.rows(), (double)m.cols(),
                               m.norm()};
        out.insert(out.end(), row, row + 7);
      };
      add(0, -1, B.L2P);
      add(1, -1, B.P2M);
      int kind = 2;
      for (std::map<int, Mat>* mp : {&B.M2L, &B.P2P, &B.M2P, &B.P2L, &B.L2P_f, &B.P2M_f, &B.M2M_f}) {
        for (auto& kv : *mp) add(kind, kv.first, kv.second);
        kind++;
      }
      add(9, -1, B.L2M_f);
    }
  return out;
}
static void put_table(std::ofstream& f, const std::vector<double>& t) {
  const int64_t n = (int64_t)(t.size() / 7);
  f.write(reinterpret_cast<const char*>(&n), 8);
  for (double v : t) put_d(f, v);
}

int main(int argc, char** argv) {
  if (argc < 8 || std::string(argv[1]) != "EFIE") {
    std::fprintf(stderr, "usage: %s EFIE nodeList patchList leaf tol_pow fillin_tol out.bin [dense] [threads]\n",
                 argv[0]);
    return 2;
  }
  const int leaf = std::atoi(argv[4]), tolPow = std::atoi(argv[5]), fillinTol = std::atoi(argv[6]);
  const bool dense = argc > 8 ? std::atoi(argv[8]) != 0 : true;
  const int threads = argc > 9 ? std::atoi(argv[9]) : 1;
  omp_set_num_threads(threads);

  inputsToKernelClass ik;
  ik.nodeListFilename = argv[2];
  ik.patchListFilename = argv[3];
  ik.n = 0;
  ik.L = 0.0;
  EFIEMatrix* K = new EFIEMatrix(ik);
  const int N = K->N;

  // solver inputs from the RWG edge midpoints, as sphere.cpp:139-170 builds them
  Eigen::MatrixXd mid(N, 3);
  int i = 0;
  for (auto it = K->edge2PatchMap.begin(); it != K->edge2PatchMap.end(); ++it, ++i) {
    Node a = K->nodeList[it->first.first];
    Node b = K->nodeList[it->first.second];
    mid.row(i) = (a + b) / 2.0;
  }
  Eigen::VectorXd mx = mid.colwise().maxCoeff();
  Eigen::VectorXd mn = mid.colwise().minCoeff();
  inputsToSolverClass is;
  is.xmin = mn(0);
  is.xmax = mx(0);
  is.ymin = mn(1);
  is.ymax = mx(1);
  is.zmin = mn(2);
  is.zmax = mx(2);
  is.leafSize = leaf;
  is.tol_pow = tolPow;
  is.locations = mid;
  is.nLevelsInput = 0;
  is.fillin_rank = 0;
  is.fillin_tol = fillinTol;

  Node einc;
  einc(0) = 1.0;
  einc(1) = 0.0;
  einc(2) = 0.0;
  Eigen::VectorXcd rhs;
  K->getRhs(einc, rhs);
  Eigen::VectorXcd xlu = Eigen::VectorXcd::Zero(N);
  if (dense) K->getCoefficients(rhs, xlu);

  double t0 = omp_get_wtime();
  AIFMM<EFIEMatrix>* S = new AIFMM<EFIEMatrix>(is, K);
  const double tAsm = omp_get_wtime() - t0;
  const int nLevels = S->A->nLevels;
  std::vector<std::vector<int>> rank0(nLevels + 1);
  for (int j = 0; j <= nLevels; ++j)
    for (size_t k = 0; k < S->A->tree->at(j).size(); ++k)
      rank0[j].push_back((int)S->A->tree->at(j)[k].L2P.cols());
  const std::vector<double> table0 = block_table(S->A);
  omp_set_num_threads(1);  // the reference factorizes and solves on one thread (sphere.cpp:206-207)
  t0 = omp_get_wtime();
  S->factorize();
  const double tFac = omp_get_wtime() - t0;
  S->backSubstitute1(rhs);
  t0 = omp_get_wtime();
  S->backSubstitute2();
  S->backSubstitute3();
  const double tSol = omp_get_wtime() - t0;
  Eigen::VectorXcd x;
  S->getPhi(x);

  std::mt19937_64 rng(20261204);
  const int nPairs = std::min(4096, N * N);
  std::ofstream f(argv[7], std::ios::binary);
  put_i(f, 0x52454631);
  put_i(f, N);
  put_i(f, nLevels);
  put_i(f, nPairs);
  for (int q = 0; q < N; ++q) put_c(f, rhs(q));
  for (int q = 0; q < N; ++q) put_c(f, xlu(q));
  for (int q = 0; q < N; ++q) put_c(f, x(q));
  for (int q = 0; q < nPairs; ++q) {
    const int a = (int)(rng() % (uint64_t)N), b = (int)(rng() % (uint64_t)N);
    put_i(f, a);
    put_i(f, b);
    put_c(f, K->getMatrixEntry(a, b));
  }
  for (int j = 0; j <= nLevels; ++j)
    for (size_t k = 0; k < S->A->tree->at(j).size(); ++k) {
      put_i(f, rank0[j][k]);
      put_i(f, (int)S->A->tree->at(j)[k].L2P.cols());
    }
  put_d(f, tAsm);
  put_d(f, tFac);
  put_d(f, tSol);
  put_table(f, table0);
  put_table(f, block_table(S->A));
  return f.good() ? 0 : 1;
}
