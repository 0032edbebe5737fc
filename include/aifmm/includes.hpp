// Drop-in replacement for the reference's include/includes.hpp: scalar types,
// physical constants, Green's functions and the solver / kernel input structs
// (include/includes.hpp:1-95, src/includes.cpp:8-59 of the reference), plus the
// binding of the C++ classes to libaifmm_b200.so.
//
// Build a driver written against the reference's classes with
//   g++ -std=c++17 -DUSE_COMPLEX64 -DUSE_THREE -I<repo>/include/aifmm driver.cpp
//       -L<repo>/rcs_b200/lib -laifmm_b200 -Wl,-rpath,<repo>/rcs_b200/lib
// (-fopenmp if the driver calls omp_* functions).  USE_COMPLEX64 / USE_DOUBLE
// choose dtype as in the reference; with neither, complex is used.
//
// Differences from the reference, all deliberate:
//   - freq is the macro AIFMM_FREQ (default 1.0e7 Hz, the reference's fixed
//     value), so a driver can be built for another frequency with
//     -DAIFMM_FREQ=1e9; lambda and kappa follow it.
//   - Library failures throw std::runtime_error with the library's message
//     (the reference has no error reporting).
//   - The CUDA device is the one named by the environment variable
//     AIFMM_DEVICE (default 0).
#ifndef AIFMM_DROPIN_INCLUDES_HPP
#define AIFMM_DROPIN_INCLUDES_HPP

#include <cfloat>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <iterator>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include <Eigen/Dense>

#include "../aifmm_b200.h"

using namespace std;
using namespace Eigen;

typedef Eigen::Vector3d Node;
typedef Eigen::Vector3cd NodeC;
typedef std::complex<double> cdouble;
#if defined(USE_DOUBLE)
typedef double dtype;
using Mat = Eigen::MatrixXd;
using Vec = Eigen::VectorXd;
#else
#ifndef USE_COMPLEX64
#define USE_COMPLEX64 1
#endif
typedef std::complex<double> dtype;
using Mat = Eigen::MatrixXcd;
using Vec = Eigen::VectorXcd;
#endif

struct pts2D {
  double x, y;
};

struct pts3D {
  double x, y, z;
};

#if defined(USE_TWO)
const int nDims = 2;
typedef pts2D ptsdD;
#else
#ifndef USE_THREE
#define USE_THREE 1
#endif
const int nDims = 3;
typedef pts3D ptsdD;
#endif

typedef cdouble (*scalarFunctionPointer)(Node&, Node&);
typedef Node (*vectorRealFunctionPointer)(Node&, Node&, Node&);
typedef NodeC (*vectorComplexFunctionPointer)(Node&, Node&, Node&);

#ifndef AIFMM_FREQ
#define AIFMM_FREQ 1.0e7
#endif

const double epsilon = 8.854187817e-12;
const std::complex<double> I(0.0, 1.0);
const double PI = 4.0 * std::atan(1.0);
const double c = 3.0e8;
const double freq = AIFMM_FREQ;
const double lambda = c / freq;
const double kappa = 2 * PI / lambda;
const double C0 = 1.0 / (4 * PI * epsilon);
const double mu = 4 * PI * 1e-7;
const double eta_0 = std::sqrt(mu / epsilon);

// Green's functions of the reference (src/includes.cpp:8-59), for drivers that
// call them; the library's GPU kernels evaluate their own copies.
inline double getDistance(Node& p1, Node& p2) { return (p1 - p2).norm(); }
inline double ElectrostaticGreensFunction(Node& ri, Node& rj) { return 1.0 / getDistance(ri, rj); }
inline cdouble EFIEGreensFunction(Node& ri, Node& rj) {
  const double R = getDistance(ri, rj);
  return (-1.0 / (4.0 * PI)) * std::exp(-I * kappa * R) / R;
}
inline cdouble nonSingularGreensFunction(Node& ri, Node& rj) {
  const double R = getDistance(ri, rj);
  return (-1.0 / (4.0 * PI)) * (std::exp(-I * kappa * R) - 1.0) / R;
}
inline NodeC rhoGreensFunction(Node& ri, Node& rj, Node&) {
  const double R = getDistance(ri, rj);
  return NodeC(rj) * ((-1.0 / (4.0 * PI)) * std::exp(-I * kappa * R) / R);
}
inline Node rhoLaplaceFunction(Node& ri, Node& rj, Node& r3) {
  const double R = getDistance(ri, rj);
  return (rj - r3) * (-1.0 / (4.0 * PI) / R);
}
inline NodeC rhoNonSingularGreensFunction(Node& ri, Node& rj, Node& r3) {
  const double R = getDistance(ri, rj);
  const Node rho = rj - r3;
  if (R < 1e-12) return NodeC(rho) * ((-1.0 / (4.0 * PI)) * (-I * kappa));  // limit R -> 0
  return NodeC(rho) * ((-1.0 / (4.0 * PI)) * (std::exp(-I * kappa * R) - 1.0) / R);
}
inline NodeC farFieldIntegrand(Node& ri, Node& rj, Node& r3) {
  return NodeC(rj - r3) * std::exp(I * kappa * rj.dot(ri));
}

struct inputsToSolverClass {
  double xmin, xmax, ymin, ymax, zmin, zmax;
  int leafSize, tol_pow, nLevelsInput, fillin_rank, fillin_tol;
  Eigen::MatrixXd locations;
  // Extensions (no counterpart in the reference; the defaults keep its
  // arithmetic): GEMM precision of the factorization (0 = complex128;
  // 1-3 = split-TF32 tensor-core Schur products, for use as a preconditioner)
  // and exact_rrqr (1 = every recompression runs the full partition-1 pass).
  int precision = 0;
  int exact_rrqr = 0;
};

struct inputsToKernelClass {
  std::string nodeListFilename;
  std::string patchListFilename;
  int n;     // plate meshes only (unused here)
  double L;  // plate meshes only (unused here)
};

namespace aifmm_dropin {

inline void check(int rc) {
  if (rc != AIFMM_OK) throw std::runtime_error(std::string("aifmm: ") + aifmm_last_error());
}

// The process-wide library context the drop-in classes share.  It lives until
// the process exits, like the kernels that the reference's drivers leak.
inline aifmm_ctx* context() {
  static aifmm_ctx* ctx = [] {
    const char* d = std::getenv("AIFMM_DEVICE");
    aifmm_ctx* c = nullptr;
    check(aifmm_ctx_create(d ? std::atoi(d) : 0, &c));
    return c;
  }();
  return ctx;
}

// dtype <-> interleaved complex128 buffers of the C ABI
inline void put(std::complex<double>* out, const std::complex<double>& v) { *out = v; }
inline void put(std::complex<double>* out, double v) { *out = std::complex<double>(v, 0.0); }
inline void get(std::complex<double>& out, const std::complex<double>& v) { out = v; }
inline void get(double& out, const std::complex<double>& v) { out = v.real(); }

template <typename M>
std::vector<std::complex<double>> to_c128(const M& m) {
  std::vector<std::complex<double>> v((size_t)m.rows() * (size_t)m.cols());
  for (Eigen::Index j = 0; j < m.cols(); ++j)
    for (Eigen::Index i = 0; i < m.rows(); ++i) put(&v[(size_t)(i + j * m.rows())], m(i, j));
  return v;
}

template <typename M>
void from_c128(const std::complex<double>* v, Eigen::Index r, Eigen::Index cols, M& m) {
  m.resize(r, cols);
  for (Eigen::Index j = 0; j < cols; ++j)
    for (Eigen::Index i = 0; i < r; ++i) get(m(i, j), v[(size_t)(i + j * r)]);
}

}  // namespace aifmm_dropin

#endif
