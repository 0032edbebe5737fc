// CPU oracle -- TEST INFRASTRUCTURE ONLY.
//
// Dense complex linear algebra used by the CPU restatement of the
// vaishna77/RCS AIFMM hot path.  The reference links Eigen 3 (header-only,
// version not pinned: CMakeLists.txt:35 reads it from $EIGEN_PATH); Eigen is
// absent here, so this file restates the semantics the reference relies on:
//   * column-major dynamic matrices of std::complex<double>;
//   * PartialPivLU (Eigen semantics: row pivot = first index of the largest
//     |a_ik| in the column, zero pivots recorded and skipped) -- used at
//     include/AIFMMTree2D_3D_memory_optimized.hpp:695,702,3569,3622,4086,
//     4120,4797,4825,4843 and src/EFIEMatrix.cpp:835;
//   * a.dot(b) = sum conj(a_i) b_i (src/ACA.cpp:752,845);
//   * |R(0,0)| of ColPivHouseholderQR = largest column 2-norm
//     (AIFMMTree2D_3D_memory_optimized.hpp:710-723).
// Nothing under oracle/ is linked by the product library; only tests, the
// smoke check and the CPU-baseline leg of bench.py load it.
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

namespace orc {

using cd = std::complex<double>;

[[noreturn]] inline void fail(const char* what) {
  throw std::runtime_error(std::string("oracle: ") + what);
}

struct Mat {
  int r = 0, c = 0;
  std::vector<cd> a;
  Mat() {}
  Mat(int rows, int cols) : r(rows), c(cols), a((size_t)rows * cols, cd(0.0, 0.0)) {
    if (rows < 0 || cols < 0) fail("negative matrix size");
  }
  static Mat Zero(int rows, int cols) { return Mat(rows, cols); }
  static Mat Identity(int rows, int cols) {
    Mat m(rows, cols);
    for (int i = 0; i < std::min(rows, cols); ++i) m(i, i) = 1.0;
    return m;
  }
  int rows() const { return r; }
  int cols() const { return c; }
  long size() const { return (long)r * c; }
  cd& operator()(int i, int j) { return a[(size_t)j * r + i]; }
  const cd& operator()(int i, int j) const { return a[(size_t)j * r + i]; }
  // vector-style access (column vector)
  cd& operator()(int i) { return a[i]; }
  const cd& operator()(int i) const { return a[i]; }

  Mat block(int i0, int j0, int nr, int nc) const {
    if (i0 < 0 || j0 < 0 || nr < 0 || nc < 0 || i0 + nr > r || j0 + nc > c) fail("block out of range");
    Mat m(nr, nc);
    for (int j = 0; j < nc; ++j)
      for (int i = 0; i < nr; ++i) m(i, j) = (*this)(i0 + i, j0 + j);
    return m;
  }
  void setBlock(int i0, int j0, const Mat& m) {
    if (i0 < 0 || j0 < 0 || i0 + m.r > r || j0 + m.c > c) fail("setBlock out of range");
    for (int j = 0; j < m.c; ++j)
      for (int i = 0; i < m.r; ++i) (*this)(i0 + i, j0 + j) = m(i, j);
  }
  Mat adjoint() const {
    Mat m(c, r);
    for (int j = 0; j < c; ++j)
      for (int i = 0; i < r; ++i) m(j, i) = std::conj((*this)(i, j));
    return m;
  }
  Mat col(int j) const { return block(0, j, r, 1); }
  // Frobenius norm, sequential sum of |a|^2.
  double norm() const {
    double s = 0.0;
    for (const cd& z : a) s += std::norm(z);
    return std::sqrt(s);
  }
  double squaredNorm() const {
    double s = 0.0;
    for (const cd& z : a) s += std::norm(z);
    return s;
  }
};

// C += a * b over n complex entries, written on doubles (same formula as the
// finite-value path of std::complex multiplication) so that it vectorises.
inline void axpyC(int n, cd b, const cd* a, cd* c) {
  const double br = b.real(), bi = b.imag();
  const double* ad = reinterpret_cast<const double*>(a);
  double* cdp = reinterpret_cast<double*>(c);
  for (int i = 0; i < n; ++i) {
    const double ar = ad[2 * i], ai = ad[2 * i + 1];
    cdp[2 * i] += ar * br - ai * bi;
    cdp[2 * i + 1] += ar * bi + ai * br;
  }
}

// Each output column is accumulated over k in increasing order by one thread,
// so the result does not depend on the number of threads.
inline Mat operator*(const Mat& A, const Mat& B) {
  if (A.c != B.r) fail("product dimension mismatch");
  Mat C(A.r, B.c);
  const long work = (long)A.r * A.c * B.c;
#pragma omp parallel for schedule(static) if (work > 200000)
  for (int j = 0; j < B.c; ++j)
    for (int k = 0; k < A.c; ++k) axpyC(A.r, B(k, j), &A.a[(size_t)k * A.r], &C.a[(size_t)j * C.r]);
  return C;
}
inline Mat operator+(const Mat& A, const Mat& B) {
  if (A.r != B.r || A.c != B.c) fail("sum dimension mismatch");
  Mat C = A;
  for (size_t i = 0; i < C.a.size(); ++i) C.a[i] += B.a[i];
  return C;
}
inline Mat operator-(const Mat& A, const Mat& B) {
  if (A.r != B.r || A.c != B.c) fail("difference dimension mismatch");
  Mat C = A;
  for (size_t i = 0; i < C.a.size(); ++i) C.a[i] -= B.a[i];
  return C;
}
inline Mat operator-(const Mat& A) {
  Mat C = A;
  for (auto& z : C.a) z = -z;
  return C;
}
inline Mat operator*(const Mat& A, cd s) {
  Mat C = A;
  for (auto& z : C.a) z *= s;
  return C;
}
inline Mat operator/(const Mat& A, cd s) {
  Mat C = A;
  for (auto& z : C.a) z /= s;
  return C;
}
inline Mat operator*(const Mat& A, double s) {
  Mat C = A;
  for (auto& z : C.a) z *= s;
  return C;
}
inline Mat operator/(const Mat& A, double s) {
  Mat C = A;
  for (auto& z : C.a) z /= s;
  return C;
}
// [A | B]
inline Mat hcat(const Mat& A, const Mat& B) {
  if (A.r != B.r) fail("hcat rows mismatch");
  Mat C(A.r, A.c + B.c);
  C.setBlock(0, 0, A);
  C.setBlock(0, A.c, B);
  return C;
}
// conj(a).b over two column vectors
inline cd dotc(const Mat& a, const Mat& b) {
  if (a.size() != b.size()) fail("dot size mismatch");
  cd s(0.0, 0.0);
  for (size_t i = 0; i < a.a.size(); ++i) s += std::conj(a.a[i]) * b.a[i];
  return s;
}

// Partial-pivoting LU with Eigen's PartialPivLU pivot rule.
struct LU {
  Mat lu;
  std::vector<int> perm;  // row i of P*A is row perm[i] of A
  int n = 0;
  LU() {}
  explicit LU(const Mat& A) { compute(A); }
  void compute(const Mat& A) {
    if (A.r != A.c) fail("LU of non-square matrix");
    n = A.r;
    lu = A;
    std::vector<int> tr(n);
    for (int k = 0; k < n; ++k) {
      int p = k;
      double best = std::abs(lu(k, k));
      for (int i = k + 1; i < n; ++i) {
        double v = std::abs(lu(i, k));
        if (v > best) { best = v; p = i; }
      }
      tr[k] = p;
      if (best != 0.0) {
        if (p != k)
          for (int j = 0; j < n; ++j) std::swap(lu(k, j), lu(p, j));
        const cd piv = lu(k, k);
        for (int i = k + 1; i < n; ++i) lu(i, k) /= piv;
      }
      const long work = (long)(n - k) * (n - k);
#pragma omp parallel for schedule(static) if (work > 100000)
      for (int j = k + 1; j < n; ++j) axpyC(n - k - 1, -lu(k, j), &lu(k + 1, k), &lu(k + 1, j));
    }
    perm.resize(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int k = 0; k < n; ++k) std::swap(perm[k], perm[tr[k]]);
  }
  Mat solve(const Mat& B) const {
    if (B.r != n) fail("LU solve size mismatch");
    Mat X(n, B.c);
    const long work = (long)n * n * B.c;
#pragma omp parallel for schedule(static) if (work > 200000)
    for (int j = 0; j < B.c; ++j) {
      cd* x = &X.a[(size_t)j * n];
      for (int i = 0; i < n; ++i) x[i] = B(perm[i], j);
      for (int k = 0; k < n; ++k)  // unit lower, column oriented
        if (x[k] != cd(0.0, 0.0)) axpyC(n - k - 1, -x[k], &lu.a[(size_t)k * n + k + 1], x + k + 1);
      for (int k = n - 1; k >= 0; --k) {  // upper, column oriented
        x[k] = x[k] / lu(k, k);
        if (x[k] != cd(0.0, 0.0)) axpyC(k, -x[k], &lu.a[(size_t)k * n], x);
      }
    }
    return X;
  }
};

// Largest column 2-norm: |R(0,0)| of a column-pivoting Householder QR.
inline double maxColumnNorm(const Mat& A) {
  if (A.c == 0) fail("maxColumnNorm of empty matrix");
  double best = -1.0;
  for (int j = 0; j < A.c; ++j) {
    double s = 0.0;
    for (int i = 0; i < A.r; ++i) s += std::norm(A(i, j));
    s = std::sqrt(s);
    if (s > best) best = s;
  }
  return best;
}

}  // namespace orc
