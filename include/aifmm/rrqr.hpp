// Drop-in replacement for the reference's include/rrqr.hpp: column-pivoted
// Householder QR in two partitions with rank truncation (include/rrqr.hpp:5-27,
// src/rrqr.cpp:3-187).  colPivHouseholderQRWithPartition runs on the GPU
// through aifmm_rrqr_full.
//
// Outputs as in the reference: Q_trunc (m x rank), R_trunc (rank x n, upper
// trapezoidal, R_trunc = Q_trunc^H A P), P (n x n permutation) and maxPivot.
// The first rank columns of P are the reference's pivots; the order of the
// remaining columns differs (the reference re-sorts them at every step).
// maxPivotPartition1/2 are not reported by the GPU kernel and stay NaN.
#ifndef AIFMM_DROPIN_RRQR_HPP
#define AIFMM_DROPIN_RRQR_HPP

#include <limits>

#include "includes.hpp"

class RRQR {
 public:
  Mat A;
  int fillInRank;
  int partition;
  double inputPivot;
  double maxPivot = 0.0;
  double maxPivotPartition1 = std::numeric_limits<double>::quiet_NaN();
  double maxPivotPartition2 = std::numeric_limits<double>::quiet_NaN();
  double tolerance1;
  double tolerance2;
  Mat Q_trunc;
  Mat R_trunc;
  Mat P;
  int flag;

  // RRQR(A, TOL_POW1, TOL_POW2, partition, inputPivot, flag, fillInRank) (rrqr.cpp:3-11)
  RRQR(Mat& A, int TOL_POW1, int TOL_POW2, int partition, double inputPivot, int flag, int fillInRank)
      : A(A),
        fillInRank(fillInRank),
        partition(partition),
        inputPivot(inputPivot),
        tolerance1(std::pow(10.0, -TOL_POW1)),
        tolerance2(std::pow(10.0, -TOL_POW2)),
        flag(flag),
        tolPow1_(TOL_POW1),
        tolPow2_(TOL_POW2) {}

  // rrqr.cpp:98-182
  void colPivHouseholderQRWithPartition() {
    const int m = (int)A.rows(), n = (int)A.cols();
    if (m == 0 || n == 0) {
      Q_trunc.resize(m, 0);
      R_trunc.resize(0, n);
      P = Mat::Identity(n, n);
      return;
    }
    const int mn = std::min(m, n);
    std::vector<std::complex<double>> a = aifmm_dropin::to_c128(A), q((size_t)m * mn), r((size_t)mn * n);
    std::vector<int> perm((size_t)n);
    int rank = 0;
#if defined(USE_DOUBLE)
    const int real_mode = 1;  // real Householder sign, as a USE_DOUBLE build of the reference
#else
    const int real_mode = 0;
#endif
    aifmm_dropin::check(aifmm_rrqr_full(aifmm_dropin::context(), reinterpret_cast<double*>(a.data()), m, n, partition,
                                        tolPow1_, tolPow2_, inputPivot, fillInRank, real_mode,
                                        reinterpret_cast<double*>(q.data()), reinterpret_cast<double*>(r.data()),
                                        perm.data(), &rank, &maxPivot));
    aifmm_dropin::from_c128(q.data(), m, rank, Q_trunc);
    aifmm_dropin::from_c128(r.data(), rank, n, R_trunc);
    P = Mat::Zero(n, n);
    for (int j = 0; j < n; ++j) P(perm[(size_t)j], j) = dtype(1.0);
  }

  void printVec(std::vector<int>& v) {
    for (int x : v) std::cout << x << ", " << std::endl;
    std::cout << std::endl;
  }
  void printVec(std::vector<double>& v) {
    for (double x : v) std::cout << x << ", " << std::endl;
    std::cout << std::endl;
  }
  // Householder vector of x over rows [i, j): v = x(i:j) + phase(x_i) |x(i:j)| e_i,
  // scaled to norm sqrt(2) (rrqr.cpp:75-96)
  void gethouselholderVec(Vec x, int i, int j, Vec& v) {
    v = Vec::Zero(x.size());
    double s = 0.0;
    for (int k = i; k < j; ++k) {
      v(k) = x(k);
      s += std::norm(x(k));
    }
    s = std::sqrt(s);
#if defined(USE_DOUBLE)
    v(i) = v(i) + mySign(x(i)) * s;
#else
    v(i) = v(i) + std::exp(I * std::arg(x(i))) * s;
#endif
    const double nv = v.norm();
    if (nv > 0) v = v * (std::sqrt(2.0) / nv);
  }
  int mySign(double x) { return x >= 0 ? 1 : -1; }
  // ||A P - Q_trunc R_trunc|| / ||A|| (rrqr.cpp:184-187), products on the GPU
  double errorInQR() {
    const int m = (int)A.rows(), n = (int)A.cols(), r = (int)Q_trunc.cols();
    if (m == 0 || n == 0) return 0.0;
    std::vector<std::complex<double>> ap((size_t)m * n), q = aifmm_dropin::to_c128(Q_trunc),
                                                         rr = aifmm_dropin::to_c128(R_trunc), a = aifmm_dropin::to_c128(A),
                                                         p = aifmm_dropin::to_c128(P);
    const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0}, minus[2] = {-1.0, 0.0};
    aifmm_dropin::check(aifmm_zgemm(aifmm_dropin::context(), 0, 0, 0, m, n, n, one, reinterpret_cast<double*>(a.data()),
                                    m, reinterpret_cast<double*>(p.data()), n, zero,
                                    reinterpret_cast<double*>(ap.data()), m));
    if (r > 0)
      aifmm_dropin::check(aifmm_zgemm(aifmm_dropin::context(), 0, 0, 0, m, n, r, minus,
                                      reinterpret_cast<double*>(q.data()), m, reinterpret_cast<double*>(rr.data()), r,
                                      one, reinterpret_cast<double*>(ap.data()), m));
    double e = 0.0, na = 0.0;
    for (auto& v : ap) e += std::norm(v);
    for (auto& v : a) na += std::norm(v);
    return na > 0 ? std::sqrt(e / na) : 0.0;
  }

 private:
  int tolPow1_, tolPow2_;
};

#endif
