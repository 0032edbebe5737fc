// Drop-in replacement for the reference's include/ACA.hpp: partially pivoted
// adaptive cross approximation of a kernel block (include/ACA.hpp:7-29,
// src/ACA.cpp:25-38 and :639-859).  ACA_only_nodes2, the variant the
// reference's tree calls, runs on the GPU through aifmm_aca; the inactive
// variants (rookPiv, ACA_only_nodes, ACA_only_nodes1) are not provided.
#ifndef AIFMM_DROPIN_ACA_HPP
#define AIFMM_DROPIN_ACA_HPP

#include "kernel.hpp"

template <typename kerneltype>
class LowRank {
 public:
  kerneltype* K;
  double tol_ACA;
  double tol_robust;
  double tolerance_or_rank;
  std::vector<int> row_indices;
  std::vector<int> col_indices;

  LowRank(kerneltype* K, double tolerance_or_rank, std::vector<int>& row_indices, std::vector<int>& col_indices)
      : K(K),
        tol_ACA(tolerance_or_rank),
        tol_robust(tolerance_or_rank),
        tolerance_or_rank(tolerance_or_rank),
        row_indices(row_indices),
        col_indices(col_indices) {}

  // Largest |v(i)| over the allowed indices; ties keep the lowest index, as the
  // strict comparison of ACA.cpp:25-38 does.
  void maxAbsVector(const Vec& v, const std::set<int>& allowed_indices, dtype& max, int& index) {
    index = -1;
    max = dtype(0.0);
    double best = -1.0;
    for (int i : allowed_indices) {
      const double a = std::abs(v(i));
      if (a > best) {
        best = a;
        max = v(i);
        index = i;
      }
    }
  }

  // Cross approximation K(rows, cols) ~ Ac Ar^... with the reference's outputs
  // (ACA.cpp:639-859): row_bases / col_bases are positions in row_indices /
  // col_indices of the pivots, Ac (rows x rank) the original columns and
  // Ar (rank x cols) the original rows at those pivots.
  void ACA_only_nodes2(std::vector<int>& row_bases, std::vector<int>& col_bases, int& computed_rank, Mat& Ac, Mat& Ar) {
    if (!K->handle) throw std::runtime_error("aifmm: ACA needs a library-backed kernel");
    const int nr = (int)row_indices.size(), nc = (int)col_indices.size();
    row_bases.clear();
    col_bases.clear();
    computed_rank = 0;
    if (nr == 0 || nc == 0) {
      Ac.resize(nr, 0);
      Ar.resize(0, nc);
      return;
    }
    const int mn = std::min(nr, nc);
    std::vector<int> rb((size_t)mn), cb((size_t)mn);
    std::vector<std::complex<double>> ac((size_t)nr * mn), ar((size_t)mn * nc);
    aifmm_dropin::check(aifmm_aca(K->handle, row_indices.data(), nr, col_indices.data(), nc, tolerance_or_rank,
                                  rb.data(), cb.data(), &computed_rank, reinterpret_cast<double*>(ac.data()),
                                  reinterpret_cast<double*>(ar.data())));
    row_bases.assign(rb.begin(), rb.begin() + computed_rank);
    col_bases.assign(cb.begin(), cb.begin() + computed_rank);
    aifmm_dropin::from_c128(ac.data(), nr, computed_rank, Ac);
    aifmm_dropin::from_c128(ar.data(), computed_rank, nc, Ar);
  }
};

#endif
