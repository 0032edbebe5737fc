// Drop-in replacement for the reference's include/kernel.hpp: the abstract
// matrix-entry kernel and its gathers (include/kernel.hpp:13-47,
// src/kernel.cpp:11-82).
//
// A kernel that is backed by the library (EFIEMatrix, ElectrostaticsMatrix)
// sets `handle`; its gathers then evaluate the whole block in one GPU launch
// instead of one virtual getMatrixEntry call per entry.  A user kernel that
// only overrides getMatrixEntry keeps the reference's per-entry gathers (and
// cannot drive AIFMM<K>, whose assembly runs on the GPU).
#ifndef AIFMM_DROPIN_KERNEL_HPP
#define AIFMM_DROPIN_KERNEL_HPP

#include "includes.hpp"

class kernel {
 public:
  bool isTrans = false;     // translation invariant K(r)
  bool isHomog = false;     // homogeneous K(r) = r^alpha
  bool isLogHomog = false;  // log-homogeneous K(r) = log(r^alpha)
  double alpha = 0.0;
  double a = 0.0;

  std::vector<pts2D> particles_X;
  std::vector<pts2D> particles_Y;

  aifmm_kernel* handle = nullptr;  // set by library-backed kernels

  kernel() {}
  virtual ~kernel() {}

  virtual dtype getMatrixEntry(const unsigned i, const unsigned j) {
    if (handle) {
      const int r = (int)i, col = (int)j;
      return gather(&r, 1, &col, 1)(0, 0);
    }
    std::cout << "virtual getInteraction" << std::endl;
    return dtype(0.0);
  }

  // row j restricted to col_indices (kernel.cpp:11-19)
  Vec getRow(const int j, std::vector<int> col_indices) {
    if (handle) return Vec(gather(&j, 1, col_indices.data(), (int)col_indices.size()).transpose());
    Vec row((Eigen::Index)col_indices.size());
    for (size_t k = 0; k < col_indices.size(); ++k) row((Eigen::Index)k) = getMatrixEntry(j, col_indices[k]);
    return row;
  }
  // column k restricted to row_indices (kernel.cpp:21-29)
  Vec getCol(const int k, std::vector<int> row_indices) {
    if (handle) return Vec(gather(row_indices.data(), (int)row_indices.size(), &k, 1));
    Vec col((Eigen::Index)row_indices.size());
    for (size_t j = 0; j < row_indices.size(); ++j) col((Eigen::Index)j) = getMatrixEntry(row_indices[j], k);
    return col;
  }
  // entries (0..n-1, k) (kernel.cpp:31-38)
  Vec getCol(const int n, const int k) {
    std::vector<int> rows(n);
    for (int j = 0; j < n; ++j) rows[j] = j;
    return getCol(k, rows);
  }
  // entries (k, 0..n-1) (kernel.cpp:40-47)
  Vec getRow(const int n, const int k) {
    std::vector<int> cols(n);
    for (int j = 0; j < n; ++j) cols[j] = j;
    return getRow(k, cols);
  }
  // K(row_indices, col_indices) (kernel.cpp:49-61)
  Mat getMatrix(std::vector<int> row_indices, std::vector<int> col_indices) {
    if (handle) return gather(row_indices.data(), (int)row_indices.size(), col_indices.data(), (int)col_indices.size());
    Mat m((Eigen::Index)row_indices.size(), (Eigen::Index)col_indices.size());
    for (size_t j = 0; j < row_indices.size(); ++j)
      for (size_t k = 0; k < col_indices.size(); ++k)
        m((Eigen::Index)j, (Eigen::Index)k) = getMatrixEntry(row_indices[j], col_indices[k]);
    return m;
  }
  // K(row_start..row_end-1, col_start..col_end-1) (kernel.cpp:63-73).  The
  // reference stores entry (j, k) at (j, k), which is only in range when both
  // starts are 0; here it goes to (j - row_start, k - col_start), the same
  // placement in that case.
  Mat getMatrix(int row_start_index, int col_start_index, int row_end_index, int col_end_index) {
    std::vector<int> rows, cols;
    for (int j = row_start_index; j < row_end_index; ++j) rows.push_back(j);
    for (int k = col_start_index; k < col_end_index; ++k) cols.push_back(k);
    return getMatrix(rows, cols);
  }
  // the dense Nsize x Nsize matrix (kernel.cpp:75-82)
  void getMatrix(Mat& mat, int Nsize) { mat = getMatrix(0, 0, Nsize, Nsize); }

 protected:
  Mat gather(const int* rows, int nr, const int* cols, int nc) {
    std::vector<std::complex<double>> buf((size_t)std::max(nr, 1) * (size_t)std::max(nc, 1));
    Mat m;
    if (nr == 0 || nc == 0) {
      m.resize(nr, nc);
      return m;
    }
    aifmm_dropin::check(aifmm_kernel_matrix(handle, rows, nr, cols, nc, 0, buf.data(), nr));
    aifmm_dropin::from_c128(buf.data(), nr, nc, m);
    return m;
  }
};

#endif
