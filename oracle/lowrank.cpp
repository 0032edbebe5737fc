// CPU oracle -- TEST INFRASTRUCTURE ONLY.  See lowrank.hpp.
#include "lowrank.hpp"

#include <cfloat>
#include <numeric>

namespace orc {

// maxAbsVector, ACA.cpp:25-38: strict '>' so the lowest allowed index wins
// ties.  An empty allowed set is undefined in the reference; it is only
// reached right before the loop exits, so index 0 is returned.
static void maxAbsVector(const Mat& v, const std::set<int>& allowed, cd& mx, int& index) {
  if (allowed.empty()) {
    index = 0;
    mx = v.size() ? v(0) : cd(0, 0);
    return;
  }
  index = *allowed.begin();
  mx = v(index);
  for (int it : allowed) {
    if (std::abs(v(it)) > std::abs(mx)) {
      index = it;
      mx = v(index);
    }
  }
}

static double vnorm(const Mat& v) { return v.norm(); }

// ACA_only_nodes2, ACA.cpp:639-859.
void acaOnlyNodes2(const Kernel& K, double tol, const std::vector<int>& row_indices,
                   const std::vector<int>& col_indices, ACAResult& out) {
  out = ACAResult();
  int col_index = 0, row_index = 0;
  const int N1 = (int)row_indices.size(), N2 = (int)col_indices.size();
  Mat row(N2, 1), col(N1, 1), v(N2, 1), u(N1, 1);
  Mat row_temp, col_temp;
  std::vector<Mat> Uvec, Vvec, AcVec, ArVec;
  int computed_rank = 0;
  cd mx;
  int mn = N1;
  if (N1 > N2) mn = N2;
  std::set<int> rrow, rcol;
  for (int l = 0; l < N1; ++l) rrow.insert(l);
  for (int l = 0; l < N2; ++l) rcol.insert(l);
  auto finish = [&]() {
    out.rank = computed_rank;
    out.Ac = Mat(N1, computed_rank);
    out.Ar = Mat(computed_rank, N2);
    for (int i = 0; i < computed_rank; ++i) {
      out.Ac.setBlock(0, i, AcVec[i]);
      for (int s = 0; s < N2; ++s) out.Ar(i, s) = ArVec[i](s);
    }
  };
  if (N1 < N2) {
    int l_local;
    for (l_local = 0; l_local < N1; l_local++) {
      row_index = l_local;
      row = K.getRow(row_indices[row_index], col_indices);
      maxAbsVector(row, rcol, mx, col_index);
      if (std::abs(row(col_index)) > std::pow(10, -16)) break;
    }
    if (l_local == N1) {
      finish();
      return;
    }
    v = row / row(col_index);
    out.rowBases.push_back(row_index);
    out.colBases.push_back(col_index);
    col = K.getCol(col_indices[col_index], row_indices);
    u = col;
    Uvec.push_back(u);
    Vvec.push_back(v);
    AcVec.push_back(col);
    ArVec.push_back(row);
    rcol.erase(col_index);
    rrow.erase(row_index);
    computed_rank = 1;
    double normS = 0.0;
    double prev_normS = DBL_MAX;
    maxAbsVector(col, rrow, mx, row_index);
    while (vnorm(u) * vnorm(v) > tol * normS && computed_rank < mn) {
      out.rowBases.push_back(row_index);
      row = K.getRow(row_indices[row_index], col_indices);
      row_temp = row;
      for (int l = 0; l <= computed_rank - 1; ++l)
        for (int s = 0; s < Vvec[l].r; ++s) row(s) -= Uvec[l](row_index) * Vvec[l](s);
      maxAbsVector(row, rcol, mx, col_index);
      out.colBases.push_back(col_index);
      for (int l = 0; l < row.r; ++l) v(l) = row(l) / row(col_index);
      col = K.getCol(col_indices[col_index], row_indices);
      col_temp = col;
      for (int l = 0; l <= computed_rank - 1; ++l)
        for (int s = 0; s < Uvec[l].r; ++s) col(s) -= Vvec[l](col_index) * Uvec[l](s);
      u = col;
      Uvec.push_back(u);
      Vvec.push_back(v);
      AcVec.push_back(col_temp);
      ArVec.push_back(row_temp);
      ++computed_rank;
      rcol.erase(col_index);
      rrow.erase(row_index);
      if (computed_rank != 2) prev_normS = normS;
      normS = std::pow(normS, 2) + std::pow(vnorm(u) * vnorm(v), 2);
      for (int l = 0; l <= computed_rank - 1; ++l) normS += 2 * std::abs(dotc(Uvec[l], u) * dotc(Vvec[l], v));
      normS = std::sqrt(normS);
      maxAbsVector(col, rrow, mx, row_index);
    }
  } else {
    int l_local;
    for (l_local = 0; l_local < N2; l_local++) {
      col_index = l_local;
      col = K.getCol(col_indices[col_index], row_indices);
      maxAbsVector(col, rrow, mx, row_index);
      if (std::abs(col(row_index)) > std::pow(10, -16)) break;
    }
    if (l_local == N2) {
      finish();
      return;
    }
    out.colBases.push_back(col_index);
    v = col / col(row_index);
    out.rowBases.push_back(row_index);
    row = K.getRow(row_indices[row_index], col_indices);
    u = row;
    Uvec.push_back(u);
    Vvec.push_back(v);
    AcVec.push_back(col);
    ArVec.push_back(row);
    computed_rank = 1;
    rrow.erase(row_index);
    rcol.erase(col_index);
    double normS = 0.0;
    double prev_normS = DBL_MAX;
    maxAbsVector(row, rcol, mx, col_index);
    while (vnorm(u) * vnorm(v) > tol * normS && computed_rank < mn) {
      out.colBases.push_back(col_index);
      col = K.getCol(col_indices[col_index], row_indices);
      col_temp = col;
      for (int l = 0; l <= computed_rank - 1; ++l)
        for (int s = 0; s < Vvec[l].r; ++s) col(s) -= Uvec[l](col_index) * Vvec[l](s);
      maxAbsVector(col, rrow, mx, row_index);
      out.rowBases.push_back(row_index);
      for (int l = 0; l < col.r; ++l) v(l) = col(l) / col(row_index);
      row = K.getRow(row_indices[row_index], col_indices);
      row_temp = row;
      for (int l = 0; l <= computed_rank - 1; ++l)
        for (int s = 0; s < Uvec[l].r; ++s) row(s) -= Vvec[l](row_index) * Uvec[l](s);
      u = row;
      Uvec.push_back(u);
      Vvec.push_back(v);
      AcVec.push_back(col_temp);
      ArVec.push_back(row_temp);
      ++computed_rank;
      rrow.erase(row_index);
      rcol.erase(col_index);
      if (computed_rank != 2) prev_normS = normS;
      normS = std::pow(normS, 2) + std::pow(vnorm(u) * vnorm(v), 2);
      for (int l = 0; l <= computed_rank - 1; ++l) normS += 2 * std::abs(dotc(Uvec[l], u) * dotc(Vvec[l], v));
      normS = std::sqrt(normS);
      maxAbsVector(row, rcol, mx, col_index);
    }
  }
  (void)mx;
  finish();
}

// gethouselholderVec, rrqr.cpp:75-96.
static void householderVec(const Mat& R, int colj, int i, int n, bool realMode, Mat& v) {
  v = Mat(n, 1);
  double sq = 0.0;
  for (int q = i; q < n; ++q) {
    v(q) = R(q, colj);
    sq += std::norm(R(q, colj));
  }
  const double sn = std::sqrt(sq);
  const cd xi = R(i, colj);
  if (realMode) {
    const int sgn = (xi.real() >= 0) ? 1 : -1;
    v(i) = v(i) + double(sgn) * sn;
  } else {
    v(i) = v(i) + std::exp(cd(0.0, 1.0) * std::arg(xi)) * sn;
  }
  const double vn = v.norm();
  if (vn > 0) v = v * std::sqrt(2.0) / vn;
}

// colPivHouseholderQRWithPartition, rrqr.cpp:98-182.  The column order is
// kept as a permutation (position -> physical column) re-sorted each step with
// the reference's two std::sort calls, so pivot choices and ties are the
// reference's.  A reflector is applied only to the columns at positions >= j:
// the others are zero in rows >= j, where the reflector acts, so the values
// are the same as applying it to all of R.  Q_trunc is formed once from the
// committed reflectors, which equals the reference's explicit accumulation.
void rrqrPartition(const Mat& A, int tolPow1, int tolPow2, int partition, double inputPivot, int fillInRank,
                   bool realMode, RRQRResult& out) {
  out = RRQRResult();
  const double tolerance1 = std::pow(10.0, -tolPow1);
  const double tolerance2 = std::pow(10.0, -tolPow2);
  const int n_rows = A.r, n_cols = A.c;
  int steps = (n_cols < n_rows) ? n_cols : n_rows;
  Mat R = A;
  std::vector<int> phys(n_cols);
  std::iota(phys.begin(), phys.end(), 0);
  std::vector<double> nsq(n_cols);
  for (int j = 0; j < n_cols; ++j) {
    double s = 0.0;
    for (int i = 0; i < n_rows; ++i) s += std::norm(R(i, j));
    nsq[j] = s;
  }
  std::vector<Mat> refl;
  double maxPivot = 0.0, mp1 = 0.0, mp2 = 0.0;
  int rank_partition1 = std::min(partition, n_rows);
  auto sortStep = [&](int j, int endSort) {
    std::vector<int> idx(nsq.size());
    std::iota(idx.begin(), idx.end(), 0);
    std::sort(idx.begin() + j, idx.begin() + endSort, [&](int i1, int i2) { return nsq[i1] > nsq[i2]; });
    std::sort(nsq.begin() + j, nsq.begin() + endSort, std::greater<double>());
    std::vector<int> np = phys;
    for (int q = j; q < endSort; ++q) np[q] = phys[idx[q]];
    phys = np;
  };
  // Householder vector of the column at position j and w_q = h^H R(:, phys[q])
  // for q >= j; returns the would-be pivot R(j, phys[j]) after the reflection.
  std::vector<cd> w(n_cols);
  auto reflect = [&](int j, Mat& h) -> cd {
    householderVec(R, phys[j], j, n_rows, realMode, h);
    for (int q = j; q < n_cols; ++q) {
      const int c = phys[q];
      cd s(0, 0);
      for (int i = j; i < n_rows; ++i) s += std::conj(h(i)) * R(i, c);
      w[q] = s;
    }
    return R(j, phys[j]) - h(j) * w[j];
  };
  auto commit = [&](int j, const Mat& h) {
    for (int q = j; q < n_cols; ++q) {
      const int c = phys[q];
      for (int i = j; i < n_rows; ++i) R(i, c) -= h(i) * w[q];
    }
    for (int i = j + 1; i < n_rows; ++i) R(i, phys[j]) = 0.0;
    refl.push_back(h);
    for (int q = j + 1; q < n_cols; ++q) nsq[q] = nsq[q] - std::abs(R(j, phys[q])) * std::abs(R(j, phys[q]));
  };
  for (int j = 0; j < rank_partition1; ++j) {
    sortStep(j, partition);
    Mat h;
    const cd rjj = reflect(j, h);
    if (j == 0) mp1 = std::abs(rjj);
    maxPivot = mp1;
    const double pivot = std::abs(rjj);
    if (pivot / mp1 < tolerance1) {
      rank_partition1 = j - 1;  // reference quirk (rrqr.cpp:116)
      break;
    }
    commit(j, h);
  }
  for (int i = rank_partition1; i < partition; ++i) nsq[i] = 0.0;
  steps = steps - (partition - rank_partition1);
  const int first = rank_partition1;
  int rank_partition2 = std::min(steps - first, n_rows);
  for (int j = first; j < steps; ++j) {
    sortStep(j, n_cols);
    Mat h;
    const cd rjj = reflect(j, h);
    if (j == first) {
      mp2 = std::abs(rjj);
      maxPivot = std::max(inputPivot, mp2);
    }
    const double pivot = std::abs(rjj);
    if (pivot / maxPivot < tolerance2 || j - first >= fillInRank) {
      rank_partition2 = j - first;
      break;
    }
    commit(j, h);
  }
  const int rank_A = rank_partition1 + rank_partition2;
  if (rank_A < 0 || rank_A > n_rows) fail("RRQR rank out of range");
  // Q_trunc = H_0 H_1 ... H_{t-1} [I; 0]
  Mat Q = Mat::Identity(n_rows, rank_A);
  for (int r = (int)refl.size() - 1; r >= 0; --r) {
    const Mat& h = refl[r];
    for (int c = 0; c < rank_A; ++c) {
      cd s(0, 0);
      for (int i = 0; i < n_rows; ++i) s += std::conj(h(i)) * Q(i, c);
      for (int i = 0; i < n_rows; ++i) Q(i, c) -= h(i) * s;
    }
  }
  out.Q = Q;
  out.R = Mat(rank_A, n_cols);
  for (int q = 0; q < n_cols; ++q)
    for (int i = 0; i < rank_A; ++i) out.R(i, q) = R(i, phys[q]);
  out.P = Mat(n_cols, n_cols);
  for (int q = 0; q < n_cols; ++q) out.P(phys[q], q) = 1.0;
  out.rank = rank_A;
  out.maxPivot = maxPivot;
  out.maxPivotPartition1 = mp1;
  out.maxPivotPartition2 = mp2;
}

double rrqrError(const Mat& A, const RRQRResult& r) {  // rrqr.cpp:184-187
  Mat E = A * r.P - r.Q * r.R;
  return E.norm() / A.norm();
}

}  // namespace orc
