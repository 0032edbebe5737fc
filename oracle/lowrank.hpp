// CPU oracle -- TEST INFRASTRUCTURE ONLY.
//
// Restatement of the low-rank layer of vaishna77/RCS:
//   LowRank<K>::ACA_only_nodes2   src/ACA.cpp:639-859 (with maxAbsVector, :25-38)
//   RRQR::colPivHouseholderQRWithPartition  src/rrqr.cpp:69-182, errorInQR :184-187
// std::sort with the reference's comparator is used for the pivot order so
// that ties are broken exactly as a libstdc++ build of the reference does.
#pragma once
#include <set>
#include <vector>

#include "kernels.hpp"

namespace orc {

struct ACAResult {
  std::vector<int> rowBases, colBases;
  int rank = 0;
  Mat Ac, Ar;
};

// rows/cols are global unknown ids; the returned bases index into them.
void acaOnlyNodes2(const Kernel& K, double tol, const std::vector<int>& rows, const std::vector<int>& cols,
                   ACAResult& out);

struct RRQRResult {
  Mat Q, R, P;  // Q_trunc, R_trunc, P (column permutation matrix)
  int rank = 0;
  double maxPivot = 0.0;
  double maxPivotPartition1 = 0.0, maxPivotPartition2 = 0.0;
};

// realMode selects the USE_DOUBLE Householder sign (rrqr.cpp:85-89).
void rrqrPartition(const Mat& A, int tolPow1, int tolPow2, int partition, double inputPivot, int fillInRank,
                   bool realMode, RRQRResult& out);
double rrqrError(const Mat& A, const RRQRResult& r);

}  // namespace orc
