// Electrostatics through the reference's class API in a USE_DOUBLE build (real
// dtype, as the reference requires for ElectrostaticsMatrix): capacitance of
// conductor 1 by AIFMM and by dense LU, and an RRQR of a real block.
//
// usage: dropin_es_double <nodeList> <patchList> <TOL_POW> <fillin_tol> <leafSize>
#include "AIFMM.hpp"
#include "rrqr.hpp"

int main(int argc, char* argv[]) {
  if (argc < 6) return 2;
  inputsToKernelClass ik;
  ik.nodeListFilename = argv[1];
  ik.patchListFilename = argv[2];
  ik.n = 0;
  ik.L = 0.0;
  ElectrostaticsMatrix E(ik);
  Eigen::MatrixX3d cen;
  E.getCentroids(cen);
  Eigen::MatrixXd loc(cen.rows(), 3);
  for (Eigen::Index r = 0; r < cen.rows(); ++r)
    for (int q = 0; q < 3; ++q) loc(r, q) = cen(r, q);
  Eigen::VectorXd hi = loc.colwise().maxCoeff(), lo = loc.colwise().minCoeff();
  inputsToSolverClass in;
  in.xmin = lo(0);
  in.xmax = hi(0);
  in.ymin = lo(1);
  in.ymax = hi(1);
  in.zmin = lo(2);
  in.zmax = hi(2);
  in.leafSize = atoi(argv[5]);
  in.tol_pow = atoi(argv[3]);
  in.fillin_tol = atoi(argv[4]);
  in.nLevelsInput = 0;
  in.fillin_rank = 5;
  in.locations = loc;
  Vec rhs, q, qLU;
  E.getRhs(1, rhs);
  E.getchargeDensityUsingLU(rhs, qLU);
  AIFMM<ElectrostaticsMatrix> S(in, &E);
  S.factorize();
  S.backSubstitute1(rhs);
  S.backSubstitute2();
  S.backSubstitute3();
  S.getPhi(q);
  std::cout.precision(17);
  std::cout << "N " << E.N << "\n";
  std::cout << "capacitance_lu " << E.getCapacitance(qLU) << "\n";
  std::cout << "capacitance_aifmm " << E.getCapacitance(q) << "\n";
  std::cout << "charge_diff " << (q - qLU).norm() / qLU.norm() << "\n";
  std::vector<int> rows, cols;
  for (int r = 0; r < E.N / 2; ++r) rows.push_back(r);
  for (int c2 = E.N / 2; c2 < E.N; ++c2) cols.push_back(c2);
  Mat B = E.getMatrix(rows, cols);
  RRQR qr(B, 8, 10, 0, 1.0, 0, (int)cols.size());
  qr.colPivHouseholderQRWithPartition();
  std::cout << "rrqr_rank " << qr.Q_trunc.cols() << "\n";
  std::cout << "rrqr_error " << qr.errorInQR() << "\n";
  std::cout << "done 1\n";
  return 0;
}
