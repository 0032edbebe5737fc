// A driver written against the reference's C++ class API (the AIFMM<K>
// facade, FMM2DTree members, EFIEMatrix / ElectrostaticsMatrix, LowRank and
// RRQR), built with include/aifmm/ and libaifmm_b200.  It follows the steps of
// a sphere scattering run and writes every result to text files that
// tests/test_dropin_gpu.py compares with the oracle.
//
// usage: dropin_driver <nodeList> <patchList> <outdir> <TOL_POW> <fillin_tol> <leafSize>
#include <cstdio>

#include "ACA.hpp"
#include "AIFMM.hpp"
#include "rrqr.hpp"

static void writeVec(const std::string& path, const Eigen::VectorXcd& v) {
  std::ofstream f(path.c_str());
  f.precision(17);
  for (Eigen::Index i = 0; i < v.size(); ++i) f << v(i).real() << " " << v(i).imag() << "\n";
}

static void writeMat(const std::string& path, const Eigen::MatrixXcd& m) {  // column by column
  std::ofstream f(path.c_str());
  f.precision(17);
  f << m.rows() << " " << m.cols() << "\n";
  for (Eigen::Index j = 0; j < m.cols(); ++j)
    for (Eigen::Index i = 0; i < m.rows(); ++i) f << m(i, j).real() << " " << m(i, j).imag() << "\n";
}

int main(int argc, char* argv[]) {
  if (argc < 7) {
    std::cerr << "usage: dropin_driver nodeList patchList outdir TOL_POW fillin_tol leafSize" << std::endl;
    return 2;
  }
  const std::string out = argv[3];
  const int TOL_POW = atoi(argv[4]), fillin_tol = atoi(argv[5]), leafSize = atoi(argv[6]);
  std::ofstream summary((out + "/summary.txt").c_str());
  summary.precision(17);

  // ---- EFIE kernel and the driver's unknown locations (edge midpoints)
  inputsToKernelClass inputsToKernel;
  inputsToKernel.nodeListFilename = argv[1];
  inputsToKernel.patchListFilename = argv[2];
  inputsToKernel.n = 0;
  inputsToKernel.L = 0.0;
  EFIEMatrix* K = new EFIEMatrix(inputsToKernel);
  const int N = K->N;
  Eigen::MatrixXd mid(N, 3);
  int i = 0;
  for (auto& kv : K->edge2PatchMap) {
    Node a = K->nodeList[kv.first.first], b = K->nodeList[kv.first.second];
    mid.row(i++) = (a + b) / 2.0;
  }
  Eigen::VectorXd hi = mid.colwise().maxCoeff(), lo = mid.colwise().minCoeff();
  inputsToSolverClass in;
  in.xmin = lo(0);
  in.xmax = hi(0);
  in.ymin = lo(1);
  in.ymax = hi(1);
  in.zmin = lo(2);
  in.zmax = hi(2);
  in.leafSize = leafSize;
  in.tol_pow = TOL_POW;
  in.nLevelsInput = 0;
  in.fillin_rank = 5;
  in.fillin_tol = fillin_tol;
  in.locations = mid;
  summary << "N " << N << "\nconductors " << K->conductorIndices.size() << "\n";

  // ---- right-hand side and the dense reference solution
  Node Einc;
  Einc(0) = 1.0;
  Einc(1) = 0.0;
  Einc(2) = 0.0;
  Eigen::VectorXcd rhs, xLU;
  K->getRhs(Einc, rhs);
  K->getCoefficients(rhs, xLU);
  writeVec(out + "/rhs.txt", rhs);
  writeVec(out + "/x_lu.txt", xLU);
  summary << "rhs_entry_5 " << std::abs(K->getRhs(Einc, 5) - rhs(5)) << "\n";
  summary << "entry_3_7 " << K->getMatrixEntry(3, 7).real() << " " << K->getMatrixEntry(3, 7).imag() << "\n";

  // ---- AIFMM: assemble, factorize, solve in the reference's three steps
  AIFMM<EFIEMatrix>* solver = new AIFMM<EFIEMatrix>(in, K);
  summary << "avg_leaf " << solver->A->getAvgLeafSize() << "\n";
  summary << "avg_rank " << solver->A->getAvgMultipoles() << "\n";
  summary << "levels " << solver->A->nLevels << "\n";
  summary << "mem " << solver->A->findMemory() << "\n";
  solver->factorize();
  summary << "mem_after " << solver->A->findMemoryAfterFactorize() << "\n";
  solver->backSubstitute1(rhs);
  solver->backSubstitute2();
  solver->backSubstitute3();
  Eigen::VectorXcd phi;
  solver->getPhi(phi);
  writeVec(out + "/phi.txt", phi);
  Vec tree = solver->solve(rhs);  // tree order, as the reference's solve()
  writeVec(out + "/phi_tree.txt", tree);
  Vec back = tree;
  solver->A->reorder(back);
  summary << "reorder_diff " << (back - phi).norm() << "\n";

  // ---- backward error with exact columns, as the reference's driver does
  Vec Ax = Vec::Zero(N);
  for (int j = 0; j < N; ++j) Ax = Ax + phi(j) * solver->A->K->getCol(N, j);
  summary << "backward_error " << (Ax - rhs).norm() / rhs.norm() << "\n";

  // ---- far field of the dense solution: centroid currents and RCS
  Eigen::MatrixXcd J;
  K->getJAtCentroids(xLU, J);
  writeMat(out + "/J.txt", J);
  {
    std::ofstream f((out + "/rcs.txt").c_str());
    f.precision(17);
    for (int deg = 0; deg <= 180; deg += 5) {
      const double th = deg / 180.0 * PI;
      f << th << " " << K->getRCS_OnePointQuadrature(th, 0.0, J) << "\n";
    }
  }

  // ---- RRQR and ACA on the block of the first half of the unknowns against the second
  std::vector<int> rows, cols;
  for (int r = 0; r < N / 2; ++r) rows.push_back(r);
  for (int q = N / 2; q < N; ++q) cols.push_back(q);
  Mat B = K->getMatrix(rows, cols);
  writeMat(out + "/block.txt", B);
  RRQR qr(B, TOL_POW, fillin_tol, 0, 1.0, 0, (int)cols.size());
  qr.colPivHouseholderQRWithPartition();
  writeMat(out + "/rrqr_q.txt", qr.Q_trunc);
  writeMat(out + "/rrqr_r.txt", qr.R_trunc);
  {
    std::ofstream f((out + "/rrqr_perm.txt").c_str());
    for (Eigen::Index q = 0; q < qr.P.cols(); ++q)
      for (Eigen::Index r = 0; r < qr.P.rows(); ++r)
        if (qr.P(r, q) == dtype(1.0)) f << r << "\n";
  }
  summary << "rrqr_rank " << qr.Q_trunc.cols() << "\nrrqr_maxpivot " << qr.maxPivot << "\n";
  summary << "rrqr_error " << qr.errorInQR() << "\n";
  LowRank<EFIEMatrix> lr(K, std::pow(10.0, -TOL_POW), rows, cols);
  std::vector<int> rb, cb;
  int rank = 0;
  Mat Ac, Ar;
  lr.ACA_only_nodes2(rb, cb, rank, Ac, Ar);
  summary << "aca_rank " << rank << "\naca_rows";
  for (int r : rb) summary << " " << r;
  summary << "\naca_cols";
  for (int q : cb) summary << " " << q;
  summary << "\n";
  writeMat(out + "/aca_ac.txt", Ac);

  // ---- electrostatics on the same mesh: capacitance by AIFMM and by dense LU
  ElectrostaticsMatrix* E = new ElectrostaticsMatrix(inputsToKernel);
  Eigen::MatrixX3d cen;
  E->getCentroids(cen);
  Eigen::MatrixXd cloc(cen.rows(), 3);
  for (Eigen::Index r = 0; r < cen.rows(); ++r)
    for (int q = 0; q < 3; ++q) cloc(r, q) = cen(r, q);
  Eigen::VectorXd chi = cloc.colwise().maxCoeff(), clo = cloc.colwise().minCoeff();
  inputsToSolverClass es = in;
  es.xmin = clo(0);
  es.xmax = chi(0);
  es.ymin = clo(1);
  es.ymax = chi(1);
  es.zmin = clo(2);
  es.zmax = chi(2);
  es.locations = cloc;
  Eigen::VectorXd v1, qLU;
  E->getRhs(1, v1);
  E->getchargeDensityUsingLU(v1, qLU);
  AIFMM<ElectrostaticsMatrix>* esSolver = new AIFMM<ElectrostaticsMatrix>(es, E);
  esSolver->factorize();
  Vec v1c(v1.size());
  for (Eigen::Index r = 0; r < v1.size(); ++r) v1c(r) = v1(r);
  esSolver->backSubstitute(v1c);
  Vec qc;
  esSolver->getPhi(qc);
  Eigen::VectorXd q(qc.size());
  for (Eigen::Index r = 0; r < qc.size(); ++r) q(r) = std::real(qc(r));
  summary << "capacitance_lu " << E->getCapacitance(qLU) << "\ncapacitance_aifmm " << E->getCapacitance(q) << "\n";
  Eigen::MatrixXd Q1(qLU.size(), 1), Cm;
  for (Eigen::Index r = 0; r < qLU.size(); ++r) Q1(r, 0) = qLU(r);
  E->getCapacitanceMatrix(Q1, Cm);
  summary << "capacitance_matrix " << Cm(0, 0) << "\n";

  delete esSolver;
  delete solver;
  summary << "done 1\n";
  return 0;
}
