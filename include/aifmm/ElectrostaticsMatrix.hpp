// Drop-in replacement for the reference's include/ElectrostaticsMatrix.hpp:
// the electrostatic collocation kernel with piecewise-constant charge on a
// triangle mesh (include/ElectrostaticsMatrix.hpp:8-40,
// src/ElectrostaticsMatrix.cpp).  Entries and the dense solve run on the GPU;
// the readers, the right-hand sides and the capacitance sums run on the host.
//
// getMatrixEntry returns dtype, so the class also builds with complex dtype
// (the reference's returns double and needs USE_DOUBLE).  The plate-mesh
// constructors and the quadrature helpers are not provided.
#ifndef AIFMM_DROPIN_ELECTROSTATICSMATRIX_HPP
#define AIFMM_DROPIN_ELECTROSTATICSMATRIX_HPP

#include <memory>

#include "Patch.hpp"
#include "includes.hpp"
#include "kernel.hpp"

class ElectrostaticsMatrix : public kernel {
 public:
  std::vector<Node> nodeList;
  std::vector<Patch> patchList;
  int N = 0;
  std::set<int> conductorIndices;
  int numConductors = 0;

  // ElectrostaticsMatrix(inputsToKernelClass) (ElectrostaticsMatrix.cpp:48-52)
  explicit ElectrostaticsMatrix(inputsToKernelClass inputsToKernel) {
    generateNodeList(inputsToKernel.nodeListFilename);
    generatePatchList(inputsToKernel.patchListFilename);
    getSizeOfMatrix();
    createHandle();
  }

  void generateNodeList(std::string fileName) { aifmm_dropin::readNodeList(fileName, nodeList); }
  void generatePatchList(std::string fileName) {
    aifmm_dropin::readPatchList(fileName, nodeList, patchList, conductorIndices);
    numConductors = (int)conductorIndices.size();
  }
  void getSizeOfMatrix() { N = (int)patchList.size(); }
  Node getCentroid(Node& v1, Node& v2, Node& v3) { return (v1 + v2 + v3) / 3.0; }
  // the collocation points (ElectrostaticsMatrix.cpp:82-88)
  void getCentroids(Eigen::MatrixX3d& centroids) {
    centroids.resize((Eigen::Index)patchList.size(), 3);
    for (size_t i = 0; i < patchList.size(); ++i)
      for (int q = 0; q < 3; ++q) centroids((Eigen::Index)i, q) = patchList[i].centroid(q);
  }
  double getAreaOfTriangle(Node& v1, Node& v2, Node& v3) { return 0.5 * (v2 - v1).cross(v3 - v1).norm(); }
  double getLargestEdge(Node& v1, Node& v2, Node& v3) { return aifmm_dropin::largestOfFirstTwoEdges(v1, v2, v3); }

  // C0 times the integral of 1/R over triangle j at the centroid of triangle i
  // (ElectrostaticsMatrix.cpp:293-340), evaluated on the GPU.
  dtype getMatrixEntry(const unsigned i, const unsigned j) override { return kernel::getMatrixEntry(i, j); }

  // dense LU solutions (ElectrostaticsMatrix.cpp:342-364)
  void getchargeDensityUsingLU(Eigen::VectorXd& rhs, Eigen::VectorXd& chargeDensity) {
    Eigen::MatrixXd r(rhs.size(), 1), x;
    for (Eigen::Index i = 0; i < rhs.size(); ++i) r(i, 0) = rhs(i);
    getchargeDensityUsingLU(r, x);
    chargeDensity.resize(x.rows());
    for (Eigen::Index i = 0; i < x.rows(); ++i) chargeDensity(i) = x(i, 0);
  }
  void getchargeDensityUsingLU(Eigen::MatrixXd& rhs, Eigen::MatrixXd& chargeDensity) {
    if (rhs.rows() != N) throw std::runtime_error("aifmm: right-hand side length differs from N");
    std::vector<int> ids((size_t)N);
    for (int i = 0; i < N; ++i) ids[(size_t)i] = i;
    const int nrhs = (int)rhs.cols();
    std::vector<std::complex<double>> Z((size_t)N * N), b = aifmm_dropin::to_c128(rhs), x((size_t)N * nrhs);
    aifmm_dropin::check(aifmm_kernel_matrix(handle, ids.data(), N, ids.data(), N, 0, Z.data(), N));
    aifmm_dropin::check(aifmm_lu_solve(aifmm_dropin::context(), reinterpret_cast<double*>(Z.data()), N,
                                       reinterpret_cast<double*>(b.data()), nrhs,
                                       reinterpret_cast<double*>(x.data())));
    aifmm_dropin::from_c128(x.data(), N, nrhs, chargeDensity);
  }
  // total charge = sum of density x area (ElectrostaticsMatrix.cpp:366-372)
  double getCapacitance(Eigen::VectorXd& chargeDensity) {
    if (chargeDensity.size() != N) throw std::runtime_error("aifmm: charge density length differs from N");
    double q = 0.0;
    for (int i = 0; i < N; ++i) q += chargeDensity(i) * patchList[(size_t)i].area;
    return q;
  }
  // 1 V on the triangles of one conductor, 0 elsewhere (:374-381)
  void getRhs(int conductorIndex, Eigen::VectorXd& rhs) {
    rhs = Eigen::VectorXd::Zero(N);
    for (int i = 0; i < N; ++i)
      if (patchList[(size_t)i].conductorIndex == conductorIndex) rhs(i) = 1.0;
  }
  // C(i, j) = charge on conductor i+1 for 1 V on conductor j+1 (:383-402).
  // The reference accumulates into an uninitialised matrix; it starts from 0.
  void getCapacitanceMatrix(Eigen::MatrixXd chargeDensityMatrix, Eigen::MatrixXd& capacitanceMatrix) {
    if (chargeDensityMatrix.rows() != N || chargeDensityMatrix.cols() < numConductors)
      throw std::runtime_error("aifmm: charge densities must be N x (number of conductors)");
    capacitanceMatrix = Eigen::MatrixXd::Zero(numConductors, numConductors);
    for (int j = 0; j < numConductors; ++j)
      for (int k = 0; k < N; ++k) {
        const int ci = patchList[(size_t)k].conductorIndex - 1;
        if (ci >= 0 && ci < numConductors) capacitanceMatrix(ci, j) += chargeDensityMatrix(k, j) * patchList[(size_t)k].area;
      }
  }

  void viewNodeList() {
    std::cout << "nodeList-------------------------" << std::endl;
    for (const Node& v : nodeList) std::cout << v(0) << " " << v(1) << " " << v(2) << std::endl;
  }
  void viewPatchList() {
    std::cout << "patchList-------------------------" << std::endl;
    for (const Patch& p : patchList)
      std::cout << p.indexOfVertex1 << " " << p.indexOfVertex2 << " " << p.indexOfVertex3 << std::endl;
  }

 private:
  void createHandle() {
    std::vector<double> xyz;
    std::vector<int> tris, cond;
    aifmm_dropin::flatten(nodeList, patchList, xyz, tris, cond);
    aifmm_kernel* k = nullptr;
    aifmm_dropin::check(aifmm_kernel_create_es(aifmm_dropin::context(), xyz.data(), (int)(xyz.size() / 3),
                                               tris.data(), cond.data(), (int)patchList.size(), &k));
    owner_.reset(k, [](aifmm_kernel* p) { aifmm_kernel_destroy(p); });
    handle = k;
  }
  std::shared_ptr<aifmm_kernel> owner_;
};

#endif
