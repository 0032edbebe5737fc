// Drop-in replacement for the reference's include/EFIEMatrix.hpp: the EFIE
// method-of-moments kernel with RWG basis functions on a triangle mesh
// (include/EFIEMatrix.hpp:8-118, src/EFIEMatrix.cpp).
//
// The mesh readers, the edge -> patch map and the RWG numbering run on the
// host exactly as the reference's (the public members a driver reads are
// filled the same way); every matrix entry, right-hand side, dense solve,
// centroid current and RCS value is computed by libaifmm_b200 on the GPU.
// The quadrature helpers that the reference exposes as public members
// (onePointGaussQuadratureRule, analyticIntegration*, get*Integration*) are
// internals of getMatrixEntry and are not provided; neither are the plate-mesh
// constructors and the seven-point RCS variants.
#ifndef AIFMM_DROPIN_EFIEMATRIX_HPP
#define AIFMM_DROPIN_EFIEMATRIX_HPP

#include <algorithm>
#include <memory>

#include "Patch.hpp"
#include "includes.hpp"
#include "kernel.hpp"

class Edge {
 public:
  std::pair<int, int> indicesOfNodes;
  double length;
  std::vector<int> indicesOfAssociatedPatches;
};

struct compare {
  bool operator()(const Edge& e1, const Edge& e2) const { return e1.indicesOfNodes.first < e2.indicesOfNodes.first; }
};

struct edgeProperties {
  double length;
  std::vector<int> indicesOfAssociatedPatches;
};

class EFIEMatrix : public kernel {
 public:
  std::vector<Node> nodeList;
  std::vector<Patch> patchList;
  std::map<int, Eigen::MatrixXd> M2L;
  std::set<int> conductorIndices;
  int numConductors = 0;
  std::set<Edge, compare> edgeList;
  std::map<std::pair<int, int>, edgeProperties> edge2PatchMap;
  int n = 0;
  double L = 0.0;
  std::multimap<std::pair<int, int>, std::complex<double>> lookUpTable[9];  // plate meshes only; stays empty
  double getMatrixEntryFromScratchTime = 0;
  double getMatrixEntryTime = 0;
  int ngetMatrixEntryFromScratch = 0;
  int ngetMatrixEntry = 0;
  int etaAnalInteg = 4;
  int N = 0;

  // EFIEMatrix(inputsToKernelClass) (EFIEMatrix.cpp:5-20)
  explicit EFIEMatrix(inputsToKernelClass inputsToKernel) {
#if defined(USE_DOUBLE)
    throw std::runtime_error("aifmm: EFIEMatrix needs complex entries (build with USE_COMPLEX64)");
#endif
    n = inputsToKernel.n;
    L = inputsToKernel.L;
    generateNodeList(inputsToKernel.nodeListFilename);
    generatePatchList(inputsToKernel.patchListFilename);
    generateEdgeList();
    deleteNonRWGEdges();
    getSizeOfMatrix();
    createHandle();
  }

  void generateNodeList(std::string fileName) { aifmm_dropin::readNodeList(fileName, nodeList); }
  void generatePatchList(std::string fileName) {
    aifmm_dropin::readPatchList(fileName, nodeList, patchList, conductorIndices);
    numConductors = (int)conductorIndices.size();
  }
  // edge -> patch map keyed by (min node, max node), patches in file order
  // (EFIEMatrix.cpp:129-197)
  void generateEdgeList() {
    for (size_t i = 0; i < patchList.size(); ++i) {
      const int v[3] = {patchList[i].indexOfVertex1, patchList[i].indexOfVertex2, patchList[i].indexOfVertex3};
      for (int e = 0; e < 3; ++e) {
        const int va = v[e], vb = v[(e + 1) % 3];
        Edge edge;
        edge.indicesOfNodes = va < vb ? std::make_pair(va, vb) : std::make_pair(vb, va);
        edge.length = (nodeList[va] - nodeList[vb]).norm();
        edgeList.insert(edge);
        auto it = edge2PatchMap.find(edge.indicesOfNodes);
        if (it == edge2PatchMap.end()) {
          edgeProperties p;
          p.length = edge.length;
          p.indicesOfAssociatedPatches.push_back((int)i);
          edge2PatchMap[edge.indicesOfNodes] = p;
        } else {
          it->second.indicesOfAssociatedPatches.push_back((int)i);
        }
      }
    }
  }
  // boundary edges (one patch) carry no RWG function (EFIEMatrix.cpp:199-209)
  void deleteNonRWGEdges() {
    for (auto it = edge2PatchMap.begin(); it != edge2PatchMap.end();) {
      if (it->second.indicesOfAssociatedPatches.size() == 1) it = edge2PatchMap.erase(it);
      else ++it;
    }
  }
  void getSizeOfMatrix() { N = (int)edge2PatchMap.size(); }
  Node getCentroid(Node& v1, Node& v2, Node& v3) { return (v1 + v2 + v3) / 3.0; }
  double getAreaOfTriangle(Node& v1, Node& v2, Node& v3) { return 0.5 * (v2 - v1).cross(v3 - v1).norm(); }
  double getLargestEdge(Node& v1, Node& v2, Node& v3) { return aifmm_dropin::largestOfFirstTwoEdges(v1, v2, v3); }
  // the vertex of a triangle that is not on the edge (EFIEMatrix.cpp:353-373)
  int getIndexOfThirdNode(int indexOfTriangle, int node1, int node2) {
    const Patch& p = patchList[indexOfTriangle];
    for (int v : {p.indexOfVertex1, p.indexOfVertex2, p.indexOfVertex3})
      if (v != node1 && v != node2) return v;
    return p.indexOfVertex1;
  }

  // Z(i, j) (EFIEMatrix.cpp:698-783), evaluated on the GPU.
  dtype getMatrixEntry(const unsigned i, const unsigned j) override {
    ++ngetMatrixEntry;
    return kernel::getMatrixEntry(i, j);
  }
  cdouble getMatrixEntryFromScratch(const unsigned i, const unsigned j) {
    ++ngetMatrixEntryFromScratch;
    return cdouble(kernel::getMatrixEntry(i, j));
  }
  // plate meshes only in the reference; nothing to tabulate for a general mesh
  void createLookUpTable() {}

  // right-hand side of the incident field Einc (EFIEMatrix.cpp:785-829),
  // with the reference's phase convention
  void getRhs(Node& Einc, Eigen::VectorXcd& rhs) {
    const double e[3] = {Einc(0), Einc(1), Einc(2)};
    std::vector<std::complex<double>> b((size_t)N);
    aifmm_dropin::check(aifmm_kernel_rhs_reference(handle, e, reinterpret_cast<double*>(b.data())));
    aifmm_dropin::from_c128(b.data(), N, 1, rhs);
  }
  cdouble getRhs(Node& Einc, int i) {
    Eigen::VectorXcd rhs;
    getRhs(Einc, rhs);
    return rhs(i);
  }
  // dense LU solution (EFIEMatrix.cpp:831-837): the whole matrix is assembled
  // and factorized on the GPU
  void getCoefficients(Eigen::VectorXcd& rhs, Eigen::VectorXcd& coefficients) {
    if (rhs.size() != N) throw std::runtime_error("aifmm: right-hand side length differs from N");
    std::vector<int> ids((size_t)N);
    for (int i = 0; i < N; ++i) ids[(size_t)i] = i;
    std::vector<std::complex<double>> Z((size_t)N * N), b = aifmm_dropin::to_c128(rhs), x((size_t)N);
    aifmm_dropin::check(aifmm_kernel_matrix(handle, ids.data(), N, ids.data(), N, 0, Z.data(), N));
    aifmm_dropin::check(aifmm_lu_solve(aifmm_dropin::context(), reinterpret_cast<double*>(Z.data()), N,
                                       reinterpret_cast<double*>(b.data()), 1, reinterpret_cast<double*>(x.data())));
    aifmm_dropin::from_c128(x.data(), N, 1, coefficients);
  }
  // current at the triangle centroids (EFIEMatrix.cpp:1100-1130)
  void getJAtCentroids(Eigen::VectorXcd& coefficients, Eigen::MatrixXcd& JAtCentroids) {
    if (coefficients.size() != N) throw std::runtime_error("aifmm: coefficient vector length differs from N");
    std::vector<std::complex<double>> cvec = aifmm_dropin::to_c128(coefficients);
    std::vector<std::complex<double>> J(patchList.size() * 3);
    aifmm_dropin::check(aifmm_kernel_currents(handle, reinterpret_cast<double*>(cvec.data()),
                                              reinterpret_cast<double*>(J.data())));
    aifmm_dropin::from_c128(J.data(), (Eigen::Index)patchList.size(), 3, JAtCentroids);
  }
  // bistatic RCS at (theta, phi) from centroid currents (EFIEMatrix.cpp:916-930)
  double getRCS_OnePointQuadrature(double theta, double phi, Eigen::MatrixXcd& JAtCentroids) {
    double out = 0.0;
    getRCS_OnePointQuadrature(1, &theta, &phi, JAtCentroids, &out);
    return out;
  }
  // Extension: many observation angles in one launch.
  void getRCS_OnePointQuadrature(int nAngles, const double* theta, const double* phi, Eigen::MatrixXcd& JAtCentroids,
                                 double* rcs) {
    if (JAtCentroids.rows() != (Eigen::Index)patchList.size() || JAtCentroids.cols() != 3)
      throw std::runtime_error("aifmm: JAtCentroids must be (number of patches) x 3");
    std::vector<std::complex<double>> J = aifmm_dropin::to_c128(JAtCentroids);
    aifmm_dropin::check(aifmm_kernel_rcs(handle, reinterpret_cast<double*>(J.data()), nAngles, theta, phi, rcs));
  }
  // Extension: 1 projects the test point onto the source triangle's own plane
  // instead of the plane through the origin (findProjectionOnTriangle,
  // EFIEMatrix.cpp:457-476); the RCS of a sphere then follows the Mie series.
  void setPlaneProjection(bool on) { aifmm_dropin::check(aifmm_kernel_set_plane_projection(handle, on ? 1 : 0)); }

  void viewNodeList() {
    std::cout << "nodeList-------------------------" << std::endl;
    for (const Node& v : nodeList) std::cout << v(0) << " " << v(1) << " " << v(2) << std::endl;
  }
  void viewPatchList() {
    std::cout << "patchList-------------------------" << std::endl;
    for (const Patch& p : patchList)
      std::cout << p.indexOfVertex1 << " " << p.indexOfVertex2 << " " << p.indexOfVertex3 << std::endl;
  }
  void viewEdgeList() {
    std::cout << "No. of patches: " << patchList.size() << std::endl;
    std::cout << "No. of edges: " << edge2PatchMap.size() << std::endl;
    int rwg = 0;
    for (auto& kv : edge2PatchMap) {
      std::cout << kv.first.first << " " << kv.first.second << " " << std::endl;
      if (kv.second.indicesOfAssociatedPatches.size() == 2) rwg++;
    }
    std::cout << "rwg: " << rwg << std::endl;
  }

 private:
  void createHandle() {
    std::vector<double> xyz;
    std::vector<int> tris, cond;
    aifmm_dropin::flatten(nodeList, patchList, xyz, tris, cond);
    aifmm_kernel* k = nullptr;
    aifmm_dropin::check(aifmm_kernel_create_efie(aifmm_dropin::context(), xyz.data(), (int)(xyz.size() / 3),
                                                 tris.data(), (int)patchList.size(), freq, &k));
    owner_.reset(k, [](aifmm_kernel* p) { aifmm_kernel_destroy(p); });
    handle = k;
    int nk = 0;
    aifmm_dropin::check(aifmm_kernel_size(k, &nk));
    if (nk != N) throw std::runtime_error("aifmm: the library's RWG count differs from the edge map's");
  }
  std::shared_ptr<aifmm_kernel> owner_;
};

#endif
