// Drop-in replacement for the reference's include/Patch.hpp: one triangle of a
// surface mesh (include/Patch.hpp:6-13, src/Patch.cpp).
#ifndef AIFMM_DROPIN_PATCH_HPP
#define AIFMM_DROPIN_PATCH_HPP

#include "includes.hpp"

class Patch {
 public:
  int indexOfVertex1, indexOfVertex2, indexOfVertex3, conductorIndex = 1;
  Node centroid;
  double area = 0.0;
  double largestEdge = 0.0;
  Patch(int indexOfVertex1, int indexOfVertex2, int indexOfVertex3)
      : indexOfVertex1(indexOfVertex1), indexOfVertex2(indexOfVertex2), indexOfVertex3(indexOfVertex3) {}
};

namespace aifmm_dropin {

// The reference's mesh readers and triangle helpers (EFIEMatrix.cpp:31-95,
// :247-268; ElectrostaticsMatrix.cpp has the same), shared by both kernels.
// Node files: "x y z" per line; node ids are 1-based, so a zero node is put
// first.  Patch files: "i1 i2 i3 [conductor]"; a missing conductor column
// reads as conductor 1 (the reference reads an uninitialised value there).
inline void readNodeList(const std::string& fileName, std::vector<Node>& nodeList) {
  std::ifstream file(fileName);
  if (!file) throw std::runtime_error("aifmm: cannot open node list " + fileName);
  nodeList.push_back(Node::Zero(3));
  std::string line;
  while (std::getline(file, line)) {
    std::stringstream ls(line);
    Node node;
    if (!(ls >> node[0] >> node[1] >> node[2])) continue;  // blank or short line
    nodeList.push_back(node);
  }
}

inline double largestOfFirstTwoEdges(const Node& v1, const Node& v2, const Node& v3) {
  // getLargestEdge looks at the first two of the three edges only (:247-254)
  const double e1 = (v1 - v2).norm(), e2 = (v2 - v3).norm();
  return e2 > e1 ? e2 : e1;
}

inline void readPatchList(const std::string& fileName, const std::vector<Node>& nodeList,
                          std::vector<Patch>& patchList, std::set<int>& conductorIndices) {
  std::ifstream file(fileName);
  if (!file) throw std::runtime_error("aifmm: cannot open patch list " + fileName);
  std::string line;
  while (std::getline(file, line)) {
    std::stringstream ls(line);
    int i1, i2, i3, cond = 1;
    if (!(ls >> i1 >> i2 >> i3)) continue;
    if (!(ls >> cond)) cond = 1;
    const int nv = (int)nodeList.size();
    if (i1 < 1 || i2 < 1 || i3 < 1 || i1 >= nv || i2 >= nv || i3 >= nv)
      throw std::runtime_error("aifmm: patch refers to a node that is not in the node list");
    Patch p(i1, i2, i3);
    const Node &a = nodeList[i1], &b = nodeList[i2], &c3 = nodeList[i3];
    p.area = 0.5 * (b - a).cross(c3 - a).norm();
    p.centroid = (a + b + c3) / 3.0;
    p.largestEdge = largestOfFirstTwoEdges(a, b, c3);
    p.conductorIndex = cond;
    conductorIndices.insert(cond);
    patchList.push_back(p);
  }
}

// Flat arrays for the C ABI: nodes without the zero node, 1-based triangles.
inline void flatten(const std::vector<Node>& nodeList, const std::vector<Patch>& patchList,
                    std::vector<double>& xyz, std::vector<int>& tris, std::vector<int>& cond) {
  xyz.clear();
  tris.clear();
  cond.clear();
  for (size_t i = 1; i < nodeList.size(); ++i)
    for (int q = 0; q < 3; ++q) xyz.push_back(nodeList[i](q));
  for (const Patch& p : patchList) {
    tris.push_back(p.indexOfVertex1);
    tris.push_back(p.indexOfVertex2);
    tris.push_back(p.indexOfVertex3);
    cond.push_back(p.conductorIndex);
  }
}

}  // namespace aifmm_dropin

#endif
