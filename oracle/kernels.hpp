// CPU oracle -- TEST INFRASTRUCTURE ONLY.
//
// Restatement of the matrix-entry ("kernel") layer of vaishna77/RCS:
//   include/includes.hpp:53-63, src/includes.cpp:8-59   (constants, Green's functions)
//   include/kernel.hpp:13-47, src/kernel.cpp:11-82       (abstract kernel + gathers)
//   src/EFIEMatrix.cpp:5-20,31-44,72-95,129-209,247-783, 785-837 (EFIE/RWG)
//   src/ElectrostaticsMatrix.cpp:48-52,60-72,100-123,140-340,374-381 (collocation)
// Differences from the reference, by design: the frequency is a runtime value
// (the reference hard-codes freq=1e7 at includes.hpp:58); the reference value is
// the default.  In "exact lookup" mode the O(N) std::next walk over the edge map
// of EFIEMatrix.cpp:700-701 is kept for timing fidelity; otherwise an O(1) table
// with identical arithmetic is used.
#pragma once
#include <array>
#include <map>
#include <set>
#include <utility>
#include <vector>

#include "linalg.hpp"

namespace orc {

struct V3 {
  double x[3];
  V3() : x{0.0, 0.0, 0.0} {}
  V3(double a, double b, double c) : x{a, b, c} {}
  double& operator[](int i) { return x[i]; }
  double operator[](int i) const { return x[i]; }
};
inline V3 operator+(const V3& a, const V3& b) { return V3(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
inline V3 operator-(const V3& a, const V3& b) { return V3(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
inline V3 operator*(const V3& a, double s) { return V3(a[0] * s, a[1] * s, a[2] * s); }
inline V3 operator*(double s, const V3& a) { return V3(s * a[0], s * a[1], s * a[2]); }
inline V3 operator/(const V3& a, double s) { return V3(a[0] / s, a[1] / s, a[2] / s); }
inline double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline double norm(const V3& a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
inline V3 cross(const V3& a, const V3& b) {
  return V3(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
inline double dist(const V3& a, const V3& b) { return norm(a - b); }

struct C3 {
  cd x[3];
  C3() : x{cd(0, 0), cd(0, 0), cd(0, 0)} {}
  C3(cd a, cd b, cd c) : x{a, b, c} {}
};
inline C3 operator+(const C3& a, const C3& b) { return C3(a.x[0] + b.x[0], a.x[1] + b.x[1], a.x[2] + b.x[2]); }
inline C3 operator+(const C3& a, const V3& b) { return C3(a.x[0] + b[0], a.x[1] + b[1], a.x[2] + b[2]); }
inline C3 operator*(double s, const C3& a) { return C3(s * a.x[0], s * a.x[1], s * a.x[2]); }
inline C3 operator*(const V3& a, cd s) { return C3(a[0] * s, a[1] * s, a[2] * s); }
inline C3 operator/(const C3& a, double s) { return C3(a.x[0] / s, a.x[1] / s, a.x[2] / s); }

// Physical constants of include/includes.hpp:53-63 with a runtime frequency.
struct Phys {
  double epsilon = 8.854187817e-12;
  cd I = cd(0.0, 1.0);
  double PI = 4.0 * std::atan(1.0);
  double c = 3.0e8;
  double freq = 1.0e7;
  double lambda, kappa, C0, mu;
  explicit Phys(double f = 1.0e7) : freq(f) {
    lambda = c / freq;
    kappa = 2 * PI / lambda;
    C0 = 1.0 / (4 * PI * epsilon);
    mu = 4 * PI * 1e-7;
  }
};

struct Patch {
  int v1, v2, v3, cond;
  V3 centroid;
  double area, largestEdge;
};

// Abstract kernel: src/kernel.cpp:11-82.
struct Kernel {
  int N = 0;
  virtual ~Kernel() {}
  virtual cd entry(unsigned i, unsigned j) const = 0;
  Mat getMatrix(const std::vector<int>& rows, const std::vector<int>& cols) const;
  Mat getRow(int i, const std::vector<int>& cols) const;  // column vector, as Vec
  Mat getCol(int j, const std::vector<int>& rows) const;
  virtual void locations(std::vector<V3>& out) const = 0;
};

// Triangle mesh shared by both kernels: nodeList with the dummy node 0
// (EFIEMatrix.cpp:31-44) and patchList with area / centroid / largestEdge
// (EFIEMatrix.cpp:72-95; largestEdge only looks at the first two edges,
// EFIEMatrix.cpp:247-254).
struct Mesh {
  std::vector<V3> nodes;
  std::vector<Patch> patches;
  void build(const double* xyz, int nv, const int* tris, int nt, const int* cond);
};

class EFIE : public Kernel {
 public:
  Phys ph;
  Mesh mesh;
  bool exactLookup = false;
  // false (default) = the reference's projection onto the plane through the
  // origin; true = projection onto the source triangle's own plane (used by
  // the physics pins only, to separate that quirk from the rest).
  bool planeProjection = false;
  int etaAnalInteg = 4;
  struct EdgeProps {
    double length;
    std::vector<int> patches;
  };
  std::map<std::pair<int, int>, EdgeProps> edgeMap;
  // flat copies, index = RWG unknown
  std::vector<std::pair<int, int>> eNodes;
  std::vector<double> eLen;
  std::vector<int> ePlus, eMinus;

  EFIE(const double* xyz, int nv, const int* tris, int nt, double freq, bool exact);
  cd entry(unsigned i, unsigned j) const override;
  void locations(std::vector<V3>& out) const override;  // RWG-edge midpoints, sphere.cpp:143-152
  cd rhsReference(const V3& Einc, int i) const;           // EFIEMatrix.cpp:792-829 (quirk kept)
  cd rhsPlaneWave(const V3& khat, const C3& E0, int i) const;  // physically correct plane wave

  // pieces (public for tests)
  int thirdNode(int tri, int a, int b) const;
  cd phiIntegration(int t, int s, int s3) const;
  cd aIntegration(int t, int s, int t3, int s3) const;
  cd scalarGreen(const V3& c, int s, int s3) const;
  C3 vectorGreen(const V3& c, int s, int s3) const;
  V3 vectorSingular(const V3& c, int s, int s3) const;
  C3 vectorNonSingular(const V3& c, int s, int s3) const;
  double analyticLaplace(const V3& c, int s, int s3) const;
  V3 analyticRhoLaplace(const V3& c, int s, int s3) const;
  V3 projection(const V3& c, int s) const;

 private:
  void edgeOf(unsigned i, std::pair<int, int>& nodes, double& len, int& tp, int& tm) const;
};

class Electrostatics : public Kernel {
 public:
  Phys ph;
  Mesh mesh;
  Electrostatics(const double* xyz, int nv, const int* tris, int nt, const int* cond);
  cd entry(unsigned i, unsigned j) const override;
  double entryReal(unsigned i, unsigned j) const;
  void locations(std::vector<V3>& out) const override;  // centroids, ElectrostaticsMatrix.cpp:82-88
  double analytic(const V3& c, const V3& v1, const V3& v2, const V3& v3) const;
};

}  // namespace orc
