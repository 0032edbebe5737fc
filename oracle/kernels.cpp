// CPU oracle -- TEST INFRASTRUCTURE ONLY.  See kernels.hpp for the reference
// line ranges restated here.  Expressions keep the reference's evaluation
// order so that the floating-point results match a -ffp-contract=off build of
// the reference to the last bit where the same libm is used.
#include "kernels.hpp"

#include <omp.h>

namespace orc {

// ---------------------------------------------------------------- gathers
// kernel.cpp:49-61 (nested omp; the inner region is serialised in practice).
Mat Kernel::getMatrix(const std::vector<int>& rows, const std::vector<int>& cols) const {
  const int nr = (int)rows.size(), nc = (int)cols.size();
  Mat m(nr, nc);
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nr; ++j)
    for (int k = 0; k < nc; ++k) m(j, k) = entry(rows[j], cols[k]);
  return m;
}
// kernel.cpp:11-19
Mat Kernel::getRow(int i, const std::vector<int>& cols) const {
  const int nc = (int)cols.size();
  Mat v(nc, 1);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nc; ++k) v(k) = entry(i, cols[k]);
  return v;
}
// kernel.cpp:21-29
Mat Kernel::getCol(int j, const std::vector<int>& rows) const {
  const int nr = (int)rows.size();
  Mat v(nr, 1);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nr; ++k) v(k) = entry(rows[k], j);
  return v;
}

// ---------------------------------------------------------------- mesh
static double areaOf(const V3& a, const V3& b, const V3& c) {  // EFIEMatrix.cpp:262-268
  V3 e1 = b - a, e2 = c - a;
  return 0.5 * norm(cross(e1, e2));
}
static V3 centroidOf(const V3& a, const V3& b, const V3& c) { return (a + b + c) / 3.0; }
static double largestEdgeOf(const V3& a, const V3& b, const V3& c) {
  // EFIEMatrix.cpp:247-254: std::max_element over the first TWO edge lengths only.
  double l1 = dist(a, b), l2 = dist(b, c);
  return (l2 > l1) ? l2 : l1;
}

void Mesh::build(const double* xyz, int nv, const int* tris, int nt, const int* cond) {
  nodes.clear();
  patches.clear();
  nodes.push_back(V3(0, 0, 0));  // dummy node 0 (1-based vertex ids)
  for (int i = 0; i < nv; ++i) nodes.push_back(V3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
  for (int t = 0; t < nt; ++t) {
    Patch p;
    p.v1 = tris[3 * t];
    p.v2 = tris[3 * t + 1];
    p.v3 = tris[3 * t + 2];
    for (int q : {p.v1, p.v2, p.v3})
      if (q < 1 || q > nv) fail("triangle vertex id out of range");
    p.cond = cond ? cond[t] : 0;
    const V3 &a = nodes[p.v1], &b = nodes[p.v2], &c = nodes[p.v3];
    p.area = areaOf(a, b, c);
    p.centroid = centroidOf(a, b, c);
    p.largestEdge = largestEdgeOf(a, b, c);
    patches.push_back(p);
  }
}

// 7-point rule of EFIEMatrix.cpp:284-286 (truncated constants kept).
static const double QA[7] = {0.3333333, 0.0597158, 0.470142, 0.470142, 0.7974269, 0.1012865, 0.1012865};
static const double QB[7] = {0.3333333, 0.470142, 0.0597158, 0.470142, 0.1012865, 0.7974269, 0.1012865};
static const double QW[7] = {0.225, 0.13239415278851, 0.13239415278851, 0.13239415278851,
                             0.12593918054483, 0.12593918054483, 0.12593918054483};

// ---------------------------------------------------------------- EFIE
EFIE::EFIE(const double* xyz, int nv, const int* tris, int nt, double freq, bool exact)
    : ph(freq), exactLookup(exact) {
  mesh.build(xyz, nv, tris, nt, nullptr);
  // generateEdgeList, EFIEMatrix.cpp:129-197: edges keyed by (min,max) node id
  // in a std::map; patches appended in file order.
  for (int i = 0; i < nt; ++i) {
    const Patch& p = mesh.patches[i];
    int idx[3] = {p.v1, p.v2, p.v3};
    for (int e = 0; e < 3; ++e) {
      int a = idx[e], b = idx[(e + 1) % 3];
      std::pair<int, int> key = (a < b) ? std::make_pair(a, b) : std::make_pair(b, a);
      auto it = edgeMap.find(key);
      if (it == edgeMap.end()) {
        EdgeProps ep;
        ep.length = dist(mesh.nodes[a], mesh.nodes[b]);
        ep.patches.push_back(i);
        edgeMap[key] = ep;
      } else {
        it->second.patches.push_back(i);
      }
    }
  }
  // deleteNonRWGEdges, EFIEMatrix.cpp:199-209
  for (auto it = edgeMap.begin(); it != edgeMap.end();) {
    if (it->second.patches.size() == 1) it = edgeMap.erase(it);
    else ++it;
  }
  N = (int)edgeMap.size();
  for (auto& kv : edgeMap) {
    eNodes.push_back(kv.first);
    eLen.push_back(kv.second.length);
    ePlus.push_back(kv.second.patches[0]);
    eMinus.push_back(kv.second.patches[1]);
  }
}

void EFIE::edgeOf(unsigned i, std::pair<int, int>& nodes, double& len, int& tp, int& tm) const {
  if (exactLookup) {
    auto it = std::next(edgeMap.begin(), i);  // O(N) walk, EFIEMatrix.cpp:700
    nodes = it->first;
    len = it->second.length;
    tp = it->second.patches[0];
    tm = it->second.patches[1];
  } else {
    nodes = eNodes[i];
    len = eLen[i];
    tp = ePlus[i];
    tm = eMinus[i];
  }
}

// EFIEMatrix.cpp:353-373 (sorted set difference).
int EFIE::thirdNode(int tri, int a, int b) const {
  int t[3] = {mesh.patches[tri].v1, mesh.patches[tri].v2, mesh.patches[tri].v3};
  int e[2] = {a, b};
  std::sort(t, t + 3);
  std::sort(e, e + 2);
  std::vector<int> diff(1);
  std::set_difference(t, t + 3, e, e + 2, diff.begin());
  return diff[0];
}

// findProjectionOnTriangle, EFIEMatrix.cpp:457-476: projects onto the plane
// through the ORIGIN with the triangle's normal (quirk kept).
V3 EFIE::projection(const V3& c, int s) const {
  const Patch& p = mesh.patches[s];
  const V3 &v1 = mesh.nodes[p.v1], &v2 = mesh.nodes[p.v2], &v3 = mesh.nodes[p.v3];
  V3 e2 = v2 - v1, e3 = v3 - v1;
  V3 e1 = c;
  V3 n = cross(e2, e3);
  n = -1.0 * n / norm(n);
  if (planeProjection) {
    double d = dot(c - v1, n);
    return c - d * n;
  }
  double d = dot(e1, n);
  return e1 - d * n;
}

static void freeFirst(const Patch& p, int s3, int& i1, int& i2, int& i3) {
  i1 = s3;
  if (p.v1 == i1) { i2 = p.v2; i3 = p.v3; }
  else if (p.v2 == i1) { i2 = p.v1; i3 = p.v3; }
  else { i2 = p.v1; i3 = p.v2; }
}

// analyticIntegrationLaplaceFunction, EFIEMatrix.cpp:478-577.
double EFIE::analyticLaplace(const V3& c, int s, int s3) const {
  int i1, i2, i3;
  freeFirst(mesh.patches[s], s3, i1, i2, i3);
  const V3 v1 = mesh.nodes[i1], v2 = mesh.nodes[i2], v3 = mesh.nodes[i3];
  V3 e2 = v2 - v1, e3 = v3 - v1, e1 = c - v1;
  V3 n = cross(e2, e3);
  n = -1.0 * n / norm(n);
  double dp = dot(e1, n);
  V3 cop = c - dp * n;
  dp = std::abs(dp);
  V3 origin(0, 0, 0);
  double acc = 0.0;
  for (int i = 0; i < 3; ++i) {
    V3 p1, p2;
    if (i == 0) { p1 = v1; p2 = v2; }
    else if (i == 1) { p1 = v2; p2 = v3; }
    else { p1 = v3; p2 = v1; }
    double lside = dist(p1, p2);
    V3 ctl = p1 - c;
    double Rp = dist(ctl, origin);
    ctl = p2 - c;
    double Rm = dist(ctl, origin);
    V3 Pp = p1 - cop, Pm = p2 - cop;
    double d = dist(p1, p2);
    V3 ul = (p1 - p2) / d;
    double Lp = dot(Pp, ul), Lm = dot(Pm, ul);
    V3 uu = cross(ul, n);
    double P0 = dot(Pp, uu);
    if (P0 < 0) P0 = P0 * -1;
    if (!(P0 < 1.0e-10 * lside)) {
      double R0 = std::sqrt((P0 * P0) + (dp * dp));
      V3 up = Pp - Lp * ul;
      d = dist(up, origin);
      up = up / d;
      double T1 = P0 * std::log((Rp + Lp) / (Rm + Lm));
      if (P0 < 1e-6 * lside) {
        if (R0 < 1e-4 * lside) T1 = 0;
      }
      double T2 = std::atan(P0 * Lp / (R0 * R0 + dp * Rp));
      double T3 = std::atan(P0 * Lm / (R0 * R0 + dp * Rm));
      double T4 = dot(up, uu);
      acc = acc + (T4 * (T1 - dp * (T2 - T3)));
    }
  }
  return acc;
}

// analyticIntegrationRhoLaplaceFunction, EFIEMatrix.cpp:579-668.
V3 EFIE::analyticRhoLaplace(const V3& c, int s, int s3) const {
  int i1, i2, i3;
  freeFirst(mesh.patches[s], s3, i1, i2, i3);
  const V3 v1 = mesh.nodes[i1], v2 = mesh.nodes[i2], v3 = mesh.nodes[i3];
  V3 e2 = v2 - v1, e3 = v3 - v1, e1 = c - v1;
  V3 n = cross(e2, e3);
  n = -1.0 * n / norm(n);
  double dp = dot(e1, n);
  V3 cop = c - dp * n;
  dp = std::abs(dp);
  V3 origin(0, 0, 0);
  V3 acc(0, 0, 0);
  for (int i = 0; i < 3; ++i) {
    V3 p1, p2;
    if (i == 0) { p1 = v1; p2 = v2; }
    else if (i == 1) { p1 = v2; p2 = v3; }
    else { p1 = v3; p2 = v1; }
    V3 ctl = p1 - c;
    double Rp = dist(ctl, origin);
    ctl = p2 - c;
    double Rm = dist(ctl, origin);
    V3 Pp = p1 - cop, Pm = p2 - cop;
    double d = dist(p1, p2);
    V3 ul = (p1 - p2) / d;
    double Lp = dot(Pp, ul), Lm = dot(Pm, ul);
    V3 uu = cross(ul, n);
    double P0 = dot(Pp, uu);
    if (P0 < 0) P0 = P0 * -1;
    double sqR0 = (P0 * P0) + (dp * dp);
    double T1;
    if ((Rm + Lm) >= 1.0e-10) T1 = sqR0 * std::log((Rp + Lp) / (Rm + Lm));
    else T1 = 0;
    double T2 = (Lp * Rp) - (Lm * Rm);
    acc = acc + (uu * 0.5 * (T1 + T2));
  }
  return acc;
}

// getScalarIntegrationGreensFunction, EFIEMatrix.cpp:670-685, with the
// quadrature rules of EFIEMatrix.cpp:270-310 and Green's functions of
// includes.cpp:13-21.
cd EFIE::scalarGreen(const V3& c, int s, int s3) const {
  const Patch& p = mesh.patches[s];
  const double PI = ph.PI, kappa = ph.kappa;
  const cd I = ph.I;
  double dcc = dist(c, p.centroid);
  auto G = [&](const V3& ri, const V3& rj) {
    double d = dist(ri, rj);
    return (-1.0 / 4.0 / PI) * std::exp(-I * kappa * d) / d;
  };
  auto Gns = [&](const V3& ri, const V3& rj) {
    double d = dist(ri, rj);
    return (-1.0 / 4.0 / PI) * (std::exp(-I * kappa * d) - 1.0) / d;
  };
  const V3 &a = mesh.nodes[p.v1], &b = mesh.nodes[p.v2], &cc = mesh.nodes[p.v3];
  if (dcc < etaAnalInteg * p.largestEdge) {
    cd sum = 0.0;
    for (int i = 0; i < 7; ++i) {
      V3 pt = a + (b - a) * QA[i] + (cc - a) * QB[i];
      if (dist(pt, c) < 1e-12) sum += QW[i] * (I * kappa) / 4.0 / PI;
      else sum += QW[i] * Gns(c, pt);
    }
    return (-1.0 / 4.0 / PI) * analyticLaplace(c, s, s3) + p.area * sum;
  } else if ((dcc >= etaAnalInteg * p.largestEdge) && (dcc < 10.0 * p.largestEdge)) {
    cd sum = 0.0;
    for (int i = 0; i < 7; ++i) {
      V3 pt = a + (b - a) * QA[i] + (cc - a) * QB[i];
      sum += QW[i] * G(c, pt);
    }
    return p.area * sum;
  } else {
    return p.area * G(c, p.centroid);
  }
}

// getVectorIntegrationSingularPart, EFIEMatrix.cpp:386-405.
V3 EFIE::vectorSingular(const V3& c, int s, int s3) const {
  const Patch& p = mesh.patches[s];
  const double PI = ph.PI;
  double dcc = dist(c, p.centroid);
  const V3& n3 = mesh.nodes[s3];
  auto rhoLap = [&](const V3& ri, const V3& rj) {
    double d = dist(ri, rj);
    V3 rho = rj - n3;
    return rho * (-1.0 / 4.0 / PI) / d;
  };
  if (dcc < etaAnalInteg * p.largestEdge) {
    V3 proj = projection(c, s);
    V3 A = analyticRhoLaplace(c, s, s3);
    double L = analyticLaplace(c, s, s3);
    V3 B = proj - n3;
    V3 r;
    for (int q = 0; q < 3; ++q) r[q] = (-1.0 / 4.0 / PI) * (A[q] + L * B[q]);
    return r;
  } else if ((dcc >= etaAnalInteg * p.largestEdge) && (dcc < 10.0 * p.largestEdge)) {
    // sevenPointGaussQuadratureRuleReal: vertices taken as (v2, v3, v1).
    const V3 &a = mesh.nodes[p.v2], &b = mesh.nodes[p.v3], &cc = mesh.nodes[p.v1];
    V3 sum(0, 0, 0);
    for (int i = 0; i < 7; ++i) {
      V3 pt = a + (b - a) * QA[i] + (cc - a) * QB[i];
      sum = sum + QW[i] * rhoLap(c, pt);
    }
    return p.area * sum;
  } else {
    return p.area * rhoLap(c, p.centroid);
  }
}

// getVectorIntegrationNonSingularPart, EFIEMatrix.cpp:407-424: always 7-point
// (sevenPointGaussQuadratureRuleComplex, vertices (v2,v3,v1)) of
// rhoNonSingularGreensFunction (includes.cpp:36-51).
C3 EFIE::vectorNonSingular(const V3& c, int s, int s3) const {
  const Patch& p = mesh.patches[s];
  const double PI = ph.PI, kappa = ph.kappa;
  const cd I = ph.I;
  const V3& n3 = mesh.nodes[s3];
  const V3 &a = mesh.nodes[p.v2], &b = mesh.nodes[p.v3], &cc = mesh.nodes[p.v1];
  C3 sum;
  for (int i = 0; i < 7; ++i) {
    V3 pt = a + (b - a) * QA[i] + (cc - a) * QB[i];
    double d = dist(c, pt);
    V3 rho = pt - n3;
    C3 val;
    if (d < 1e-12) {
      val = (rho * (-1.0 / 4.0 / PI)) * (-I * kappa);
    } else {
      cd g = (std::exp(-I * kappa * d) - 1.0);
      V3 rs = rho * (-1.0 / 4.0 / PI);
      val = C3(rs[0] * g / d, rs[1] * g / d, rs[2] * g / d);
    }
    sum = sum + QW[i] * val;
  }
  return p.area * sum;
}

C3 EFIE::vectorGreen(const V3& c, int s, int s3) const {  // EFIEMatrix.cpp:436-446
  return vectorNonSingular(c, s, s3) + vectorSingular(c, s, s3);
}

cd EFIE::phiIntegration(int t, int s, int s3) const {  // EFIEMatrix.cpp:448-455
  return mesh.patches[t].area * scalarGreen(mesh.patches[t].centroid, s, s3);
}

cd EFIE::aIntegration(int t, int s, int t3, int s3) const {  // EFIEMatrix.cpp:375-384
  V3 rc = mesh.patches[t].centroid - mesh.nodes[t3];
  V3 ar = mesh.patches[t].area * rc;
  C3 v = vectorGreen(mesh.patches[t].centroid, s, s3);
  return ar[0] * v.x[0] + ar[1] * v.x[1] + ar[2] * v.x[2];
}

// getMatrixEntry, EFIEMatrix.cpp:698-783.
cd EFIE::entry(unsigned i, unsigned j) const {
  const double PI = ph.PI, freq = ph.freq, epsilon = ph.epsilon, mu = ph.mu;
  const cd I = ph.I;
  std::pair<int, int> te, se;
  double Lt, Ls;
  int tp, tm, sp, sm;
  edgeOf(i, te, Lt, tp, tm);
  edgeOf(j, se, Ls, sp, sm);
  int tp3 = thirdNode(tp, te.first, te.second);
  int tm3 = thirdNode(tm, te.first, te.second);
  int sp3 = thirdNode(sp, se.first, se.second);
  int sm3 = thirdNode(sm, se.first, se.second);
  const auto& P = mesh.patches;
  cd phiPP = -Lt * Ls / (I * 2.0 * PI * freq * epsilon * P[tp].area * P[sp].area);
  cd phiPM = Lt * Ls / (I * 2.0 * PI * freq * epsilon * P[tp].area * P[sm].area);
  cd phiMP = Lt * Ls / (I * 2.0 * PI * freq * epsilon * P[tm].area * P[sp].area);
  cd phiMM = -Lt * Ls / (I * 2.0 * PI * freq * epsilon * P[tm].area * P[sm].area);
  cd ePP = phiPP * phiIntegration(tp, sp, sp3);
  cd ePM = phiPM * phiIntegration(tp, sm, sm3);
  cd eMP = phiMP * phiIntegration(tm, sp, sp3);
  cd eMM = phiMM * phiIntegration(tm, sm, sm3);
  cd aPP = -(I * 2.0 * PI * freq * mu * Lt * Ls) / (4.0 * P[tp].area * P[sp].area);
  cd aPM = (I * 2.0 * PI * freq * mu * Lt * Ls) / (4.0 * P[tp].area * P[sm].area);
  cd aMP = (I * 2.0 * PI * freq * mu * Lt * Ls) / (4.0 * P[tm].area * P[sp].area);
  cd aMM = -(I * 2.0 * PI * freq * mu * Lt * Ls) / (4.0 * P[tm].area * P[sm].area);
  cd fPP = aPP * aIntegration(tp, sp, tp3, sp3);
  cd fPM = aPM * aIntegration(tp, sm, tp3, sm3);
  cd fMP = aMP * aIntegration(tm, sp, tm3, sp3);
  cd fMM = aMM * aIntegration(tm, sm, tm3, sm3);
  cd z = ePP + ePM + eMP + eMM;
  z += fPP + fPM + fMP + fMM;
  return z;
}

void EFIE::locations(std::vector<V3>& out) const {
  out.resize(N);
  for (int i = 0; i < N; ++i) {
    std::pair<int, int> e;
    double L;
    int tp, tm;
    edgeOf(i, e, L, tp, tm);
    out[i] = (mesh.nodes[e.first] + mesh.nodes[e.second]) / 2.0;
  }
}

// getRhs, EFIEMatrix.cpp:792-829.  Quirk kept: theta=phi=0 and the phase
// vector's z component is cos(theta) (no kappa), so the phase is exp(i z).
cd EFIE::rhsReference(const V3& Einc, int i) const {
  const cd I = ph.I;
  std::pair<int, int> te;
  double Lt;
  int tp, tm;
  edgeOf(i, te, Lt, tp, tm);
  int tp3 = thirdNode(tp, te.first, te.second);
  int tm3 = thirdNode(tm, te.first, te.second);
  const auto& P = mesh.patches;
  V3 rp = P[tp].centroid - mesh.nodes[tp3];
  V3 rm = P[tm].centroid - mesh.nodes[tm3];
  double theta = 0.0, phi = 0.0;
  V3 kv(ph.kappa * std::sin(theta) * std::cos(phi), ph.kappa * std::sin(theta) * std::sin(phi), std::cos(theta));
  double kp = dot(kv, P[tp].centroid);
  double km = dot(kv, P[tm].centroid);
  cd ep = std::exp(I * kp), em = std::exp(I * km);
  cd dp = (Einc[0] * ep) * rp[0] + (Einc[1] * ep) * rp[1] + (Einc[2] * ep) * rp[2];
  cd dm = (Einc[0] * em) * rm[0] + (Einc[1] * em) * rm[1] + (Einc[2] * em) * rm[2];
  return Lt / 2.0 * (dp - dm);
}

// A physically correct plane wave E0 exp(-i kappa khat.r) sampled like the
// reference (centroid rule): khat is the propagation direction.
cd EFIE::rhsPlaneWave(const V3& khat, const C3& E0, int i) const {
  const cd I = ph.I;
  std::pair<int, int> te;
  double Lt;
  int tp, tm;
  edgeOf(i, te, Lt, tp, tm);
  int tp3 = thirdNode(tp, te.first, te.second);
  int tm3 = thirdNode(tm, te.first, te.second);
  const auto& P = mesh.patches;
  V3 rp = P[tp].centroid - mesh.nodes[tp3];
  V3 rm = P[tm].centroid - mesh.nodes[tm3];
  cd ep = std::exp(-I * ph.kappa * dot(khat, P[tp].centroid));
  cd em = std::exp(-I * ph.kappa * dot(khat, P[tm].centroid));
  cd dp = (E0.x[0] * rp[0] + E0.x[1] * rp[1] + E0.x[2] * rp[2]) * ep;
  cd dm = (E0.x[0] * rm[0] + E0.x[1] * rm[1] + E0.x[2] * rm[2]) * em;
  return Lt / 2.0 * (dp - dm);
}

// ---------------------------------------------------------------- ES
Electrostatics::Electrostatics(const double* xyz, int nv, const int* tris, int nt, const int* cond) {
  mesh.build(xyz, nv, tris, nt, cond);
  N = (int)mesh.patches.size();
}

// analyticIntegration, ElectrostaticsMatrix.cpp:179-281.
double Electrostatics::analytic(const V3& c, const V3& v1, const V3& v2, const V3& v3) const {
  V3 e2 = v2 - v1, e3 = v3 - v1, e1 = c - v1;
  V3 n = cross(e2, e3);
  n = -1.0 * n / norm(n);
  double dp = dot(e1, n);
  V3 cop = c - dp * n;
  dp = std::abs(dp);
  V3 origin(0, 0, 0);
  double acc = 0.0;
  for (int i = 0; i < 3; ++i) {
    V3 p1, p2;
    if (i == 0) { p1 = v1; p2 = v2; }
    else if (i == 1) { p1 = v2; p2 = v3; }
    else { p1 = v3; p2 = v1; }
    double lside = dist(p1, p2);
    V3 ctl = p1 - c;
    double Rp = dist(ctl, origin);
    ctl = p2 - c;
    double Rm = dist(ctl, origin);
    V3 Pp = p1 - cop, Pm = p2 - cop;
    double d = dist(p1, p2);
    V3 ul = (p1 - p2) / d;
    double Lp = dot(Pp, ul), Lm = dot(Pm, ul);
    V3 uu = cross(ul, n);
    double P0 = dot(Pp, uu);
    if (P0 < 0) P0 = P0 * -1;
    if (!(P0 < 1.0e-10 * lside)) {
      double R0 = std::sqrt((P0 * P0) + (dp * dp));
      V3 up = Pp - Lp * ul;
      d = dist(up, origin);
      up = up / d;
      double T1 = P0 * std::log((Rp + Lp) / (Rm + Lm));
      if (P0 < 1e-6 * lside) {
        if (R0 < 1e-4 * lside) T1 = 0;
      }
      double T2 = std::atan(P0 * Lp / (R0 * R0 + dp * Rp));
      double T3 = std::atan(P0 * Lm / (R0 * R0 + dp * Rm));
      double T4 = dot(up, uu);
      acc = acc + (T4 * (T1 - dp * (T2 - T3)));
    }
  }
  return acc;
}

// getMatrixEntry, ElectrostaticsMatrix.cpp:293-340.
double Electrostatics::entryReal(unsigned i, unsigned j) const {
  const Patch& pi = mesh.patches[i];
  const Patch& pj = mesh.patches[j];
  const V3 &v1 = mesh.nodes[pj.v1], &v2 = mesh.nodes[pj.v2], &v3 = mesh.nodes[pj.v3];
  double d = dist(pi.centroid, pj.centroid);
  if (d < 4.0 * pj.largestEdge) {
    return ph.C0 * analytic(pi.centroid, v1, v2, v3);
  } else if ((d >= 4.0 * pj.largestEdge) && (d < 10.0 * pj.largestEdge)) {
    double sum = 0.0;
    for (int q = 0; q < 7; ++q) {
      V3 pt = v1 + (v2 - v1) * QA[q] + (v3 - v1) * QB[q];
      sum += pj.area * QW[q] * (1.0 / dist(pi.centroid, pt));
    }
    return ph.C0 * sum;
  } else {
    return ph.C0 * (pj.area * (1.0 / dist(pi.centroid, pj.centroid)));
  }
}

cd Electrostatics::entry(unsigned i, unsigned j) const { return cd(entryReal(i, j), 0.0); }

void Electrostatics::locations(std::vector<V3>& out) const {
  out.resize(N);
  for (int i = 0; i < N; ++i) out[i] = mesh.patches[i].centroid;
}

}  // namespace orc
