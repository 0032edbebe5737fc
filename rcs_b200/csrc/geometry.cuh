// Device-resident geometry of a triangle mesh and the FP64 matrix-entry
// formulas of the EFIE (RWG basis) and electrostatics kernels.
//
// The formulas follow vaishna77/RCS term by term so that the FP64 entries
// agree with the reference arithmetic up to the last bits of exp/log/atan:
//   Green's functions           src/includes.cpp:13-51
//   quadrature rules            src/EFIEMatrix.cpp:270-350 (truncated 7-point constants)
//   singularity extraction      src/EFIEMatrix.cpp:386-424, :457-685
//   EFIE entry                  src/EFIEMatrix.cpp:698-783
//   electrostatics entry        src/ElectrostaticsMatrix.cpp:179-340
// Reference quirks kept on purpose: the "largest edge" only compares the
// first two edges (EFIEMatrix.cpp:252), the projection used by the singular
// vector term is onto the plane through the origin (EFIEMatrix.cpp:469-474),
// and the vector non-singular part is always the 7-point rule (:419).
#pragma once
#include "common.cuh"

namespace aifmm {

// Per triangle, 16 doubles (128 B): v1, v2, v3, centroid, area, largestEdge, pad2.
constexpr int TRI_STRIDE = 16;
// Per RWG side (edge i, side 0 = "+", 1 = "-"): source triangle vertices with
// the free vertex first (the order analyticIntegration* use, EFIEMatrix.cpp:480-494).
constexpr int SIDE_STRIDE = 12;

struct EfieGeom {
  int N;          // RWG unknowns
  int nt;         // triangles
  const double* tri;    // nt x TRI_STRIDE
  const double* node;   // (nv+1) x 4, one-based ids (row 0 = dummy node)
  const int4* rwg;      // N: {t+, t-, free vertex +, free vertex -}
  const double* len;    // N
  const double* side;   // N x 2 x SIDE_STRIDE
  double kappa, freq, eps, mu, PI;
  double c4;            // -1/4/PI
  int plane_projection; // 0 = reference (plane through the origin), 1 = triangle plane
};

struct EsGeom {
  int N;                // = triangles
  const double* tri;    // nt x TRI_STRIDE
  double C0;            // 1/(4 pi eps)
};

// 7-point rule of EFIEMatrix.cpp:284-286.
__constant__ static const double kQA[7] = {0.3333333, 0.0597158, 0.470142, 0.470142, 0.7974269, 0.1012865, 0.1012865};
__constant__ static const double kQB[7] = {0.3333333, 0.470142, 0.0597158, 0.470142, 0.1012865, 0.7974269, 0.1012865};
__constant__ static const double kQW[7] = {0.225, 0.13239415278851, 0.13239415278851, 0.13239415278851,
                                           0.12593918054483, 0.12593918054483, 0.12593918054483};

struct d3 {
  double x, y, z;
};
__device__ __forceinline__ d3 mk3(double a, double b, double c) { return d3{a, b, c}; }
__device__ __forceinline__ d3 add3(d3 a, d3 b) { return d3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 sub3(d3 a, d3 b) { return d3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 mul3(d3 a, double s) { return d3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ d3 div3(d3 a, double s) { return d3{a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ double dot3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double nrm3(d3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ d3 cross3(d3 a, d3 b) {
  return d3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double dist3(d3 a, d3 b) { return nrm3(sub3(a, b)); }
__device__ __forceinline__ d3 ld3(const double* p) { return d3{p[0], p[1], p[2]}; }

struct zd3 {
  zd x, y, z;
};

// analyticIntegrationLaplaceFunction (EFIEMatrix.cpp:478-577) and, for the
// electrostatics kernel, ElectrostaticsMatrix::analyticIntegration (:179-281):
// the same edge-by-edge formula on vertices (v1, v2, v3) in the given order.
static __device__ __noinline__ double analytic_laplace(d3 c, d3 v1, d3 v2, d3 v3) {
  d3 e2 = sub3(v2, v1), e3 = sub3(v3, v1), e1 = sub3(c, v1);
  d3 n = cross3(e2, e3);
  n = div3(mul3(n, -1.0), nrm3(n));
  double dp = dot3(e1, n);
  d3 cop = sub3(c, mul3(n, dp));
  dp = fabs(dp);
  double acc = 0.0;
#pragma unroll 1
  for (int i = 0; i < 3; ++i) {
    d3 p1 = (i == 0) ? v1 : ((i == 1) ? v2 : v3);
    d3 p2 = (i == 0) ? v2 : ((i == 1) ? v3 : v1);
    double lside = dist3(p1, p2);
    double Rp = nrm3(sub3(p1, c));
    double Rm = nrm3(sub3(p2, c));
    d3 Pp = sub3(p1, cop), Pm = sub3(p2, cop);
    double d = dist3(p1, p2);
    d3 ul = div3(sub3(p1, p2), d);
    double Lp = dot3(Pp, ul), Lm = dot3(Pm, ul);
    d3 uu = cross3(ul, n);
    double P0 = dot3(Pp, uu);
    if (P0 < 0) P0 = P0 * -1;
    if (!(P0 < 1.0e-10 * lside)) {
      double R0 = sqrt((P0 * P0) + (dp * dp));
      d3 up = sub3(Pp, mul3(ul, Lp));
      up = div3(up, nrm3(up));
      double T1 = P0 * log((Rp + Lp) / (Rm + Lm));
      if (P0 < 1e-6 * lside) {
        if (R0 < 1e-4 * lside) T1 = 0;
      }
      double T2 = atan(P0 * Lp / (R0 * R0 + dp * Rp));
      double T3 = atan(P0 * Lm / (R0 * R0 + dp * Rm));
      double T4 = dot3(up, uu);
      acc = acc + (T4 * (T1 - dp * (T2 - T3)));
    }
  }
  return acc;
}

// analyticIntegrationRhoLaplaceFunction, EFIEMatrix.cpp:579-668.
static __device__ __noinline__ d3 analytic_rho_laplace(d3 c, d3 v1, d3 v2, d3 v3) {
  d3 e2 = sub3(v2, v1), e3 = sub3(v3, v1), e1 = sub3(c, v1);
  d3 n = cross3(e2, e3);
  n = div3(mul3(n, -1.0), nrm3(n));
  double dp = dot3(e1, n);
  d3 cop = sub3(c, mul3(n, dp));
  dp = fabs(dp);
  d3 acc = mk3(0, 0, 0);
#pragma unroll 1
  for (int i = 0; i < 3; ++i) {
    d3 p1 = (i == 0) ? v1 : ((i == 1) ? v2 : v3);
    d3 p2 = (i == 0) ? v2 : ((i == 1) ? v3 : v1);
    double Rp = nrm3(sub3(p1, c));
    double Rm = nrm3(sub3(p2, c));
    d3 Pp = sub3(p1, cop), Pm = sub3(p2, cop);
    double d = dist3(p1, p2);
    d3 ul = div3(sub3(p1, p2), d);
    double Lp = dot3(Pp, ul), Lm = dot3(Pm, ul);
    d3 uu = cross3(ul, n);
    double P0 = dot3(Pp, uu);
    if (P0 < 0) P0 = P0 * -1;
    double sqR0 = (P0 * P0) + (dp * dp);
    double T1;
    if ((Rm + Lm) >= 1.0e-10) T1 = sqR0 * log((Rp + Lp) / (Rm + Lm));
    else T1 = 0;
    double T2 = (Lp * Rp) - (Lm * Rm);
    acc = add3(acc, mul3(mul3(uu, 0.5), (T1 + T2)));
  }
  return acc;
}

// exp(-i kappa d) = (cos(kappa d), -sin(kappa d))
__device__ __forceinline__ zd expmikd(double kd) {
  double s, c;
  sincos(kd, &s, &c);
  return zmk(c, -s);
}

// Scalar and vector source integrals of one test-centroid / source-side pair
// (getScalarIntegrationGreensFunction, EFIEMatrix.cpp:670-685, and
// getVectorIntegrationGreensFunction, :436-446).
static __device__ __noinline__ void efie_pair(const EfieGeom& g, d3 c, int s, const double* side, zd& scal,
                                              zd3& vec) {
  const double* T = g.tri + (size_t)s * TRI_STRIDE;
  const d3 v1 = ld3(T), v2 = ld3(T + 3), v3 = ld3(T + 6), cs = ld3(T + 9);
  const double area = T[12], LE = T[13];
  const d3 n3 = ld3(side);  // free vertex
  const double kappa = g.kappa, c4 = g.c4;
  const double dcc = dist3(c, cs);
  const bool near = dcc < 4 * LE;
  const bool mid = (dcc >= 4 * LE) && (dcc < 10.0 * LE);

  // ---- vector non-singular part: always 7-point on (v2, v3, v1)
  zd3 vn = {zmk(0, 0), zmk(0, 0), zmk(0, 0)};
#pragma unroll 1
  for (int i = 0; i < 7; ++i) {
    d3 pt = add3(add3(v2, mul3(sub3(v3, v2), kQA[i])), mul3(sub3(v1, v2), kQB[i]));
    double d = dist3(c, pt);
    d3 rho = sub3(pt, n3);
    d3 rs = mul3(rho, c4);
    zd vx, vy, vz;
    if (d < 1e-12) {
      // (rho * c4) * (-i kappa)
      vx = zmk(rs.x * -0.0, rs.x * -kappa);
      vy = zmk(rs.y * -0.0, rs.y * -kappa);
      vz = zmk(rs.z * -0.0, rs.z * -kappa);
    } else {
      zd e = expmikd(kappa * d);
      zd gm = zmk(e.x - 1.0, e.y);
      vx = zmk((rs.x * gm.x) / d, (rs.x * gm.y) / d);
      vy = zmk((rs.y * gm.x) / d, (rs.y * gm.y) / d);
      vz = zmk((rs.z * gm.x) / d, (rs.z * gm.y) / d);
    }
    const double w = kQW[i];
    vn.x = zadd(vn.x, zscale(vx, w));
    vn.y = zadd(vn.y, zscale(vy, w));
    vn.z = zadd(vn.z, zscale(vz, w));
  }
  vn.x = zscale(vn.x, area);
  vn.y = zscale(vn.y, area);
  vn.z = zscale(vn.z, area);

  d3 vsing;
  if (near) {
    const d3 a1 = ld3(side), a2 = ld3(side + 3), a3 = ld3(side + 6);
    const double L = analytic_laplace(c, a1, a2, a3);
    const d3 A = analytic_rho_laplace(c, a1, a2, a3);
    // projection onto the plane through the origin (findProjectionOnTriangle)
    d3 nn = cross3(sub3(v2, v1), sub3(v3, v1));
    nn = div3(mul3(nn, -1.0), nrm3(nn));
    const double dd = g.plane_projection ? dot3(sub3(c, v1), nn) : dot3(c, nn);
    const d3 proj = sub3(c, mul3(nn, dd));
    const d3 B = sub3(proj, n3);
    vsing = mk3(c4 * (A.x + L * B.x), c4 * (A.y + L * B.y), c4 * (A.z + L * B.z));
    // scalar: c4 * analytic + area * sum_i w_i Gns(c, pt_i) on (v1, v2, v3)
    zd sum = zmk(0, 0);
#pragma unroll 1
    for (int i = 0; i < 7; ++i) {
      d3 pt = add3(add3(v1, mul3(sub3(v2, v1), kQA[i])), mul3(sub3(v3, v1), kQB[i]));
      double d = dist3(pt, c);
      zd t;
      if (d < 1e-12) {
        t = zmk(0.0, ((kQW[i] * kappa) / 4.0) / g.PI);
      } else {
        zd e = expmikd(kappa * d);
        zd gm = zmk(e.x - 1.0, e.y);
        zd gg = zmk((c4 * gm.x) / d, (c4 * gm.y) / d);
        t = zscale(gg, kQW[i]);
      }
      sum = zadd(sum, t);
    }
    const zd as = zscale(sum, area);
    scal = zmk(c4 * L + as.x, as.y);
  } else if (mid) {
    d3 acc = mk3(0, 0, 0);
    zd sum = zmk(0, 0);
#pragma unroll 1
    for (int i = 0; i < 7; ++i) {
      // rhoLaplace on (v2, v3, v1)
      d3 pt = add3(add3(v2, mul3(sub3(v3, v2), kQA[i])), mul3(sub3(v1, v2), kQB[i]));
      double d = dist3(c, pt);
      d3 rho = sub3(pt, n3);
      acc = add3(acc, mul3(div3(mul3(rho, c4), d), kQW[i]));
      // EFIE Green's function on (v1, v2, v3)
      d3 ps = add3(add3(v1, mul3(sub3(v2, v1), kQA[i])), mul3(sub3(v3, v1), kQB[i]));
      double ds = dist3(c, ps);
      zd e = expmikd(kappa * ds);
      zd gg = zmk((c4 * e.x) / ds, (c4 * e.y) / ds);
      sum = zadd(sum, zscale(gg, kQW[i]));
    }
    vsing = mul3(acc, area);
    scal = zscale(sum, area);
  } else {
    double d = dist3(c, cs);
    d3 rho = sub3(cs, n3);
    vsing = mul3(div3(mul3(rho, c4), d), area);
    zd e = expmikd(kappa * d);
    zd gg = zmk((c4 * e.x) / d, (c4 * e.y) / d);
    scal = zscale(gg, area);
  }
  vec.x = zmk(vn.x.x + vsing.x, vn.x.y);
  vec.y = zmk(vn.y.x + vsing.y, vn.y.y);
  vec.z = zmk(vn.z.x + vsing.z, vn.z.y);
}

// EFIEMatrix::getMatrixEntry, EFIEMatrix.cpp:698-783.
__device__ __forceinline__ zd efie_entry(const EfieGeom& g, int i, int j) {
  const int4 ti = g.rwg[i], sj = g.rwg[j];
  const double Lt = g.len[i], Ls = g.len[j];
  const double* side_s[2] = {g.side + ((size_t)j * 2 + 0) * SIDE_STRIDE, g.side + ((size_t)j * 2 + 1) * SIDE_STRIDE};
  const double As[2] = {g.tri[(size_t)sj.x * TRI_STRIDE + 12], g.tri[(size_t)sj.y * TRI_STRIDE + 12]};
  const double LtLs = Lt * Ls;
  // The four triangle pairs in the reference's summation order ++, +-, -+, --;
  // the loop is kept rolled so that the kernel fits the instruction cache.
  zd z = zmk(0, 0), f = zmk(0, 0);
#pragma unroll 1
  for (int p4 = 0; p4 < 4; ++p4) {
    const int a = p4 >> 1, b = p4 & 1;
    const int ta = a ? ti.y : ti.x;
    const double* Tt = g.tri + (size_t)ta * TRI_STRIDE;
    const d3 ct = ld3(Tt + 9);
    const double At = Tt[12];
    const d3 n3t = ld3(g.node + (size_t)(a ? ti.w : ti.z) * 4);
    const d3 rc = sub3(ct, n3t);
    const d3 ar = mul3(rc, At);
    const double Asb = b ? As[1] : As[0];
    zd scal;
    zd3 vec;
    efie_pair(g, ct, b ? sj.y : sj.x, b ? side_s[1] : side_s[0], scal, vec);
    // phi term: sign * i * Lt Ls / (2 pi f eps At As) * At * scalar
    const double D = (((2.0 * g.PI) * g.freq) * g.eps) * At * Asb;
    const double p = LtLs / D;
    const double sgn = (a == b) ? 1.0 : -1.0;  // ++, -- : +i ;  +-, -+ : -i
    const zd phiI = zmk(At * scal.x, At * scal.y);
    const zd ephi = zmk(-(sgn * p) * phiI.y, (sgn * p) * phiI.x);
    // A term: -/+ i 2 pi f mu Lt Ls / (4 At As) * (At rho_c . vec)
    const double X = (((((2.0 * g.PI) * g.freq) * g.mu) * Lt) * Ls) / ((4.0 * At) * Asb);
    const zd ai = zadd(zadd(zscale(vec.x, ar.x), zscale(vec.y, ar.y)), zscale(vec.z, ar.z));
    const double q = (a == b) ? -X : X;
    const zd eA = zmk(-q * ai.y, q * ai.x);
    if (p4 == 0) {
      z = ephi;
      f = eA;
    } else {
      z = zadd(z, ephi);
      f = zadd(f, eA);
    }
  }
  return zadd(z, f);
}

// ElectrostaticsMatrix::getMatrixEntry, ElectrostaticsMatrix.cpp:293-340.
__device__ __forceinline__ double es_entry(const EsGeom& g, int i, int j) {
  const double* Ti = g.tri + (size_t)i * TRI_STRIDE;
  const double* Tj = g.tri + (size_t)j * TRI_STRIDE;
  const d3 ci = ld3(Ti + 9);
  const d3 v1 = ld3(Tj), v2 = ld3(Tj + 3), v3 = ld3(Tj + 6), cj = ld3(Tj + 9);
  const double area = Tj[12], LE = Tj[13];
  const double d = dist3(ci, cj);
  if (d < 4.0 * LE) return g.C0 * analytic_laplace(ci, v1, v2, v3);
  if ((d >= 4.0 * LE) && (d < 10.0 * LE)) {
    double sum = 0.0;
#pragma unroll 1
    for (int q = 0; q < 7; ++q) {
      d3 pt = add3(add3(v1, mul3(sub3(v2, v1), kQA[q])), mul3(sub3(v3, v1), kQB[q]));
      sum += area * kQW[q] * (1.0 / dist3(ci, pt));
    }
    return g.C0 * sum;
  }
  return g.C0 * (area * (1.0 / d));
}

}  // namespace aifmm
