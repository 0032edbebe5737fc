// Post-solve far field of an EFIE solution: surface current at the triangle
// centroids (EFIEMatrix::getJAtCentroids, src/EFIEMatrix.cpp:1100-1130) and the
// bistatic radar cross-section by one-point quadrature
// (EFIEMatrix::getRCS_OnePointQuadrature, :916-930).
//
// Currents: one thread per triangle sums the contributions of the RWG edges
// that touch it, in ascending edge order (the order of the reference's loop
// over unknowns), from a triangle -> edge incidence list built once per kernel.
// Each contribution is formed in the reference's operation order,
// ((c rho) L / 2) / A, and this file is compiled without FMA contraction.
//
// RCS: one CTA per observation angle; its threads stride over the triangles
// and a fixed-shape tree reduction combines the partial sums, so the result is
// the same on every run.  Traffic per angle is the current array (48 bytes a
// triangle) plus the centroid/area table; both stay in L2 across angles.
#include <algorithm>
#include <cmath>
#include <vector>

#include "capi_guard.cuh"
#include "context.cuh"

using namespace aifmm;

namespace {

constexpr int RCS_NT = 256;

__global__ void centroid_current_kernel(const double* __restrict__ tri, const double* __restrict__ node,
                                        const int4* __restrict__ rwg, const double* __restrict__ len,
                                        const int* __restrict__ off, const int* __restrict__ inc,
                                        const zd* __restrict__ coeff, int N, int nt, zd* __restrict__ J) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const double* T = tri + (size_t)t * TRI_STRIDE;
  const double area = T[12];
  zd acc[3] = {zmk(0, 0), zmk(0, 0), zmk(0, 0)};
  for (int e = off[t]; e < off[t + 1]; ++e) {
    const int code = inc[e];
    const int i = code >> 1, minus = code & 1;
    const int4 r = rwg[i];
    const int fv = minus ? r.w : r.z;
    zd c = coeff[i];
    if (minus) c = zmk(-c.x, -c.y);
    const double L = len[i];
    for (int q = 0; q < 3; ++q) {
      const double rho = T[9 + q] - node[(size_t)fv * 4 + q];
      const double re = ((c.x * rho) * L * 0.5) / area;
      const double im = ((c.y * rho) * L * 0.5) / area;
      acc[q] = zadd(acc[q], zmk(re, im));
    }
  }
  for (int q = 0; q < 3; ++q) J[(size_t)q * nt + t] = acc[q];  // nt x 3, column-major
}

__global__ void rcs_kernel(const double* __restrict__ tri, const zd* __restrict__ J, int nt,
                           const double* __restrict__ theta, const double* __restrict__ phi, double kappa,
                           double PI, double* __restrict__ out) {
  const int a = blockIdx.x;
  double st, ct, sp, cp;
  sincos(theta[a], &st, &ct);
  sincos(phi[a], &sp, &cp);
  const double kx = kappa * st * cp, ky = kappa * st * sp, kz = kappa * ct;
  double s0r = 0, s0i = 0, s1r = 0, s1i = 0;
  for (int t = threadIdx.x; t < nt; t += RCS_NT) {
    const double* T = tri + (size_t)t * TRI_STRIDE;
    const zd j0 = J[t], j1 = J[(size_t)nt + t], j2 = J[2 * (size_t)nt + t];
    double sn, cs;
    sincos(kx * T[9] + ky * T[10] + kz * T[11], &sn, &cs);
    // theta and phi components of J (the reference's dot products with the
    // spherical unit vectors), times exp(i k.r) and the area
    const double ar = j0.x * ct * cp + j1.x * ct * sp - j2.x * st, ai = j0.y * ct * cp + j1.y * ct * sp - j2.y * st;
    const double br = -j0.x * sp + j1.x * cp, bi = -j0.y * sp + j1.y * cp;
    const double area = T[12];
    s0r += (ar * cs - ai * sn) * area;
    s0i += (ar * sn + ai * cs) * area;
    s1r += (br * cs - bi * sn) * area;
    s1i += (br * sn + bi * cs) * area;
  }
  __shared__ double red[4][RCS_NT];
  red[0][threadIdx.x] = s0r;
  red[1][threadIdx.x] = s0i;
  red[2][threadIdx.x] = s1r;
  red[3][threadIdx.x] = s1i;
  __syncthreads();
  for (int w = RCS_NT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int q = 0; q < 4; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double neta = 377.0;
    const double at = std::hypot(red[0][0], red[1][0]), ap = std::hypot(red[2][0], red[3][0]);
    out[a] = kappa * kappa / (4.0 * PI) * neta * at * neta * at + kappa * kappa / (4.0 * PI) * neta * ap * neta * ap;
  }
}

// Triangle -> (edge, side) incidence in ascending edge order; code = 2 edge + side.
void ensure_incidence(aifmm_kernel* k) {
  if (k->d_t2e_off.p) return;
  const int nt = k->geom.ge.nt, N = k->geom.N;
  std::vector<int> off(nt + 1, 0), inc(2 * (size_t)N);
  for (int i = 0; i < N; ++i)
    for (int s = 0; s < 2; ++s) off[k->rwg_host[4 * i + s] + 1]++;
  for (int t = 0; t < nt; ++t) off[t + 1] += off[t];
  std::vector<int> fill(off.begin(), off.end() - 1);
  for (int i = 0; i < N; ++i)
    for (int s = 0; s < 2; ++s) inc[fill[k->rwg_host[4 * i + s]]++] = 2 * i + s;
  k->d_t2e_inc = upload(k->ctx, inc);
  k->d_t2e_off = upload(k->ctx, off);
}

}  // namespace

extern "C" {

int aifmm_kernel_currents(aifmm_kernel* k, const double* coeff, double* J) {
  API_BEGIN
  AIFMM_REQUIRE(k && coeff && J, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(k->geom.efie, AIFMM_EINVAL, "not an EFIE kernel");
  aifmm_ctx* c = k->ctx;
  AIFMM_CUDA(cudaSetDevice(c->device));
  ensure_incidence(k);
  const int N = k->geom.N, nt = k->geom.ge.nt;
  DevBuf dc(c, sizeof(zd) * N), dJ(c, sizeof(zd) * 3 * (size_t)nt);
  AIFMM_CUDA(cudaMemcpyAsync(dc.p, coeff, sizeof(zd) * N, cudaMemcpyHostToDevice, c->stream));
  centroid_current_kernel<<<ceil_div(nt, 128), 128, 0, c->stream>>>(
      k->geom.ge.tri, k->geom.ge.node, k->geom.ge.rwg, k->geom.ge.len, k->d_t2e_off.as<int>(),
      k->d_t2e_inc.as<int>(), dc.as<zd>(), N, nt, dJ.as<zd>());
  AIFMM_LAUNCHED();
  AIFMM_CUDA(cudaMemcpyAsync(J, dJ.p, sizeof(zd) * 3 * (size_t)nt, cudaMemcpyDeviceToHost, c->stream));
  AIFMM_CUDA(cudaStreamSynchronize(c->stream));
  API_END
}

int aifmm_kernel_rcs(aifmm_kernel* k, const double* J, int n_angles, const double* theta, const double* phi,
                     double* rcs) {
  API_BEGIN
  AIFMM_REQUIRE(k && J && theta && phi && rcs, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(k->geom.efie, AIFMM_EINVAL, "not an EFIE kernel");
  AIFMM_REQUIRE(n_angles > 0, AIFMM_EINVAL, "no observation angle");
  for (int a = 0; a < n_angles; ++a)
    AIFMM_REQUIRE(std::isfinite(theta[a]) && std::isfinite(phi[a]), AIFMM_EINVAL, "non-finite angle");
  aifmm_ctx* c = k->ctx;
  AIFMM_CUDA(cudaSetDevice(c->device));
  const int nt = k->geom.ge.nt;
  DevBuf dJ(c, sizeof(zd) * 3 * (size_t)nt), dang(c, sizeof(double) * 2 * (size_t)n_angles),
      dout(c, sizeof(double) * n_angles);
  AIFMM_CUDA(cudaMemcpyAsync(dJ.p, J, sizeof(zd) * 3 * (size_t)nt, cudaMemcpyHostToDevice, c->stream));
  AIFMM_CUDA(cudaMemcpyAsync(dang.p, theta, sizeof(double) * n_angles, cudaMemcpyHostToDevice, c->stream));
  AIFMM_CUDA(cudaMemcpyAsync(dang.as<double>() + n_angles, phi, sizeof(double) * n_angles, cudaMemcpyHostToDevice,
                             c->stream));
  rcs_kernel<<<n_angles, RCS_NT, 0, c->stream>>>(k->geom.ge.tri, dJ.as<zd>(), nt, dang.as<double>(),
                                                 dang.as<double>() + n_angles, k->geom.ge.kappa, k->geom.ge.PI,
                                                 dout.as<double>());
  AIFMM_LAUNCHED();
  AIFMM_CUDA(cudaMemcpyAsync(rcs, dout.p, sizeof(double) * n_angles, cudaMemcpyDeviceToHost, c->stream));
  AIFMM_CUDA(cudaStreamSynchronize(c->stream));
  API_END
}

}  // extern "C"
