// Matrix-entry assembly kernels (FP64 reference-exact formulas; the file is
// compiled with -fmad=false so that a*b+c rounds like the reference) and the
// electrostatic kernel's geometry tables (the EFIE tables are built on the
// GPU, mesh_build.cu).
#include <algorithm>
#include <cmath>
#include <vector>

#include "assemble.cuh"

namespace aifmm {

// ------------------------------------------------------------------ kernels
// One thread per entry; consecutive threads take consecutive rows of one
// column so that the column-major output is written with coalesced stores.
template <typename OutT>
__device__ __forceinline__ void store_entry(OutT* out, size_t idx, zd v);
template <>
__device__ __forceinline__ void store_entry<zd>(zd* out, size_t idx, zd v) {
  out[idx] = v;
}
template <>
__device__ __forceinline__ void store_entry<zf>(zf* out, size_t idx, zd v) {
  out[idx] = make_float2((float)v.x, (float)v.y);
}

template <typename OutT>
__global__ void __launch_bounds__(256, 2) efie_gather_kernel(EfieGeom g, const int* __restrict__ rows, int nr,
                                                          const int* __restrict__ cols, int nc, OutT* out, int ld) {
  const long total = (long)nr * nc;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const int a = (int)(t % nr), b = (int)(t / nr);
    store_entry<OutT>(out, (size_t)b * ld + a, efie_entry(g, rows[a], cols[b]));
  }
}

template <typename OutT>
__global__ void __launch_bounds__(256) es_gather_kernel(EsGeom g, const int* __restrict__ rows, int nr,
                                                        const int* __restrict__ cols, int nc, OutT* out, int ld) {
  const long total = (long)nr * nc;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const int a = (int)(t % nr), b = (int)(t / nr);
    store_entry<OutT>(out, (size_t)b * ld + a, zmk(es_entry(g, rows[a], cols[b]), 0.0));
  }
}

// Many blocks in one launch: blocks[q] describes an nr x nc tile, start[q]
// the prefix sum of entries; each thread finds its tile by binary search.
template <typename OutT, bool EFIE>
__global__ void __launch_bounds__(256, 2) batched_gather_kernel(EfieGeom ge, EsGeom gs, const GatherBlock* __restrict__ blocks,
                                                             const long* __restrict__ start, int nblocks, long total) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nblocks - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (start[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    const GatherBlock& B = blocks[lo];
    const long u = t - start[lo];
    const int a = (int)(u % B.nr), b = (int)(u / B.nr);
    zd v = EFIE ? efie_entry(ge, B.rows[a], B.cols[b]) : zmk(es_entry(gs, B.rows[a], B.cols[b]), 0.0);
    store_entry<OutT>(reinterpret_cast<OutT*>(B.out), (size_t)b * B.ld + a, v);
  }
}

// EFIEMatrix::getRhs (EFIEMatrix.cpp:792-829) with the default incidence
// (theta = phi = 0) and its phase vector (kappa sin.cos, kappa sin.sin, cos).
__global__ void efie_rhs_reference_kernel(EfieGeom g, double e0, double e1, double e2, zd* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const int4 r = g.rwg[i];
  const double Lt = g.len[i];
  const double *Tp = g.tri + (size_t)r.x * TRI_STRIDE, *Tm = g.tri + (size_t)r.y * TRI_STRIDE;
  const d3 cp = ld3(Tp + 9), cm = ld3(Tm + 9);
  const d3 rp = sub3(cp, ld3(g.node + (size_t)r.z * 4)), rm = sub3(cm, ld3(g.node + (size_t)r.w * 4));
  const double theta = 0.0, phi = 0.0;
  const d3 kv = mk3(g.kappa * sin(theta) * cos(phi), g.kappa * sin(theta) * sin(phi), cos(theta));
  const double kp = dot3(kv, cp), km = dot3(kv, cm);
  double sp, cpp, sm, cmm;
  sincos(kp, &sp, &cpp);
  sincos(km, &sm, &cmm);
  const zd ep = zmk(cpp, sp), em = zmk(cmm, sm);
  zd dp = zadd(zadd(zscale(zscale(ep, e0), rp.x), zscale(zscale(ep, e1), rp.y)), zscale(zscale(ep, e2), rp.z));
  zd dm = zadd(zadd(zscale(zscale(em, e0), rm.x), zscale(zscale(em, e1), rm.y)), zscale(zscale(em, e2), rm.z));
  out[i] = zscale(zsub(dp, dm), Lt / 2.0);
}

// Plane wave E0 exp(-i kappa khat.r) sampled at the test-triangle centroids.
__global__ void efie_rhs_plane_kernel(EfieGeom g, d3 khat, zd3 E0, zd* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const int4 r = g.rwg[i];
  const double Lt = g.len[i];
  const double *Tp = g.tri + (size_t)r.x * TRI_STRIDE, *Tm = g.tri + (size_t)r.y * TRI_STRIDE;
  const d3 cp = ld3(Tp + 9), cm = ld3(Tm + 9);
  const d3 rp = sub3(cp, ld3(g.node + (size_t)r.z * 4)), rm = sub3(cm, ld3(g.node + (size_t)r.w * 4));
  const zd ep = expmikd(g.kappa * dot3(khat, cp));
  const zd em = expmikd(g.kappa * dot3(khat, cm));
  zd dp = zadd(zadd(zscale(E0.x, rp.x), zscale(E0.y, rp.y)), zscale(E0.z, rp.z));
  zd dm = zadd(zadd(zscale(E0.x, rm.x), zscale(E0.y, rm.y)), zscale(E0.z, rm.z));
  out[i] = zscale(zsub(zmul(dp, ep), zmul(dm, em)), Lt / 2.0);
}

// ------------------------------------------------------------------ launches
static int grid_for(long total) {
  long g = (total + 255) / 256;
  return (int)std::max<long>(1, std::min<long>(g, 148L * 64));
}

void launch_gather(const KernelGeom& k, const int* rows, int nr, const int* cols, int nc, int precision, void* out,
                   int ld, cudaStream_t s) {
  if (nr <= 0 || nc <= 0) return;
  const int grid = grid_for((long)nr * nc);
  if (k.efie) {
    if (precision == 0) efie_gather_kernel<zd><<<grid, 256, 0, s>>>(k.ge, rows, nr, cols, nc, (zd*)out, ld);
    else efie_gather_kernel<zf><<<grid, 256, 0, s>>>(k.ge, rows, nr, cols, nc, (zf*)out, ld);
  } else {
    if (precision == 0) es_gather_kernel<zd><<<grid, 256, 0, s>>>(k.gs, rows, nr, cols, nc, (zd*)out, ld);
    else es_gather_kernel<zf><<<grid, 256, 0, s>>>(k.gs, rows, nr, cols, nc, (zf*)out, ld);
  }
  AIFMM_LAUNCHED();
}

void launch_batched_gather(const KernelGeom& k, const GatherBlock* blocks_dev, const long* start_dev, int nblocks,
                           long total, int precision, cudaStream_t s) {
  if (nblocks <= 0 || total <= 0) return;
  const int grid = grid_for(total);
  if (k.efie) {
    if (precision == 0) batched_gather_kernel<zd, true><<<grid, 256, 0, s>>>(k.ge, k.gs, blocks_dev, start_dev, nblocks, total);
    else batched_gather_kernel<zf, true><<<grid, 256, 0, s>>>(k.ge, k.gs, blocks_dev, start_dev, nblocks, total);
  } else {
    if (precision == 0) batched_gather_kernel<zd, false><<<grid, 256, 0, s>>>(k.ge, k.gs, blocks_dev, start_dev, nblocks, total);
    else batched_gather_kernel<zf, false><<<grid, 256, 0, s>>>(k.ge, k.gs, blocks_dev, start_dev, nblocks, total);
  }
  AIFMM_LAUNCHED();
}

void launch_rhs_reference(const KernelGeom& k, const double* einc, zd* out, cudaStream_t s) {
  efie_rhs_reference_kernel<<<ceil_div(k.N, 256), 256, 0, s>>>(k.ge, einc[0], einc[1], einc[2], out);
  AIFMM_LAUNCHED();
}

void launch_rhs_plane(const KernelGeom& k, const double* khat, const double* e0, zd* out, cudaStream_t s) {
  d3 kh{khat[0], khat[1], khat[2]};
  zd3 E{zmk(e0[0], e0[1]), zmk(e0[2], e0[3]), zmk(e0[4], e0[5])};
  efie_rhs_plane_kernel<<<ceil_div(k.N, 256), 256, 0, s>>>(k.ge, kh, E, out);
  AIFMM_LAUNCHED();
}

// ------------------------------------------------------------------ host tables
static double hdist(const double* a, const double* b) {
  double x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
  return std::sqrt(x * x + y * y + z * z);
}

// Triangle table: vertices, centroid, area, "largest edge" of the first two
// edges (EFIEMatrix.cpp:247-268).
static void build_tri_table(const double* xyz, int nv, const int* tris, int nt, std::vector<double>& tri) {
  tri.assign((size_t)nt * TRI_STRIDE, 0.0);
  for (int t = 0; t < nt; ++t) {
    int id[3] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
    for (int q = 0; q < 3; ++q)
      AIFMM_REQUIRE(id[q] >= 1 && id[q] <= nv, AIFMM_EINVAL, "triangle vertex id out of range");
    const double *a = xyz + 3 * (id[0] - 1), *b = xyz + 3 * (id[1] - 1), *c = xyz + 3 * (id[2] - 1);
    double* T = &tri[(size_t)t * TRI_STRIDE];
    for (int q = 0; q < 3; ++q) {
      T[q] = a[q];
      T[3 + q] = b[q];
      T[6 + q] = c[q];
      T[9 + q] = (a[q] + b[q] + c[q]) / 3.0;
    }
    double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    T[12] = 0.5 * std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    double l1 = hdist(a, b), l2 = hdist(b, c);
    T[13] = (l2 > l1) ? l2 : l1;
  }
}

void build_es_tables(const double* xyz, int nv, const int* tris, int nt, std::vector<double>& tri,
                     std::vector<double>& locations) {
  build_tri_table(xyz, nv, tris, nt, tri);
  locations.assign((size_t)nt * 3, 0.0);
  for (int t = 0; t < nt; ++t)
    for (int q = 0; q < 3; ++q) locations[3 * t + q] = tri[(size_t)t * TRI_STRIDE + 9 + q];
}

}  // namespace aifmm
