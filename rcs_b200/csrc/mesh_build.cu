// Mesh -> RWG tables and octree binning on the GPU.
//
// RWG numbering (src/EFIEMatrix.cpp:129-209, :353-373): every triangle t
// contributes its three edges (v1,v2), (v2,v3), (v3,v1), keyed by (min node,
// max node); the reference's unknowns are the keys of a std::map in
// ascending key order, dropping keys seen once (boundary edges); the first
// triangle in file order that contains an edge is its "+" side, the second its
// "-" side; the free vertex is the triangle's third node.  Here the 3 nt
// (key, 3 t + e) pairs are sorted by key with a stable radix sort (equal keys
// keep file order), so the first two entries of a key's run are its "+" and
// "-" triangles and the ascending runs of length >= 2 are the unknowns in the
// map's order.  Triangle geometry, edge lengths, side tables and the edge
// midpoints are computed with the host build's operation order (this file is
// compiled without contraction), so the tables are bit-identical to it.
//
// Octree binning (T:576-625): each point walks from the root to its leaf,
// choosing at every level the child of the box whose centre it is compared
// with (z, then x, then y, with <=); the reference appends a box's points to
// its children in order, so a leaf's list is the points of that leaf in index
// order -- a stable sort of the point indices by leaf id.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "assemble.cuh"
#include "context.cuh"

namespace aifmm {

namespace {

__device__ __forceinline__ double mb_dist(const double* a, const double* b) {
  const double x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
  return sqrt(x * x + y * y + z * z);
}

// triangle table (build_tri_table's arithmetic) and the three edge keys
__global__ void mb_tri_kernel(const double* __restrict__ xyz, int nv, const int* __restrict__ tris, int nt,
                              double* __restrict__ tri, unsigned long long* __restrict__ keys,
                              int* __restrict__ vals, int* __restrict__ bad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int id[3] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
  for (int q = 0; q < 3; ++q)
    if (id[q] < 1 || id[q] > nv) {
      atomicExch(bad, 1);
      for (int e = 0; e < 3; ++e) {
        keys[3 * t + e] = ~0ull;
        vals[3 * t + e] = 3 * t + e;
      }
      return;
    }
  const double *a = xyz + 3 * (id[0] - 1), *b = xyz + 3 * (id[1] - 1), *c = xyz + 3 * (id[2] - 1);
  double* T = tri + (size_t)t * TRI_STRIDE;
  for (int q = 0; q < 3; ++q) {
    T[q] = a[q];
    T[3 + q] = b[q];
    T[6 + q] = c[q];
    T[9 + q] = (a[q] + b[q] + c[q]) / 3.0;
  }
  const double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  const double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
  T[12] = 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
  const double l1 = mb_dist(a, b), l2 = mb_dist(b, c);
  T[13] = (l2 > l1) ? l2 : l1;
  T[14] = T[15] = 0.0;
  for (int e = 0; e < 3; ++e) {
    const int u = id[e], v = id[(e + 1) % 3];
    const unsigned long long lo = (unsigned)min(u, v), hi = (unsigned)max(u, v);
    keys[3 * t + e] = (lo << 32) | hi;
    vals[3 * t + e] = 3 * t + e;
  }
}

// 1 where a sorted run of length >= 2 starts (an RWG unknown)
__global__ void mb_flag_kernel(const unsigned long long* __restrict__ keys, int n, int* __restrict__ flag) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const bool start = (p == 0) || keys[p] != keys[p - 1];
  flag[p] = (start && p + 1 < n && keys[p + 1] == keys[p] && keys[p] != ~0ull) ? 1 : 0;
}

__device__ __forceinline__ int mb_third(const int* tris, int t, int a, int b) {
  for (int q = 0; q < 3; ++q) {
    const int v = tris[3 * t + q];
    if (v != a && v != b) return v;
  }
  return tris[3 * t];  // degenerate triangle: the reference's set difference is empty too
}

// per unknown: rwg {t+, t-, free+, free-}, length, edge nodes, side table, midpoint
__global__ void mb_rwg_kernel(const unsigned long long* __restrict__ keys, const int* __restrict__ vals,
                              const int* __restrict__ flag, const int* __restrict__ idx, int n,
                              const double* __restrict__ xyz, const int* __restrict__ tris, int* __restrict__ rwg,
                              double* __restrict__ len, int* __restrict__ edge, double* __restrict__ side,
                              double* __restrict__ loc) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n || !flag[p]) return;
  const int i = idx[p];
  const int a = (int)(keys[p] >> 32), b = (int)(keys[p] & 0xFFFFFFFFull);
  const int tp = vals[p] / 3, tm = vals[p + 1] / 3;
  const int fp = mb_third(tris, tp, a, b), fm = mb_third(tris, tm, a, b);
  rwg[4 * i] = tp;
  rwg[4 * i + 1] = tm;
  rwg[4 * i + 2] = fp;
  rwg[4 * i + 3] = fm;
  // the first occurrence's orientation (vertex order within its triangle)
  const int e = vals[p] % 3;
  const int u = tris[3 * tp + e], v = tris[3 * tp + (e + 1) % 3];
  len[i] = mb_dist(xyz + 3 * (u - 1), xyz + 3 * (v - 1));
  edge[2 * i] = a;
  edge[2 * i + 1] = b;
  for (int s = 0; s < 2; ++s) {
    const int t = s ? tm : tp, fv = s ? fm : fp;
    const int v1 = tris[3 * t], v2 = tris[3 * t + 1], v3 = tris[3 * t + 2];
    int i2, i3;  // free vertex first (EFIEMatrix.cpp:480-494)
    if (v1 == fv) { i2 = v2; i3 = v3; }
    else if (v2 == fv) { i2 = v1; i3 = v3; }
    else { i2 = v1; i3 = v2; }
    double* S = side + ((size_t)i * 2 + s) * SIDE_STRIDE;
    const int ids[3] = {fv, i2, i3};
    for (int q = 0; q < 3; ++q)
      for (int c = 0; c < 3; ++c) S[3 * q + c] = xyz[3 * (ids[q] - 1) + c];
    for (int q = 9; q < SIDE_STRIDE; ++q) S[q] = 0.0;
  }
  for (int q = 0; q < 3; ++q) loc[3 * i + q] = (xyz[3 * (a - 1) + q] + xyz[3 * (b - 1) + q]) / 2.0;
}

__global__ void mb_bin_kernel(const double* __restrict__ pts, int n, const double* __restrict__ centers, int nLevels,
                              unsigned* __restrict__ leaf, int* __restrict__ order) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* p = pts + 3 * (size_t)i;
  long k = 0, levelStart = 0, boxes = 1;
  for (int j = 0; j < nLevels; ++j) {
    const double* c = centers + 3 * (size_t)(levelStart + k);
    int ch;
    if (p[2] <= c[2]) {
      if (p[0] <= c[0]) ch = (p[1] <= c[1]) ? 0 : 3;
      else ch = (p[1] <= c[1]) ? 1 : 2;
    } else {
      if (p[0] <= c[0]) ch = (p[1] <= c[1]) ? 4 : 7;
      else ch = (p[1] <= c[1]) ? 5 : 6;
    }
    levelStart += boxes;
    boxes *= 8;
    k = 8 * k + ch;
  }
  leaf[i] = (unsigned)k;
  order[i] = i;
}

// cub's stable radix sort of (key, value) pairs, on the context stream
template <typename K, typename V>
void mb_sort(aifmm_ctx* ctx, const K* kin, K* kout, const V* vin, V* vout, int n, int bits) {
  size_t tmp = 0;
  AIFMM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, kin, kout, vin, vout, n, 0, bits, ctx->stream));
  DevBuf t(ctx, std::max<size_t>(tmp, 16));
  AIFMM_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, kin, kout, vin, vout, n, 0, bits, ctx->stream));
}

template <typename T>
std::vector<T> mb_download(aifmm_ctx* ctx, const DevBuf& b, size_t n) {
  std::vector<T> h(n);
  if (n) AIFMM_CUDA(cudaMemcpyAsync(h.data(), b.p, sizeof(T) * n, cudaMemcpyDeviceToHost, ctx->stream));
  return h;
}

}  // namespace

void build_efie_tables_gpu(aifmm_ctx* ctx, const double* xyz, int nv, const int* tris, int nt, EfieHostTables& h) {
  AIFMM_REQUIRE(nt > 0 && nv > 0 && (long)nt * 3 < (long)INT32_MAX, AIFMM_EINVAL, "bad mesh size");
  const int ne = 3 * nt;
  std::vector<double> vxyz(xyz, xyz + 3 * (size_t)nv);
  std::vector<int> vtris(tris, tris + 3 * (size_t)nt);
  DevBuf dxyz = upload(ctx, vxyz), dtris = upload(ctx, vtris);
  DevBuf dtri(ctx, sizeof(double) * (size_t)nt * TRI_STRIDE);
  DevBuf k0(ctx, sizeof(unsigned long long) * ne), k1(ctx, sizeof(unsigned long long) * ne);
  DevBuf v0(ctx, sizeof(int) * ne), v1(ctx, sizeof(int) * ne), flag(ctx, sizeof(int) * ne), idx(ctx, sizeof(int) * ne);
  DevBuf bad(ctx, sizeof(int));
  AIFMM_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
  mb_tri_kernel<<<(nt + 255) / 256, 256, 0, ctx->stream>>>(dxyz.as<double>(), nv, dtris.as<int>(), nt,
                                                           dtri.as<double>(), k0.as<unsigned long long>(),
                                                           v0.as<int>(), bad.as<int>());
  AIFMM_LAUNCHED();
  mb_sort(ctx, k0.as<unsigned long long>(), k1.as<unsigned long long>(), v0.as<int>(), v1.as<int>(), ne, 64);
  mb_flag_kernel<<<(ne + 255) / 256, 256, 0, ctx->stream>>>(k1.as<unsigned long long>(), ne, flag.as<int>());
  AIFMM_LAUNCHED();
  {
    size_t tmp = 0;
    AIFMM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, flag.as<int>(), idx.as<int>(), ne, ctx->stream));
    DevBuf t(ctx, std::max<size_t>(tmp, 16));
    AIFMM_CUDA(cub::DeviceScan::ExclusiveSum(t.p, tmp, flag.as<int>(), idx.as<int>(), ne, ctx->stream));
  }
  int last[2] = {0, 0}, badh = 0;
  AIFMM_CUDA(cudaMemcpyAsync(&last[0], idx.as<int>() + ne - 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  AIFMM_CUDA(cudaMemcpyAsync(&last[1], flag.as<int>() + ne - 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  AIFMM_CUDA(cudaMemcpyAsync(&badh, bad.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
  AIFMM_REQUIRE(badh == 0, AIFMM_EINVAL, "triangle vertex id out of range");
  const int N = last[0] + last[1];
  h.tri = mb_download<double>(ctx, dtri, (size_t)nt * TRI_STRIDE);
  h.node.assign((size_t)(nv + 1) * 4, 0.0);
  for (int i = 0; i < nv; ++i)
    for (int q = 0; q < 3; ++q) h.node[(size_t)(i + 1) * 4 + q] = xyz[3 * i + q];
  if (N > 0) {
    DevBuf drwg(ctx, sizeof(int) * 4 * (size_t)N), dlen(ctx, sizeof(double) * N), dedge(ctx, sizeof(int) * 2 * (size_t)N);
    DevBuf dside(ctx, sizeof(double) * (size_t)N * 2 * SIDE_STRIDE), dloc(ctx, sizeof(double) * 3 * (size_t)N);
    mb_rwg_kernel<<<(ne + 255) / 256, 256, 0, ctx->stream>>>(
        k1.as<unsigned long long>(), v1.as<int>(), flag.as<int>(), idx.as<int>(), ne, dxyz.as<double>(),
        dtris.as<int>(), drwg.as<int>(), dlen.as<double>(), dedge.as<int>(), dside.as<double>(), dloc.as<double>());
    AIFMM_LAUNCHED();
    h.rwg = mb_download<int>(ctx, drwg, 4 * (size_t)N);
    h.len = mb_download<double>(ctx, dlen, N);
    h.edge = mb_download<int>(ctx, dedge, 2 * (size_t)N);
    h.side = mb_download<double>(ctx, dside, (size_t)N * 2 * SIDE_STRIDE);
    h.locations = mb_download<double>(ctx, dloc, 3 * (size_t)N);
  } else {
    h.rwg.clear();
    h.len.clear();
    h.edge.clear();
    h.side.clear();
    h.locations.clear();
  }
  AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
}

std::vector<int> bin_points_gpu(aifmm_ctx* ctx, const std::vector<double>& pts, const std::vector<double>& centers,
                                int nLevels, std::vector<int>& leafStart) {
  const int n = (int)(pts.size() / 3);
  long nLeaves = 1;
  for (int j = 0; j < nLevels; ++j) nLeaves *= 8;
  AIFMM_REQUIRE(nLeaves < (1L << 31) && n > 0, AIFMM_EINVAL, "bad octree binning size");
  DevBuf dp = upload(ctx, pts), dc = upload(ctx, centers);
  DevBuf l0(ctx, sizeof(unsigned) * n), l1(ctx, sizeof(unsigned) * n), o0(ctx, sizeof(int) * n),
      o1(ctx, sizeof(int) * n);
  mb_bin_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(dp.as<double>(), n, dc.as<double>(), nLevels,
                                                           l0.as<unsigned>(), o0.as<int>());
  AIFMM_LAUNCHED();
  int bits = 1;
  while ((1L << bits) < nLeaves) ++bits;
  mb_sort(ctx, l0.as<unsigned>(), l1.as<unsigned>(), o0.as<int>(), o1.as<int>(), n, bits);
  std::vector<unsigned> leaf = mb_download<unsigned>(ctx, l1, n);
  std::vector<int> order = mb_download<int>(ctx, o1, n);
  AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
  leafStart.assign((size_t)nLeaves + 1, 0);
  for (int i = 0; i < n; ++i) leafStart[leaf[i] + 1]++;
  for (long k = 0; k < nLeaves; ++k) leafStart[k + 1] += leafStart[k];
  return order;
}

}  // namespace aifmm
