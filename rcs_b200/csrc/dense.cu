#include <map>
#include <tuple>
// Dense complex128 kernels: grouped SIMT GEMM (64x64 tiles, 4x4 complex
// micro-tiles per thread), blocked LU with a single-CTA panel, blocked
// triangular solves, batched copies and norms.
#include <algorithm>

#include "dense.cuh"
#include "dmat.cuh"

namespace aifmm {

// ------------------------------------------------------------------ GEMM
constexpr int GBM = 64, GBN = 64, GBK = 8;

__device__ __forceinline__ zd ldA(const GemmProblem& P, int i, int k) {
  if (i >= P.m || k >= P.k) return zmk(0, 0);
  if (P.opA == OP_N) return P.A[(size_t)k * P.lda + i];
  return zconj(P.A[(size_t)i * P.lda + k]);
}
__device__ __forceinline__ zd ldB(const GemmProblem& P, int k, int j) {
  if (k >= P.k || j >= P.n) return zmk(0, 0);
  if (P.opB == OP_N) return P.B[(size_t)j * P.ldb + k];
  return zconj(P.B[(size_t)k * P.ldb + j]);
}

// acc += op(A) op(B) over the 64x64 tile at (row0, col0).  K advances in
// slices of 16 through a three-stage shared-memory ring filled with
// cp.async (16-byte copies, zero-filled outside the matrix), so two slices
// are in flight while one is consumed; conjugation of op = C is applied when
// an element is read from shared memory.
constexpr int PBK = 16, PSTAGES = 3;
struct GemmSmem {
  zd A[PSTAGES][PBK][GBM];
  zd B[PSTAGES][PBK][GBN];
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Issue the copies of K slice kt into ring stage st: 1024 A and 1024 B
// elements, four of each per thread, consecutive threads along the operand's
// contiguous dimension.
__device__ __forceinline__ void gemm_load_slice(const GemmProblem& P, int row0, int col0, int kt, GemmSmem& S, int st) {
  const int k0 = kt * PBK;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int e = threadIdx.x + 256 * q;
    int i, k;
    if (P.opA == OP_N) { i = e & 63; k = e >> 6; }
    else { k = e & 15; i = e >> 4; }
    const int gi = row0 + i, gk = k0 + k;
    const bool ok = gi < P.m && gk < P.k;
    const zd* src = ok ? (P.opA == OP_N ? P.A + (size_t)gk * P.lda + gi : P.A + (size_t)gi * P.lda + gk) : P.A;
    cp_async16(&S.A[st][k][i], src, ok);
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int e = threadIdx.x + 256 * q;
    int j, k;
    if (P.opB == OP_N) { k = e & 15; j = e >> 4; }
    else { j = e & 63; k = e >> 6; }
    const int gj = col0 + j, gk = k0 + k;
    const bool ok = gj < P.n && gk < P.k;
    const zd* src = ok ? (P.opB == OP_N ? P.B + (size_t)gj * P.ldb + gk : P.B + (size_t)gk * P.ldb + gj) : P.B;
    cp_async16(&S.B[st][k][j], src, ok);
  }
}

__device__ __forceinline__ void gemm_tile_accumulate(const GemmProblem& P, int row0, int col0, zd (&acc)[4][4],
                                                     GemmSmem& S) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int nk = (P.k + PBK - 1) / PBK;
  const double sa = (P.opA == OP_N) ? 1.0 : -1.0, sb = (P.opB == OP_N) ? 1.0 : -1.0;  // imaginary sign
#pragma unroll
  for (int s = 0; s < PSTAGES - 1; ++s) {
    if (s < nk) gemm_load_slice(P, row0, col0, s, S, s);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<PSTAGES - 2>();  // slice kt has landed (this thread's copies)
    __syncthreads();               // ... and everyone's; stage of kt-1 is free
    const int nxt = kt + PSTAGES - 1;
    if (nxt < nk) gemm_load_slice(P, row0, col0, nxt, S, nxt % PSTAGES);
    cp_async_commit();
    const int st = kt % PSTAGES;
#pragma unroll
    for (int kk = 0; kk < PBK; ++kk) {
      zd a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a[i] = S.A[st][kk][tx + 16 * i];
        a[i].y *= sa;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        b[j] = S.B[st][kk][ty + 16 * j];
        b[j].y *= sb;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x = fma(a[i].x, b[j].x, acc[i][j].x);
          acc[i][j].x = fma(-a[i].y, b[j].y, acc[i][j].x);
          acc[i][j].y = fma(a[i].x, b[j].y, acc[i][j].y);
          acc[i][j].y = fma(a[i].y, b[j].x, acc[i][j].y);
        }
    }
  }
  cp_async_wait<0>();
  __syncthreads();  // the next chained problem reuses the ring
}

template <bool INLINE>
__global__ void __launch_bounds__(256, 2) zgemm_grouped_kernel(const __grid_constant__ GemmArgs a) {
  extern __shared__ unsigned char gemm_raw[];
  GemmSmem& S = *reinterpret_cast<GemmSmem*>(gemm_raw);
  const GemmGroup* G = INLINE ? a.ig : a.groups;
  const GemmProblem* probs = INLINE ? a.ip : a.probs;
  int lo = 0, hi = a.ngroups - 1;
  const int tile = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (G[mid].tileStart <= tile) lo = mid;
    else hi = mid - 1;
  }
  const GemmGroup g = G[lo];
  const int local = tile - g.tileStart;
  const int row0 = (local / g.tilesN) * GBM, col0 = (local % g.tilesN) * GBN;
  zd acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = zmk(0, 0);
  for (int q = 0; q < g.nchain; ++q)
    if (probs[g.head + q].k > 0) gemm_tile_accumulate(probs[g.head + q], row0, col0, acc, S);
  const GemmProblem& P = probs[g.head];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const bool beta0 = (P.beta.x == 0.0 && P.beta.y == 0.0);
  // each row's 4 C entries are loaded together before its stores, so an
  // accumulating tile waits for memory 4 times instead of 16 (a whole
  // micro-tile at once would spill: the kernel is at its register cap)
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = row0 + tx + 16 * i;
    if (r >= P.m) continue;
    zd cv[4];
    if (!beta0) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = col0 + ty + 16 * j;
        if (c < P.n) cv[j] = __ldcg(P.C + (size_t)c * P.ldc + r);
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = col0 + ty + 16 * j;
      if (c >= P.n) continue;
      zd v = zmul(P.alpha, acc[i][j]);
      if (!beta0) v = zadd(v, zmul(P.beta, cv[j]));
      P.C[(size_t)c * P.ldc + r] = v;
    }
  }
}

// ------------------------------------------------------------------ GEMM, split TF32
// Mixed-precision variant of the same grouped/chained GEMM on the tensor
// cores: every FP64 complex operand is rounded to FP32 and split into a TF32
// high part and a TF32 remainder, and each real product X Y is formed as
// Xh Yh + Xh Yl + Xl Yh with FP32 accumulation (~FP32 accuracy, not FP64).
// The complex product takes 12 m16n8k8 MMAs per k-step:
//   Cr += Ar Br - Ai Bi,  Ci += Ar Bi + Ai Br.
// Tile 64x64 complex, K slices of 16, 8 warps of 32x16; operands staged in
// shared memory as four TF32 planes (re/im x hi/lo), rows padded to 20 words
// so the fragment loads hit 32 distinct banks.
constexpr int TK = 16, TLD = TK + 4;

__device__ __forceinline__ uint32_t tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void tf32_split(double v, uint32_t& hi, uint32_t& lo) {
  const float f = (float)v;
  hi = tf32_round(f);
  lo = tf32_round(f - __uint_as_float(hi));
}
__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

struct TcSmem {
  uint32_t A[4][GBM * TLD];  // planes: re hi, re lo, im hi, im lo; [m][k]
  uint32_t B[4][GBN * TLD];  // same, [n][k]
};

// Element e (0..1023) of the 64x16 A slice and of the 16x64 B slice: the
// index mapping follows the operand's contiguous dimension.
__device__ __forceinline__ void tc_coords_A(const GemmProblem& P, int e, int& m, int& k) {
  if (P.opA == OP_N) { m = e & 63; k = e >> 6; }
  else { k = e & 15; m = e >> 4; }
}
__device__ __forceinline__ void tc_coords_B(const GemmProblem& P, int e, int& n, int& k) {
  if (P.opB == OP_N) { k = e & 15; n = e >> 4; }
  else { n = e & 63; k = e >> 6; }
}

__device__ __forceinline__ void tc_accumulate(const GemmProblem& P, int row0, int col0, float (&cr)[2][2][4],
                                              float (&ci)[2][2][4], TcSmem& S) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;
  zd ra[4], rb[4];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int m, k, n, kb;
      tc_coords_A(P, tid + 256 * q, m, k);
      ra[q] = ldA(P, row0 + m, k0 + k);
      tc_coords_B(P, tid + 256 * q, n, kb);
      rb[q] = ldB(P, k0 + kb, col0 + n);
    }
  };
  fetch(0);
  for (int k0 = 0; k0 < P.k; k0 += TK) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int m, k, n, kb;
      tc_coords_A(P, tid + 256 * q, m, k);
      tf32_split(ra[q].x, S.A[0][m * TLD + k], S.A[1][m * TLD + k]);
      tf32_split(ra[q].y, S.A[2][m * TLD + k], S.A[3][m * TLD + k]);
      tc_coords_B(P, tid + 256 * q, n, kb);
      tf32_split(rb[q].x, S.B[0][n * TLD + kb], S.B[1][n * TLD + kb]);
      tf32_split(rb[q].y, S.B[2][n * TLD + kb], S.B[3][n * TLD + kb]);
    }
    __syncthreads();
    if (k0 + TK < P.k) fetch(k0 + TK);
#pragma unroll
    for (int ks = 0; ks < TK; ks += 8) {
      uint32_t a[4][2][4];  // plane, m-tile, fragment
      uint32_t b[4][2][2];  // plane, n-tile, fragment
#pragma unroll
      for (int pl = 0; pl < 4; ++pl) {
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) {
          const uint32_t* base = S.A[pl] + (wm + mi * 16 + g) * TLD + ks + t;
          a[pl][mi][0] = base[0];
          a[pl][mi][1] = base[8 * TLD];
          a[pl][mi][2] = base[4];
          a[pl][mi][3] = base[8 * TLD + 4];
        }
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) {
          const uint32_t* base = S.B[pl] + (wn + ni * 8 + g) * TLD + ks + t;
          b[pl][ni][0] = base[0];
          b[pl][ni][1] = base[4];
        }
      }
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) {
          const uint32_t nbh0 = b[2][ni][0] ^ 0x80000000u, nbh1 = b[2][ni][1] ^ 0x80000000u;
          const uint32_t nbl0 = b[3][ni][0] ^ 0x80000000u, nbl1 = b[3][ni][1] ^ 0x80000000u;
          // Cr += Ar Br - Ai Bi
          mma_tf32(cr[mi][ni], a[0][mi], b[0][ni][0], b[0][ni][1]);
          mma_tf32(cr[mi][ni], a[0][mi], b[1][ni][0], b[1][ni][1]);
          mma_tf32(cr[mi][ni], a[1][mi], b[0][ni][0], b[0][ni][1]);
          mma_tf32(cr[mi][ni], a[2][mi], nbh0, nbh1);
          mma_tf32(cr[mi][ni], a[2][mi], nbl0, nbl1);
          mma_tf32(cr[mi][ni], a[3][mi], nbh0, nbh1);
          // Ci += Ar Bi + Ai Br
          mma_tf32(ci[mi][ni], a[0][mi], b[2][ni][0], b[2][ni][1]);
          mma_tf32(ci[mi][ni], a[0][mi], b[3][ni][0], b[3][ni][1]);
          mma_tf32(ci[mi][ni], a[1][mi], b[2][ni][0], b[2][ni][1]);
          mma_tf32(ci[mi][ni], a[2][mi], b[0][ni][0], b[0][ni][1]);
          mma_tf32(ci[mi][ni], a[2][mi], b[1][ni][0], b[1][ni][1]);
          mma_tf32(ci[mi][ni], a[3][mi], b[0][ni][0], b[0][ni][1]);
        }
    }
    __syncthreads();
  }
}

template <bool INLINE>
__global__ void __launch_bounds__(256) zgemm_tf32x3_kernel(const __grid_constant__ GemmArgs a) {
  __shared__ TcSmem S;
  const GemmGroup* G = INLINE ? a.ig : a.groups;
  const GemmProblem* probs = INLINE ? a.ip : a.probs;
  int lo = 0, hi = a.ngroups - 1;
  const int tile = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (G[mid].tileStart <= tile) lo = mid;
    else hi = mid - 1;
  }
  const GemmGroup g = G[lo];
  const int local = tile - g.tileStart;
  const int row0 = (local / g.tilesN) * GBM, col0 = (local % g.tilesN) * GBN;
  float cr[2][2][4], ci[2][2][4];
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 2; ++ni)
#pragma unroll
      for (int r = 0; r < 4; ++r) cr[mi][ni][r] = ci[mi][ni][r] = 0.f;
  for (int q = 0; q < g.nchain; ++q) tc_accumulate(probs[g.head + q], row0, col0, cr, ci, S);
  const GemmProblem& P = probs[g.head];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gr = lane >> 2, t = lane & 3;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;
  const bool beta0 = (P.beta.x == 0.0 && P.beta.y == 0.0);
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 2; ++ni)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int row = row0 + wm + mi * 16 + gr + ((r & 2) ? 8 : 0);
        const int col = col0 + wn + ni * 8 + 2 * t + (r & 1);
        if (row >= P.m || col >= P.n) continue;
        zd* cp = P.C + (size_t)col * P.ldc + row;
        zd v = zmul(P.alpha, zmk((double)cr[mi][ni][r], (double)ci[mi][ni][r]));
        if (!beta0) v = zadd(v, zmul(P.beta, *cp));
        *cp = v;
      }
}

// Optional per-launch timing of the grouped GEMM (events on the launching
// stream) for the roofline figure; off unless a caller enables it.
// Each record carries the path of the instrumented scopes it was issued
// from (opprof::path), so the time can be split by call site.
struct GemmProfile {
  bool on = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
  std::vector<std::string> tag;
  std::vector<double> fl;
  double flops = 0;
  long launches = 0;
};
static GemmProfile g_prof;

void gemm_profile_enable(bool on) {
  for (auto& e : g_prof.ev) {
    cudaEventDestroy(e.first);
    cudaEventDestroy(e.second);
  }
  g_prof = GemmProfile();
  g_prof.on = on;
}

bool gemm_profile_on() { return g_prof.on; }

void device_span_record(cudaEvent_t e0, cudaEvent_t e1, const std::string& tag, double flops) {
  g_prof.ev.push_back({e0, e1});
  g_prof.tag.push_back(tag);
  g_prof.fl.push_back(flops);
}

void gemm_profile_read(double* ms, double* flops, long* launches) {
  double t = 0;
  for (size_t i = 0; i < g_prof.ev.size(); ++i) {
    if (g_prof.tag[i].compare(0, 5, "gemm:") != 0) continue;
    auto& e = g_prof.ev[i];
    AIFMM_CUDA(cudaEventSynchronize(e.second));
    float x = 0;
    AIFMM_CUDA(cudaEventElapsedTime(&x, e.first, e.second));
    t += x;
  }
  *ms = t;
  *flops = g_prof.flops;
  *launches = g_prof.launches;
}

std::string gemm_profile_table() {
  std::map<std::string, std::tuple<long, double, double>> by;
  for (size_t i = 0; i < g_prof.ev.size(); ++i) {
    auto& e = g_prof.ev[i];
    AIFMM_CUDA(cudaEventSynchronize(e.second));
    float x = 0;
    AIFMM_CUDA(cudaEventElapsedTime(&x, e.first, e.second));
    auto& r = by[g_prof.tag[i]];
    std::get<0>(r)++;
    std::get<1>(r) += x;
    std::get<2>(r) += g_prof.fl[i];
  }
  std::string out;
  char line[512];
  for (auto& kv : by) {
    snprintf(line, sizeof(line), "%s %ld %.6f %.6e\n", kv.first.c_str(), std::get<0>(kv.second),
             std::get<1>(kv.second) / 1e3, std::get<2>(kv.second));
    out += line;
  }
  return out;
}

// ------------------------------------------------------------------ GEMM, skinny split-K
// Products with at most 16 columns (the solve sweeps: a box block times a few
// right-hand sides) are latency-bound in 64x64 tiles: one tile column, the K
// loop of a whole chain in a handful of CTAs.  Here every (32-row block,
// problem, K chunk of up to 512) is its own CTA: it stages its chunk of B in
// shared memory, its 8 warps split the chunk's depths (lane = row, so the
// loads of A are 512 contiguous bytes per warp, several in flight), and the
// warps' sums are added in a fixed order.  An output that one CTA covers
// (depth up to 512, no chain) is written with alpha and beta by that CTA;
// otherwise the CTAs write partial sums and a second kernel adds each
// output's partials in a fixed order (deterministic) and applies alpha, beta.
constexpr int SK_ROWS = 32, SK_KC = 512, SK_NR = 16;
struct SkItem {
  int prob, row0, k0, klen, slot;
};
struct SkOut {
  int head, row0, s0, ns;
};

// NR: columns held per thread (8 or 16, at least the launch's widest problem)
template <bool DIRECT, int NR>
__global__ void __launch_bounds__(256) zskinny_partial_kernel(const GemmProblem* __restrict__ probs,
                                                              const SkItem* __restrict__ items, zd* __restrict__ part,
                                                              int nmax) {
  extern __shared__ zd sk_b[];  // the item's chunk of B: depth kk, column r at sk_b[kk * nmax + r]
  __shared__ zd red[8][8][SK_ROWS];
  const SkItem it = items[blockIdx.x];
  const GemmProblem& P = probs[it.prob];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int row = it.row0 + lane;
  const bool live = row < P.m;
  const int n = P.n;
  for (int t = threadIdx.x; t < it.klen * n; t += blockDim.x) {
    const int kk = t % it.klen, r = t / it.klen;  // consecutive threads: consecutive depths of one column
    sk_b[kk * nmax + r] = P.B[(size_t)r * P.ldb + it.k0 + kk];
  }
  __syncthreads();
  zd acc[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) acc[r] = zmk(0, 0);
  const zd* A = P.A + (size_t)it.k0 * P.lda + (live ? row : 0);
  // 8 depths per warp in flight: each is a 512-byte row segment of A
#pragma unroll 8
  for (int kk = w; kk < it.klen; kk += 8) {
    const zd a = live ? A[(size_t)kk * P.lda] : zmk(0, 0);
    const zd* bk = sk_b + kk * nmax;
#pragma unroll
    for (int r = 0; r < NR; ++r)
      if (r < n) {
        const zd b = bk[r];
        acc[r].x = fma(a.x, b.x, acc[r].x);
        acc[r].x = fma(-a.y, b.y, acc[r].x);
        acc[r].y = fma(a.x, b.y, acc[r].y);
        acc[r].y = fma(a.y, b.x, acc[r].y);
      }
  }
  zd* out = part + (size_t)it.slot * SK_NR * SK_ROWS;
#pragma unroll
  for (int half = 0; half < NR / 8; ++half) {
#pragma unroll
    for (int r = 0; r < 8; ++r) red[w][r][lane] = acc[half * 8 + r];
    __syncthreads();
    const int r = threadIdx.x >> 5, l = threadIdx.x & 31;  // 8 columns x 32 rows
    zd sum = red[0][r][l];
#pragma unroll
    for (int q = 1; q < 8; ++q) sum = zadd(sum, red[q][r][l]);
    if (DIRECT) {
      const int c = half * 8 + r, rr = it.row0 + l;
      if (c < n && rr < P.m) {
        zd* cp = P.C + (size_t)c * P.ldc + rr;
        zd v = zmul(P.alpha, sum);
        if (!(P.beta.x == 0.0 && P.beta.y == 0.0)) v = zadd(v, zmul(P.beta, *cp));
        *cp = v;
      }
    } else {
      out[(size_t)(half * 8 + r) * SK_ROWS + l] = sum;
    }
    __syncthreads();
  }
}

__global__ void zskinny_reduce_kernel(const GemmProblem* __restrict__ probs, const SkOut* __restrict__ outs,
                                      const zd* __restrict__ part) {
  const SkOut o = outs[blockIdx.x];
  const GemmProblem& P = probs[o.head];
  const int l = threadIdx.x & 31, r = threadIdx.x >> 5;
  const int row = o.row0 + l;
  if (r >= P.n || row >= P.m) return;
  zd s = zmk(0, 0);
  for (int i = 0; i < o.ns; ++i) s = zadd(s, part[((size_t)(o.s0 + i) * SK_NR + r) * SK_ROWS + l]);
  zd* cp = P.C + (size_t)r * P.ldc + row;
  zd v = zmul(P.alpha, s);
  if (!(P.beta.x == 0.0 && P.beta.y == 0.0)) v = zadd(v, zmul(P.beta, *cp));
  *cp = v;
}

static bool skinny_eligible(const std::vector<GemmProblem>& probs) {
  bool any = false;
  for (const GemmProblem& p : probs) {
    if (p.m <= 0 || p.n <= 0) continue;
    if (p.n > SK_NR || p.opA != OP_N || p.opB != OP_N) return false;
    any = true;
  }
  return any;
}

static void zgemm_skinny_chained(aifmm_ctx* ctx, const std::vector<GemmProblem>& probs, const std::vector<int>& chain) {
  std::vector<GemmProblem> ps;
  std::vector<SkItem> items;
  std::vector<SkOut> outs;
  int slots = 0;
  for (size_t i = 0; i < probs.size();) {
    const int len = chain[i];
    const GemmProblem& h = probs[i];
    if (h.m > 0 && h.n > 0) {
      const int head = (int)ps.size();
      for (int q = 0; q < len; ++q) ps.push_back(probs[i + q]);
      for (int r0 = 0; r0 < h.m; r0 += SK_ROWS) {
        SkOut o{head, r0, slots, 0};
        for (int q = 0; q < len; ++q) {
          const GemmProblem& p = probs[i + q];
          for (int k0 = 0; k0 < p.k; k0 += SK_KC) {
            items.push_back({head + q, r0, k0, std::min(SK_KC, p.k - k0), slots++});
            o.ns++;
          }
        }
        outs.push_back(o);
      }
    }
    i += len;
  }
  if (outs.empty()) return;
  int nmax = 1;
  bool direct = true;  // every output covered by one CTA
  for (const GemmProblem& p : ps) nmax = std::max(nmax, p.n);
  for (const SkOut& o : outs) direct = direct && o.ns == 1;
  const size_t smem = sizeof(zd) * (size_t)SK_KC * nmax;
  // one instantiation per (direct, columns per thread)
  auto kernel = [&](bool d) -> void (*)(const GemmProblem*, const SkItem*, zd*, int) {
    if (nmax <= 8) return d ? zskinny_partial_kernel<true, 8> : zskinny_partial_kernel<false, 8>;
    return d ? zskinny_partial_kernel<true, 16> : zskinny_partial_kernel<false, 16>;
  };
  smem_attr_once((const void*)kernel(direct), ctx->device, (int)(sizeof(zd) * SK_KC * SK_NR));
  DevBuf dp = upload(ctx, ps), di = upload(ctx, items);
  if (direct) {
    kernel(true)<<<(unsigned)items.size(), 256, smem, ctx->stream>>>(dp.as<GemmProblem>(), di.as<SkItem>(), nullptr,
                                                                     nmax);
    AIFMM_LAUNCHED();
    return;
  }
  DevBuf dout = upload(ctx, outs);
  DevBuf part(ctx, sizeof(zd) * (size_t)std::max(slots, 1) * SK_NR * SK_ROWS);
  if (!items.empty()) {
    kernel(false)<<<(unsigned)items.size(), 256, smem, ctx->stream>>>(dp.as<GemmProblem>(), di.as<SkItem>(),
                                                                      part.as<zd>(), nmax);
    AIFMM_LAUNCHED();
  }
  zskinny_reduce_kernel<<<(unsigned)outs.size(), SK_ROWS * SK_NR, 0, ctx->stream>>>(dp.as<GemmProblem>(),
                                                                                   dout.as<SkOut>(), part.as<zd>());
  AIFMM_LAUNCHED();
}

static void zgemm_chained_dispatch(aifmm_ctx* ctx, const std::vector<GemmProblem>& probs,
                                   const std::vector<int>& chain);

// ---- split-K for FP64 launches with few output tiles and long depths
// (the Gram-Schmidt projections Q^H F of the recompressions: a few dozen
// 64 x 64 tiles over depths of 500-2,000).  Every chain's depth is cut into S
// ranges that become separate chains writing partial sums into a workspace;
// a second kernel adds the partials in a fixed order (deterministic) and
// applies alpha and beta.
struct SplitOut {
  zd* C;
  int m, n, ldc, parts;
  zd alpha, beta;
  long part0;  // first element of this chain's partials in the workspace
};

__global__ void zsplitk_reduce_kernel(const SplitOut* __restrict__ outs, const long* __restrict__ start, int nouts,
                                      long total, const zd* __restrict__ work) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nouts - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (start[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    const SplitOut& O = outs[lo];
    const long u = t - start[lo];
    const int r = (int)(u % O.m), c = (int)(u / O.m);
    const long mn = (long)O.m * O.n;
    zd acc = work[O.part0 + u];
    for (int s = 1; s < O.parts; ++s) acc = zadd(acc, work[O.part0 + (long)s * mn + u]);
    zd* cp = O.C + (size_t)c * O.ldc + r;
    zd v = zmul(O.alpha, acc);
    if (O.beta.x != 0.0 || O.beta.y != 0.0) v = zadd(v, zmul(O.beta, *cp));
    *cp = v;
  }
}

// true when the FP64 launch fills under a third of the SMs with long depths
static bool splitk_wanted(aifmm_ctx* ctx, const std::vector<GemmProblem>& probs, const std::vector<int>& chain) {
  long tiles = 0, depth = 0, chains = 0;
  for (size_t i = 0; i < probs.size();) {
    const GemmProblem& h = probs[i];
    long k = 0;
    for (int q = 0; q < chain[i]; ++q) k += std::max(probs[i + q].k, 0);
    if (h.m > 0 && h.n > 0) {
      tiles += (long)((h.m + GBM - 1) / GBM) * ((h.n + GBN - 1) / GBN);
      depth = std::max(depth, k);
      chains++;
    }
    i += chain[i];
  }
  const int sms = ctx->numSMs > 0 ? ctx->numSMs : 148;
  return chains > 0 && tiles * 3 <= sms && depth >= 384;
}

static void zgemm_splitk(aifmm_ctx* ctx, const std::vector<GemmProblem>& probs, const std::vector<int>& chain) {
  const int sms = ctx->numSMs > 0 ? ctx->numSMs : 148;
  long tiles = 0;
  for (size_t i = 0; i < probs.size(); i += chain[i])
    if (probs[i].m > 0 && probs[i].n > 0)
      tiles += (long)((probs[i].m + GBM - 1) / GBM) * ((probs[i].n + GBN - 1) / GBN);
  const int S = (int)std::max(2L, std::min(16L, (2L * sms + tiles - 1) / std::max(tiles, 1L)));
  std::vector<GemmProblem> ps;
  std::vector<int> ch;
  std::vector<long> woff;  // workspace offset of each piece's partial
  std::vector<SplitOut> outs;
  long work = 0;
  for (size_t i = 0; i < probs.size(); i += chain[i]) {
    const GemmProblem& h = probs[i];
    if (h.m <= 0 || h.n <= 0) continue;
    long K = 0;
    for (int q = 0; q < chain[i]; ++q) K += std::max(probs[i + q].k, 0);
    const int parts = (int)std::max(1L, std::min((long)S, K / 128));
    const long kc = (K + parts - 1) / parts;
    const long mn = (long)h.m * h.n;
    outs.push_back({h.C, h.m, h.n, h.ldc, parts, h.alpha, h.beta, work});
    for (int s = 0; s < parts; ++s) {
      const long lo = s * kc, hi = std::min(K, lo + kc);
      // the pieces of the chain's problems that fall in [lo, hi)
      std::vector<GemmProblem> piece;
      long base = 0;
      for (int q = 0; q < chain[i]; ++q) {
        const GemmProblem& p = probs[i + q];
        const long a = std::max(lo, base), b = std::min(hi, base + std::max(p.k, 0));
        if (a < b) {
          GemmProblem x = p;
          const long k0 = a - base;
          x.k = (int)(b - a);
          x.A = (p.opA == OP_N) ? p.A + k0 * p.lda : p.A + k0;
          x.B = (p.opB == OP_N) ? p.B + k0 : p.B + k0 * p.ldb;
          piece.push_back(x);
        }
        base += std::max(p.k, 0);
      }
      if (piece.empty()) {  // an empty range: a zero product keeps the partial defined
        GemmProblem x = h;
        x.k = 0;
        piece.push_back(x);
      }
      for (size_t q = 0; q < piece.size(); ++q) {
        GemmProblem x = piece[q];
        x.C = nullptr;  // set below, once the workspace exists
        x.ldc = h.m;
        x.alpha = zmk(1, 0);
        x.beta = q == 0 ? zmk(0, 0) : zmk(1, 0);
        woff.push_back(work + s * mn);
        ps.push_back(x);
        ch.push_back(q == 0 ? (int)piece.size() : 0);
      }
    }
    work += (long)parts * mn;
  }
  DevBuf ws(ctx, sizeof(zd) * std::max(work, 1L));
  for (size_t q = 0; q < ps.size(); ++q) ps[q].C = ws.as<zd>() + woff[q];
  zgemm_chained_dispatch(ctx, ps, ch);
  std::vector<long> start;
  long total = 0;
  for (const SplitOut& o : outs) {
    start.push_back(total);
    total += (long)o.m * o.n;
  }
  DevBuf dout = upload(ctx, outs), dst = upload(ctx, start);
  const int grid = (int)std::min<long>((total + 255) / 256, 148L * 16);
  zsplitk_reduce_kernel<<<grid, 256, 0, ctx->stream>>>(dout.as<SplitOut>(), dst.as<long>(), (int)outs.size(), total,
                                                       ws.as<zd>());
  AIFMM_LAUNCHED();
}

void zgemm_chained(aifmm_ctx* ctx, const std::vector<GemmProblem>& probs, const std::vector<int>& chain) {
  AIFMM_REQUIRE(probs.size() == chain.size(), AIFMM_EINVAL, "chain lengths do not match the problems");
  if (ctx->gemmPrecision == 0 && ctx->splitK && !skinny_eligible(probs) && splitk_wanted(ctx, probs, chain)) {
    zgemm_splitk(ctx, probs, chain);
    return;
  }
  zgemm_chained_dispatch(ctx, probs, chain);
}

// One launch of the kernel the context's GEMM precision selects.
static void zgemm_chained_dispatch(aifmm_ctx* ctx, const std::vector<GemmProblem>& probs,
                                   const std::vector<int>& chain) {
  std::vector<GemmProblem> ps;
  std::vector<GemmGroup> gs;
  long tiles = 0;
  double flops = 0;
  const int mode = ctx->gemmPrecision;
  if (mode == 5) {
    zgemm_tuned(ctx, probs, chain);
    return;
  }
  const int bm = (mode >= 2) ? 128 : GBM;  // row tile of the tcgen05 kernels
  const int bn = (mode == 4) ? 128 : GBN;  // complex columns per tile
  for (size_t i = 0; i < probs.size();) {
    const int len = chain[i];
    AIFMM_REQUIRE(len >= 1 && i + len <= probs.size(), AIFMM_EINVAL, "bad chain length");
    const GemmProblem& h = probs[i];
    for (int q = 1; q < len; ++q) {
      const GemmProblem& p = probs[i + q];
      AIFMM_REQUIRE(p.C == h.C && p.m == h.m && p.n == h.n && p.ldc == h.ldc && p.alpha.x == h.alpha.x &&
                        p.alpha.y == h.alpha.y && p.beta.x == 1.0 && p.beta.y == 0.0,
                    AIFMM_EINVAL, "chained GEMMs must share C, shape and alpha, with beta 1 after the first");
    }
    if (h.m > 0 && h.n > 0) {
      GemmGroup g;
      g.head = (int)ps.size();
      g.nchain = len;
      g.tilesN = (h.n + bn - 1) / bn;
      g.tileStart = (int)tiles;
      for (int q = 0; q < len; ++q) {
        ps.push_back(probs[i + q]);
        flops += 8.0 * probs[i + q].m * (double)probs[i + q].n * std::max(probs[i + q].k, 0);
      }
      gs.push_back(g);
      tiles += (long)((h.m + bm - 1) / bm) * g.tilesN;
    }
    i += len;
  }
  if (gs.empty()) return;
  if (skinny_eligible(probs)) {
    zgemm_skinny_chained(ctx, probs, chain);
    return;
  }
  AIFMM_REQUIRE(tiles < (long)INT32_MAX, AIFMM_EOVERFLOW, "too many GEMM tiles");
  static_assert(sizeof(GemmArgs) < 32000, "GEMM arguments exceed the kernel parameter space");
  GemmArgs a;
  a.ngroups = (int)gs.size();
  a.probs = nullptr;
  a.groups = nullptr;
  tc_wait_args(ctx, a);
  DevBuf dp, dg;
  const bool inl = gs.size() <= (size_t)GEMM_INLINE && ps.size() <= (size_t)GEMM_INLINE;
  if (inl) {
    std::copy(ps.begin(), ps.end(), a.ip);
    std::copy(gs.begin(), gs.end(), a.ig);
  } else {
    dp = upload(ctx, ps);
    dg = upload(ctx, gs);
    a.probs = dp.as<GemmProblem>();
    a.groups = dg.as<GemmGroup>();
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (g_prof.on) {
    AIFMM_CUDA(cudaEventCreate(&e0));
    AIFMM_CUDA(cudaEventCreate(&e1));
    AIFMM_CUDA(cudaEventRecord(e0, ctx->stream));
  }
  if (mode == 4) {
    zgemm_tc6(ctx, ps, gs);
  } else if (mode == 3) {
    zgemm_tc5p(ctx, ps, gs, tiles);
  } else if (mode == 2) {
    zgemm_tc5_launch(ctx, a, inl, tiles);
  } else if (mode == 1) {
    if (inl) zgemm_tf32x3_kernel<true><<<(unsigned)tiles, 256, 0, ctx->stream>>>(a);
    else zgemm_tf32x3_kernel<false><<<(unsigned)tiles, 256, 0, ctx->stream>>>(a);
  } else {
    smem_attr_once((const void*)zgemm_grouped_kernel<true>, ctx->device, (int)sizeof(GemmSmem));
    smem_attr_once((const void*)zgemm_grouped_kernel<false>, ctx->device, (int)sizeof(GemmSmem));
    if (inl) zgemm_grouped_kernel<true><<<(unsigned)tiles, 256, sizeof(GemmSmem), ctx->stream>>>(a);
    else zgemm_grouped_kernel<false><<<(unsigned)tiles, 256, sizeof(GemmSmem), ctx->stream>>>(a);
  }
  AIFMM_LAUNCHED();
  if (g_prof.on) {
    AIFMM_CUDA(cudaEventRecord(e1, ctx->stream));
    device_span_record(e0, e1, "gemm:" + std::to_string(mode) + ":" + opprof::path(), flops);
    g_prof.flops += flops;
    g_prof.launches++;
  }
}

void zgemm_grouped(aifmm_ctx* ctx, const std::vector<GemmProblem>& probs) {
  zgemm_chained(ctx, probs, std::vector<int>(probs.size(), 1));
}

// ------------------------------------------------------------------ copies
constexpr int COPY_INLINE = 128;
struct CopyArgs {
  int nprob;
  long total;
  const CopyProblem* probs;
  const long* start;
  CopyProblem ip[COPY_INLINE];
  long is[COPY_INLINE];
};

template <bool INLINE>
__global__ void zcopy_grouped_kernel(const __grid_constant__ CopyArgs a) {
  const CopyProblem* probs = INLINE ? a.ip : a.probs;
  const long* start = INLINE ? a.is : a.start;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < a.total; t += (long)gridDim.x * blockDim.x) {
    int lo = 0, hi = a.nprob - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (start[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    const CopyProblem& P = probs[lo];
    const long u = t - start[lo];
    const int i = (int)(u % P.rows), j = (int)(u / P.rows);
    zd v = zmk(0, 0);  // src == nullptr: zero fill
    if (P.src) v = zmul(P.scale, P.conjTrans ? zconj(P.src[(size_t)i * P.lds + j]) : P.src[(size_t)j * P.lds + i]);
    zd* d = P.dst + (size_t)j * P.ldd + i;
    *d = P.accumulate ? zadd(*d, v) : v;
  }
}

void zcopy_grouped(aifmm_ctx* ctx, const std::vector<CopyProblem>& probs) {
  std::vector<CopyProblem> ps;
  std::vector<long> start;
  long total = 0;
  for (const CopyProblem& p : probs) {
    if (p.rows <= 0 || p.cols <= 0) continue;
    ps.push_back(p);
    start.push_back(total);
    total += (long)p.rows * p.cols;
  }
  if (ps.empty()) return;
  static_assert(sizeof(CopyArgs) < 32000, "copy arguments exceed the kernel parameter space");
  CopyArgs a;
  a.nprob = (int)ps.size();
  a.total = total;
  a.probs = nullptr;
  a.start = nullptr;
  const int grid = (int)std::min<long>((total + 255) / 256, 148L * 32);
  if (ps.size() <= (size_t)COPY_INLINE) {
    std::copy(ps.begin(), ps.end(), a.ip);
    std::copy(start.begin(), start.end(), a.is);
    zcopy_grouped_kernel<true><<<grid, 256, 0, ctx->stream>>>(a);
  } else {
    DevBuf dp = upload(ctx, ps), ds = upload(ctx, start);
    a.probs = dp.as<CopyProblem>();
    a.start = ds.as<long>();
    zcopy_grouped_kernel<false><<<grid, 256, 0, ctx->stream>>>(a);
  }
  AIFMM_LAUNCHED();
}

__global__ void zfill_kernel(zd* p, size_t n, zd v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}
void zfill(aifmm_ctx* ctx, zd* p, size_t n, zd v) {
  if (n == 0) return;
  const int grid = (int)std::min<size_t>((n + 255) / 256, 148 * 32);
  zfill_kernel<<<grid, 256, 0, ctx->stream>>>(p, n, v);
  AIFMM_LAUNCHED();
}

__global__ void zident_kernel(zd* p, int rows, int cols, zd diag) {
  const size_t n = (size_t)rows * cols;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % rows), j = (int)(t / rows);
    p[t] = (i == j) ? diag : zmk(0, 0);
  }
}
void zset_identity(aifmm_ctx* ctx, zd* p, int rows, int cols, zd diag) {
  const size_t n = (size_t)rows * cols;
  if (n == 0) return;
  const int grid = (int)std::min<size_t>((n + 255) / 256, 148 * 32);
  zident_kernel<<<grid, 256, 0, ctx->stream>>>(p, rows, cols, diag);
  AIFMM_LAUNCHED();
}

// ------------------------------------------------------------------ norms
__global__ void znorm_kernel(const NormProblem* __restrict__ probs, double* out) {
  const NormProblem P = probs[blockIdx.x];
  double s = 0.0;
  const size_t n = (size_t)P.rows * P.cols;
  for (size_t t = threadIdx.x; t < n; t += blockDim.x) {
    const int i = (int)(t % P.rows), j = (int)(t / P.rows);
    s += zabs2(P.p[(size_t)j * P.ld + i]);
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffff, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = (threadIdx.x < blockDim.x / 32) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffff, s, o);
    if (threadIdx.x == 0) out[blockIdx.x] = sqrt(s);
  }
}
void znorm_grouped(aifmm_ctx* ctx, const std::vector<NormProblem>& probs, double* out_dev) {
  if (probs.empty()) return;
  DevBuf dp = upload(ctx, probs);
  znorm_kernel<<<(unsigned)probs.size(), 256, 0, ctx->stream>>>(dp.as<NormProblem>(), out_dev);
  AIFMM_LAUNCHED();
}

// ------------------------------------------------------------------ LU
constexpr int LU_NB = 32;

// Factor columns [j0, j0+nb) of the n x n matrix: pivot search over the whole
// column below the diagonal (largest |a|, lowest row on ties), full-row
// swaps, division by the pivot, rank-1 update inside the panel.
__global__ void __launch_bounds__(1024) zgetrf_panel_kernel(zd* A, int n, int lda, int j0, int nb, int* piv,
                                                             int* info) {
  __shared__ double sv[32];
  __shared__ int si[32];
  __shared__ int s_p;
  __shared__ zd s_piv;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int k = j0; k < j0 + nb; ++k) {
    // pivot search
    double best = -1.0;
    int bi = n;
    for (int i = k + tid; i < n; i += nt) {
      const double v = hypot(A[(size_t)k * lda + i].x, A[(size_t)k * lda + i].y);
      if (v > best) { best = v; bi = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffff, best, o);
      const int oi = __shfl_xor_sync(0xffffffff, bi, o);
      if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
    }
    if ((tid & 31) == 0) { sv[tid >> 5] = best; si[tid >> 5] = bi; }
    __syncthreads();
    if (tid < 32) {
      best = (tid < (nt >> 5)) ? sv[tid] : -1.0;
      bi = (tid < (nt >> 5)) ? si[tid] : n;
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffff, best, o);
        const int oi = __shfl_xor_sync(0xffffffff, bi, o);
        if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
      }
      if (tid == 0) {
        s_p = (best > 0.0) ? bi : -1;
        piv[k] = (best > 0.0) ? bi : k;
        if (best <= 0.0 && *info == 0) *info = k + 1;
      }
    }
    __syncthreads();
    const int p = s_p;
    if (p >= 0 && p != k)
      for (int j = tid; j < n; j += nt) {
        zd a = A[(size_t)j * lda + k];
        A[(size_t)j * lda + k] = A[(size_t)j * lda + p];
        A[(size_t)j * lda + p] = a;
      }
    __syncthreads();
    if (tid == 0) s_piv = A[(size_t)k * lda + k];
    __syncthreads();
    if (p >= 0)
      for (int i = k + 1 + tid; i < n; i += nt) A[(size_t)k * lda + i] = zdiv(A[(size_t)k * lda + i], s_piv);
    __syncthreads();
    // rank-1 update of the remaining panel columns
    const int ncol = j0 + nb - k - 1, nrow = n - k - 1;
    for (int t = tid; t < ncol * nrow; t += nt) {
      const int i = k + 1 + t % nrow, j = k + 1 + t / nrow;
      A[(size_t)j * lda + i] = zsub(A[(size_t)j * lda + i], zmul(A[(size_t)k * lda + i], A[(size_t)j * lda + k]));
    }
    __syncthreads();
  }
}

// X <- T^{-1} X for a triangular nb x nb block T (unit lower or non-unit
// upper) and X = nb rows x ncols columns; one thread per column, launched
// kTrsmThreads to a CTA so that a box's few hundred columns spread over as
// many SMs.
constexpr int kTrsmThreads = 32;
template <bool LOWER_UNIT>
__global__ void ztrsm_block_kernel(const zd* __restrict__ T, int ldt, int nb, zd* X, int ldx, int ncols) {
  __shared__ zd Ts[LU_NB * LU_NB];
  for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) Ts[t] = T[(size_t)(t / nb) * ldt + (t % nb)];
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncols) return;
  zd x[LU_NB];
#pragma unroll
  for (int i = 0; i < LU_NB; ++i)
    if (i < nb) x[i] = X[(size_t)c * ldx + i];
  if (LOWER_UNIT) {
#pragma unroll
    for (int i = 0; i < LU_NB; ++i) {
      if (i >= nb) break;
#pragma unroll
      for (int l = 0; l < LU_NB; ++l)
        if (l < i) x[i] = zsub(x[i], zmul(Ts[l * nb + i], x[l]));
    }
  } else {
#pragma unroll
    for (int i = LU_NB - 1; i >= 0; --i) {
      if (i >= nb) continue;
#pragma unroll
      for (int l = 0; l < LU_NB; ++l)
        if (l > i && l < nb) x[i] = zsub(x[i], zmul(Ts[l * nb + i], x[l]));
      x[i] = zdiv(x[i], Ts[i * nb + i]);
    }
  }
#pragma unroll
  for (int i = 0; i < LU_NB; ++i)
    if (i < nb) X[(size_t)c * ldx + i] = x[i];
}

__global__ void zlaswp_kernel(zd* B, int ldb, int nrhs, const int* __restrict__ piv, int n) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nrhs) return;
  zd* b = B + (size_t)c * ldb;
  for (int k = 0; k < n; ++k) {
    const int p = piv[k];
    if (p != k) {
      zd t = b[k];
      b[k] = b[p];
      b[p] = t;
    }
  }
}

// The row interchanges of an LU solve as one gather per column: every CTA
// first composes the n interchanges into the permutation src (row i of the
// result is row src[i] of the input: the swaps replayed in order on an index
// array in shared memory), then each warp copies its column through shared
// memory.  The same result as applying the swaps one by one, without one
// thread walking n dependent swaps per column.
__global__ void zlaswp_perm_kernel(zd* B, int ldb, int nrhs, const int* __restrict__ piv, int n) {
  extern __shared__ __align__(16) unsigned char laswp_sm[];
  int* src = reinterpret_cast<int*>(laswp_sm);
  int* pv = src + n;
  zd* buf = reinterpret_cast<zd*>(laswp_sm + (((size_t)2 * n * sizeof(int) + 15) & ~(size_t)15));
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    src[i] = i;
    pv[i] = piv[i];
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < n; ++k) {
      const int p = pv[k];
      if (p != k) {
        const int t = src[k];
        src[k] = src[p];
        src[p] = t;
      }
    }
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int c = blockIdx.x * nw + w;
  if (c >= nrhs) return;
  zd* b = B + (size_t)c * ldb;
  zd* t = buf + (size_t)w * n;
  for (int i = lane; i < n; i += 32) t[i] = b[src[i]];
  __syncwarp();
  for (int i = lane; i < n; i += 32) b[i] = t[i];
}

static void zlaswp(aifmm_ctx* ctx, zd* B, int ldb, int nrhs, const int* piv, int n) {
  constexpr size_t kSmemMax = 200 * 1024;
  const size_t idx = ((size_t)2 * n * sizeof(int) + 15) & ~(size_t)15;
  const size_t perWarp = sizeof(zd) * (size_t)n;
  const int warps = (int)std::min<size_t>(8, idx + perWarp <= kSmemMax ? (kSmemMax - idx) / perWarp : 0);
  if (warps == 0) {  // a column does not fit in shared memory: the swaps one by one
    zlaswp_kernel<<<ceil_div(nrhs, 128), 128, 0, ctx->stream>>>(B, ldb, nrhs, piv, n);
    AIFMM_LAUNCHED();
    return;
  }
  smem_attr_once((const void*)zlaswp_perm_kernel, ctx->device, (int)kSmemMax);
  zlaswp_perm_kernel<<<ceil_div(nrhs, warps), 32 * warps, idx + perWarp * warps, ctx->stream>>>(B, ldb, nrhs, piv, n);
  AIFMM_LAUNCHED();
}

void zgetrf(aifmm_ctx* ctx, zd* A, int n, int lda, int* piv, int* info) {
  if (n <= 0) return;
  AIFMM_CUDA(cudaMemsetAsync(info, 0, sizeof(int), ctx->stream));
  for (int j0 = 0; j0 < n; j0 += LU_NB) {
    const int nb = std::min(LU_NB, n - j0);
    zgetrf_panel_kernel<<<1, 1024, 0, ctx->stream>>>(A, n, lda, j0, nb, piv, info);
    AIFMM_LAUNCHED();
    const int rest = n - j0 - nb;
    if (rest <= 0) continue;
    // U12 = L11^{-1} A12
    ztrsm_block_kernel<true><<<ceil_div(rest, kTrsmThreads), kTrsmThreads, 0, ctx->stream>>>(A + (size_t)j0 * lda + j0, lda, nb,
                                                                           A + (size_t)(j0 + nb) * lda + j0, lda,
                                                                           rest);
    AIFMM_LAUNCHED();
    // A22 -= L21 U12
    GemmProblem g{A + (size_t)j0 * lda + j0 + nb, A + (size_t)(j0 + nb) * lda + j0, A + (size_t)(j0 + nb) * lda + j0 + nb,
                  rest, rest, nb, lda, lda, lda, OP_N, OP_N, zmk(-1, 0), zmk(1, 0)};
    zgemm_grouped(ctx, {g});
  }
}

// Whole solve for a few right-hand sides in one CTA: B staged in shared
// memory (n x nrhs, ld n), row interchanges, then forward (unit lower) and
// backward (upper) substitution in 32-row blocks -- a warp per right-hand
// side solves the diagonal block with lane = row, then all threads update
// the remaining rows, thread = (row, column).
constexpr int GS_NT = 256;
constexpr size_t GS_SMEM_MAX = 200 * 1024;

__global__ void __launch_bounds__(GS_NT) zgetrs_smem_kernel(const zd* __restrict__ LU, int n, int lda,
                                                            const int* __restrict__ piv, zd* B, int nrhs, int ldb) {
  extern __shared__ zd xs[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int t = tid; t < n * nrhs; t += GS_NT) xs[t] = B[(size_t)(t / n) * ldb + (t % n)];
  __syncthreads();
  if (tid < nrhs) {
    zd* x = xs + (size_t)tid * n;
    for (int k = 0; k < n; ++k) {
      const int p = piv[k];
      if (p != k) {
        const zd t = x[k];
        x[k] = x[p];
        x[p] = t;
      }
    }
  }
  __syncthreads();
  for (int b0 = 0; b0 < n; b0 += 32) {  // forward, unit lower
    const int nb = min(32, n - b0);
    for (int c = warp; c < nrhs; c += GS_NT / 32) {
      zd* x = xs + (size_t)c * n + b0;
      zd xi = lane < nb ? x[lane] : zmk(0, 0);
      for (int l = 0; l < nb; ++l) {
        zd xl;
        xl.x = __shfl_sync(0xffffffff, xi.x, l);
        xl.y = __shfl_sync(0xffffffff, xi.y, l);
        if (lane > l && lane < nb) xi = zsub(xi, zmul(LU[(size_t)(b0 + l) * lda + b0 + lane], xl));
      }
      if (lane < nb) x[lane] = xi;
    }
    __syncthreads();
    const int r0 = b0 + nb, rest = n - r0;
    for (int t = tid; t < rest * nrhs; t += GS_NT) {
      const int i = r0 + t % rest, c = t / rest;
      const zd* xb = xs + (size_t)c * n + b0;
      zd s = zmk(0, 0);
      for (int l = 0; l < nb; ++l) s = zadd(s, zmul(LU[(size_t)(b0 + l) * lda + i], xb[l]));
      xs[(size_t)c * n + i] = zsub(xs[(size_t)c * n + i], s);
    }
    __syncthreads();
  }
  for (int b0 = ((n - 1) / 32) * 32; b0 >= 0; b0 -= 32) {  // backward, upper
    const int nb = min(32, n - b0);
    for (int c = warp; c < nrhs; c += GS_NT / 32) {
      zd* x = xs + (size_t)c * n + b0;
      zd xi = lane < nb ? x[lane] : zmk(0, 0);
      for (int l = nb - 1; l >= 0; --l) {
        if (lane == l) xi = zdiv(xi, LU[(size_t)(b0 + l) * lda + b0 + l]);
        zd xl;
        xl.x = __shfl_sync(0xffffffff, xi.x, l);
        xl.y = __shfl_sync(0xffffffff, xi.y, l);
        if (lane < l) xi = zsub(xi, zmul(LU[(size_t)(b0 + l) * lda + b0 + lane], xl));
      }
      if (lane < nb) x[lane] = xi;
    }
    __syncthreads();
    for (int t = tid; t < b0 * nrhs; t += GS_NT) {
      const int i = t % b0, c = t / b0;
      const zd* xb = xs + (size_t)c * n + b0;
      zd s = zmk(0, 0);
      for (int l = 0; l < nb; ++l) s = zadd(s, zmul(LU[(size_t)(b0 + l) * lda + i], xb[l]));
      xs[(size_t)c * n + i] = zsub(xs[(size_t)c * n + i], s);
    }
    __syncthreads();
  }
  for (int t = tid; t < n * nrhs; t += GS_NT) B[(size_t)(t / n) * ldb + (t % n)] = xs[t];
}

void zgetrs(aifmm_ctx* ctx, const zd* LU, int n, int lda, const int* piv, zd* B, int nrhs, int ldb) {
  if (n <= 0 || nrhs <= 0) return;
  const size_t smem = sizeof(zd) * (size_t)n * nrhs;
  if (nrhs <= 16 && smem <= GS_SMEM_MAX) {
    smem_attr_once((const void*)zgetrs_smem_kernel, ctx->device, (int)GS_SMEM_MAX);
    zgetrs_smem_kernel<<<1, GS_NT, smem, ctx->stream>>>(LU, n, lda, piv, B, nrhs, ldb);
    AIFMM_LAUNCHED();
    return;
  }
  zlaswp(ctx, B, ldb, nrhs, piv, n);
  // forward: unit lower
  for (int i0 = 0; i0 < n; i0 += LU_NB) {
    const int nb = std::min(LU_NB, n - i0);
    ztrsm_block_kernel<true><<<ceil_div(nrhs, kTrsmThreads), kTrsmThreads, 0, ctx->stream>>>(LU + (size_t)i0 * lda + i0, lda, nb,
                                                                           B + i0, ldb, nrhs);
    AIFMM_LAUNCHED();
    const int rest = n - i0 - nb;
    if (rest > 0) {
      GemmProblem g{LU + (size_t)i0 * lda + i0 + nb, B + i0, B + i0 + nb, rest, nrhs, nb, lda, ldb, ldb, OP_N, OP_N,
                    zmk(-1, 0), zmk(1, 0)};
      zgemm_grouped(ctx, {g});
    }
  }
  // backward: upper
  const int last = ((n - 1) / LU_NB) * LU_NB;
  for (int i0 = last; i0 >= 0; i0 -= LU_NB) {
    const int nb = std::min(LU_NB, n - i0);
    ztrsm_block_kernel<false><<<ceil_div(nrhs, kTrsmThreads), kTrsmThreads, 0, ctx->stream>>>(LU + (size_t)i0 * lda + i0, lda, nb,
                                                                            B + i0, ldb, nrhs);
    AIFMM_LAUNCHED();
    if (i0 > 0) {
      GemmProblem g{LU + (size_t)i0 * lda, B + i0, B, i0, nrhs, nb, lda, ldb, ldb, OP_N, OP_N, zmk(-1, 0),
                    zmk(1, 0)};
      zgemm_grouped(ctx, {g});
    }
  }
}

}  // namespace aifmm
