// Split-TF32 complex grouped GEMM on the fifth-generation tensor cores
// (tcgen05): the same chained problem lists as zgemm_grouped, 128x64 complex
// tiles, one CTA of eight warps per tile.
//
// Each K slice of 16 complex values (two MMA k-steps of 8) is staged by all
// threads: FP64 operands are rounded to FP32 and split into a TF32 high part
// and a TF32 remainder, real and imaginary parts in separate planes, written
// in the no-swizzle K-major core-matrix layout (8 rows x 16 bytes per core
// matrix, K-adjacent cores 128 bytes apart, 8-row groups 256 bytes apart).
// One thread issues the slice's 24 MMAs of 128x64x8 (twelve per k-step) into
// two FP32 accumulators in tensor memory (Cr: columns 0..63, Ci: 64..127):
//   Cr += Ar Br - Ai Bi,  Ci += Ar Bi + Ai Br,  each product hi*hi + hi*lo + lo*hi,
// the subtraction by the instruction's negate-B bit, and commits them to the
// stage's mbarrier; the slice after next waits on that barrier before reusing
// the stage (double buffering).  The epilogue reads the accumulators with
// tcgen05.ld (warp w: rows 32 (w % 4).., columns 32 (w / 4)..) and applies
// alpha, beta in FP64.
//
// Every wait is bounded (one second of GPU time); a wait that runs out leaves
// its tile unwritten, counts a timeout and waits once more, bounded, for the
// MMAs in flight before freeing tensor memory.
#include <algorithm>

#include "dense.cuh"

namespace aifmm {

constexpr int C5_M = 128, C5_N = 64, C5_K = 8, C5_KS = 16;  // MMA k-step, staged slice
constexpr int C5_THREADS = 256;
constexpr uint32_t C5_TMEM_COLS = 128;
constexpr unsigned long long C5_WAIT_NS = 1000000000ull;

struct C5Stage {
  uint32_t A[4][C5_KS / C5_K][C5_M * C5_K];  // plane (re hi, re lo, im hi, im lo), k-step, core layout
  uint32_t B[4][C5_KS / C5_K][C5_N * C5_K];
};
struct C5Smem {
  C5Stage st[2];
  unsigned long long bar[2];
  uint32_t tmem_slot;
};

__device__ unsigned long long g_c5_timeouts;

// Word offset of (row, k) in the no-swizzle K-major canonical layout.
__device__ __forceinline__ int c5_off(int row, int k) { return (row >> 3) * 64 + (k >> 2) * 32 + (row & 7) * 4 + (k & 3); }

__device__ __forceinline__ uint32_t c5_smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start >> 4, LBO 128 B, SBO 256 B,
// descriptor version 1, base offset 0, no swizzle.
__device__ __forceinline__ uint64_t c5_desc(const void* p) {
  uint64_t d = (uint64_t)((c5_smem_addr(p) >> 4) & 0x3FFF);
  d |= (uint64_t)(128 >> 4) << 16;
  d |= (uint64_t)(256 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B, both
// K-major, N = 64, M = 128, optional negation of B.
__host__ __device__ constexpr uint32_t c5_idesc(bool negB) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((negB ? 1u : 0u) << 14) | ((uint32_t)(C5_N >> 3) << 17) |
         ((uint32_t)(C5_M >> 4) << 24);
}

__device__ __forceinline__ void c5_mma(uint32_t d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void c5_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(c5_smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ unsigned long long c5_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for the completion of the barrier phase with the given parity; false
// if that takes longer than C5_WAIT_NS.
__device__ __forceinline__ bool c5_wait(unsigned long long* bar, uint32_t parity,
                                        unsigned long long limit = C5_WAIT_NS) {
  const uint32_t a = c5_smem_addr(bar);
  const unsigned long long t0 = c5_now();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (c5_now() - t0 > limit) return false;
  }
}
// Bounded wait until *flag != 0 (the wait test's hold flag).
__device__ __forceinline__ bool c5_hold(const int* flag, unsigned long long limit) {
  const unsigned long long t0 = c5_now();
  while (*(const volatile int*)flag == 0)
    if (c5_now() - t0 > limit) return false;
  return true;
}

__device__ __forceinline__ uint32_t c5_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void c5_split(double v, uint32_t* hi, uint32_t* lo, int off) {
  const float f = (float)v;
  const uint32_t h = c5_tf32(f);
  hi[off] = h;
  lo[off] = c5_tf32(f - __uint_as_float(h));
}

__device__ __forceinline__ zd c5_ldA(const GemmProblem& P, int i, int k) {
  if (i >= P.m || k >= P.k) return zmk(0, 0);
  if (P.opA == OP_N) return P.A[(size_t)k * P.lda + i];
  return zconj(P.A[(size_t)i * P.lda + k]);
}
__device__ __forceinline__ zd c5_ldB(const GemmProblem& P, int k, int j) {
  if (k >= P.k || j >= P.n) return zmk(0, 0);
  if (P.opB == OP_N) return P.B[(size_t)j * P.ldb + k];
  return zconj(P.B[(size_t)k * P.ldb + j]);
}
// Element e of the 128x16 A slice / 16x64 B slice.  A warp covers 8 rows x 4
// k values of one core-matrix group, so its 32 shared-memory stores hit 32
// distinct banks (word (row % 8) * 4 + k % 4); along the operand's contiguous
// dimension it reads runs of 8 (m or n) or 4 (k) complex values.
__device__ __forceinline__ void c5_coordA(int opA, int e, int& m, int& k) {
  const int lane = e & 31, wid = e >> 5;  // wid: 0..63
  if (opA == OP_N) { m = (wid & 15) * 8 + (lane & 7); k = (wid >> 4) * 4 + (lane >> 3); }
  else { m = (wid & 15) * 8 + (lane >> 2); k = (wid >> 4) * 4 + (lane & 3); }
}
__device__ __forceinline__ void c5_coordB(int opB, int e, int& n, int& k) {
  const int lane = e & 31, wid = e >> 5;  // wid: 0..31
  if (opB == OP_N) { n = (wid & 7) * 8 + (lane >> 2); k = (wid >> 3) * 4 + (lane & 3); }
  else { n = (wid & 7) * 8 + (lane & 7); k = (wid >> 3) * 4 + (lane >> 3); }
}

template <bool INLINE>
__global__ void __launch_bounds__(C5_THREADS, 2) zgemm_tc5_kernel(const __grid_constant__ GemmArgs a) {
  extern __shared__ unsigned char c5_raw[];
  C5Smem& S = *reinterpret_cast<C5Smem*>((reinterpret_cast<uintptr_t>(c5_raw) + 1023) & ~uintptr_t(1023));
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
  const int row0 = (local / g.tilesN) * C5_M, col0 = (local % g.tilesN) * C5_N;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(c5_smem_addr(&S.tmem_slot)),
                 "r"(C5_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(c5_smem_addr(&S.bar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(c5_smem_addr(&S.bar[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = S.tmem_slot;

  uint32_t phase[2] = {0, 0};
  int it = 0;
  bool ok = true, crInit = false, ciInit = false;
  if (a.hold) {  // the wait test's hold: before any MMA, so nothing is in flight if it runs out
    bool mine = true;
    if (tid == 0) mine = c5_hold(a.hold, a.waitNs);
    ok = __syncthreads_and(mine);
  }
  for (int q = 0; q < g.nchain && ok; ++q) {
    const GemmProblem& P = probs[g.head + q];
    if (P.k <= 0) continue;
    zd ra[8], rb[4];  // 2048 A and 1024 B elements per slice over 256 threads
    auto fetch = [&](int k0) {
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        int m, k;
        c5_coordA(P.opA, tid + C5_THREADS * r, m, k);
        ra[r] = c5_ldA(P, row0 + m, k0 + k);
      }
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        int n, k;
        c5_coordB(P.opB, tid + C5_THREADS * r, n, k);
        rb[r] = c5_ldB(P, k0 + k, col0 + n);
      }
    };
    fetch(0);
    for (int k0 = 0; k0 < P.k; k0 += C5_KS) {
      const int s = it & 1;
      if (it >= 2) {  // the MMAs that read this stage two slices ago must be done
        bool mine = true;
        if (tid == 0) mine = c5_wait(&S.bar[s], phase[s], a.waitNs);
        ok = __syncthreads_and(mine);
        phase[s] ^= 1;
        if (!ok) break;
      }
      C5Stage& st = S.st[s];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        int m, k;
        c5_coordA(P.opA, tid + C5_THREADS * r, m, k);
        const int ks = k >> 3, o = c5_off(m, k & 7);
        c5_split(ra[r].x, st.A[0][ks], st.A[1][ks], o);
        c5_split(ra[r].y, st.A[2][ks], st.A[3][ks], o);
      }
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        int n, k;
        c5_coordB(P.opB, tid + C5_THREADS * r, n, k);
        const int ks = k >> 3, o = c5_off(n, k & 7);
        c5_split(rb[r].x, st.B[0][ks], st.B[1][ks], o);
        c5_split(rb[r].y, st.B[2][ks], st.B[3][ks], o);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        constexpr uint32_t ip = c5_idesc(false), in = c5_idesc(true);
        const uint32_t dr = tmem, di = tmem + C5_N;
#pragma unroll
        for (int ks = 0; ks < C5_KS / C5_K; ++ks) {
          const uint64_t dA[4] = {c5_desc(st.A[0][ks]), c5_desc(st.A[1][ks]), c5_desc(st.A[2][ks]),
                                  c5_desc(st.A[3][ks])};
          const uint64_t dB[4] = {c5_desc(st.B[0][ks]), c5_desc(st.B[1][ks]), c5_desc(st.B[2][ks]),
                                  c5_desc(st.B[3][ks])};
          // Cr += Ar Br - Ai Bi
          c5_mma(dr, dA[0], dB[0], ip, (crInit || ks) ? 1u : 0u);
          c5_mma(dr, dA[0], dB[1], ip, 1u);
          c5_mma(dr, dA[1], dB[0], ip, 1u);
          c5_mma(dr, dA[2], dB[2], in, 1u);
          c5_mma(dr, dA[2], dB[3], in, 1u);
          c5_mma(dr, dA[3], dB[2], in, 1u);
          // Ci += Ar Bi + Ai Br
          c5_mma(di, dA[0], dB[2], ip, (ciInit || ks) ? 1u : 0u);
          c5_mma(di, dA[0], dB[3], ip, 1u);
          c5_mma(di, dA[1], dB[2], ip, 1u);
          c5_mma(di, dA[2], dB[0], ip, 1u);
          c5_mma(di, dA[2], dB[1], ip, 1u);
          c5_mma(di, dA[3], dB[0], ip, 1u);
        }
        c5_commit(&S.bar[s]);
      }
      crInit = ciInit = true;
      if (k0 + C5_KS < P.k) fetch(k0 + C5_KS);
      ++it;
    }
  }
  if (ok && it > 0) {  // the last commit covers every MMA issued before it
    const int s = (it - 1) & 1;
    bool mine = true;
    if (tid == 0) mine = c5_wait(&S.bar[s], phase[s], a.waitNs);
    ok = __syncthreads_and(mine);
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const GemmProblem& P = probs[g.head];
  if (ok) {
    // warp w reads tensor-memory lanes 32 (w % 4) .. +31 (its rows) and columns
    // 32 (w / 4) .. +31 of both accumulators
    const int quarter = warp & 3, half = warp >> 2;
    const int row = row0 + quarter * 32 + lane;
    const bool beta0 = (P.beta.x == 0.0 && P.beta.y == 0.0);
    for (int c0 = half * 32; c0 < half * 32 + 32; c0 += 16) {
      uint32_t vr[16], vi[16];
      if (it > 0) {
        const uint32_t ta = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(vr[0]), "=r"(vr[1]), "=r"(vr[2]), "=r"(vr[3]), "=r"(vr[4]), "=r"(vr[5]), "=r"(vr[6]), "=r"(vr[7]),
              "=r"(vr[8]), "=r"(vr[9]), "=r"(vr[10]), "=r"(vr[11]), "=r"(vr[12]), "=r"(vr[13]), "=r"(vr[14]),
              "=r"(vr[15])
            : "r"(ta));
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(vi[0]), "=r"(vi[1]), "=r"(vi[2]), "=r"(vi[3]), "=r"(vi[4]), "=r"(vi[5]), "=r"(vi[6]), "=r"(vi[7]),
              "=r"(vi[8]), "=r"(vi[9]), "=r"(vi[10]), "=r"(vi[11]), "=r"(vi[12]), "=r"(vi[13]), "=r"(vi[14]),
              "=r"(vi[15])
            : "r"(ta + C5_N));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) vr[j] = vi[j] = 0u;
      }
      if (row < P.m) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = col0 + c0 + j;
          if (col >= P.n) break;
          zd* cp = P.C + (size_t)col * P.ldc + row;
          zd v = zmul(P.alpha, zmk((double)__uint_as_float(vr[j]), (double)__uint_as_float(vi[j])));
          if (!beta0) v = zadd(v, zmul(P.beta, *cp));
          *cp = v;
        }
      }
    }
  } else if (tid == 0) {
    atomicAdd(&g_c5_timeouts, 1ull);
    if (it > 0) c5_wait(&S.bar[(it - 1) & 1], phase[(it - 1) & 1]);  // bounded: MMAs still in flight
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C5_TMEM_COLS) : "memory");
}

void zgemm_tc5_launch(aifmm_ctx* ctx, const GemmArgs& a, bool inl, long tiles) {
  const size_t smem = sizeof(C5Smem) + 1024;
  smem_attr_once((const void*)zgemm_tc5_kernel<true>, ctx->device, (int)smem);
  smem_attr_once((const void*)zgemm_tc5_kernel<false>, ctx->device, (int)smem);
  if (inl) zgemm_tc5_kernel<true><<<(unsigned)tiles, C5_THREADS, smem, ctx->stream>>>(a);
  else zgemm_tc5_kernel<false><<<(unsigned)tiles, C5_THREADS, smem, ctx->stream>>>(a);
  AIFMM_LAUNCHED();
}

long zgemm_tc5_timeouts() {
  unsigned long long v = 0;
  AIFMM_CUDA(cudaMemcpyFromSymbol(&v, g_c5_timeouts, sizeof(v)));
  return (long)v;
}

}  // namespace aifmm
