// Split-TF32 complex grouped GEMM on the tcgen05 tensor cores with the
// operands converted once, outside the tile loop.
//
// Converting FP64 operands inside the GEMM (zgemm_tc5.cu) repeats the split
// for every output tile that reads an operand tile and leaves the tensor pipe
// mostly idle.  Here a conversion kernel first writes, for every problem,
// op(A) as 128-row x 16-k chunks and op(B) as 64-row x 16-k chunks: each chunk
// holds the four TF32 planes (re hi, re lo, im hi, im lo) of two 8-wide
// k-steps in the no-swizzle K-major core-matrix layout that the MMA reads
// (32 KB for A, 16 KB for B, zero-padded at the edges).  The GEMM CTA then
// only moves bytes: one thread copies each K slice's two chunks into a
// four-stage shared-memory ring with bulk copies completing on the slot's
// "full" barrier, issues the slice's 24 MMAs of 128x64x8 into the FP32
// accumulators Cr (tensor-memory columns 0..63) and Ci (64..127) as in
// zgemm_tc5.cu, and commits them to the slot's "empty" barrier; the slot of
// the previous slice is refilled once its MMAs have completed.  Four warps
// read the accumulators back (tcgen05.ld, warp w: rows 32w..32w+31) and apply
// alpha, beta in FP64.  Every wait is bounded (one second); a wait that runs
// out leaves the tile unwritten and is counted (zgemm_tc5p_timeouts()).
#include <algorithm>
#include <map>

#include "dense.cuh"

namespace aifmm {

constexpr int P5_M = 128, P5_N = 64, P5_KS = 16, P5_STAGES = 4, P5_THREADS = 128;
constexpr uint32_t P5_TMEM_COLS = 128;
constexpr uint32_t P5_A_BYTES = 4 * 2 * P5_M * 8 * 4, P5_B_BYTES = 4 * 2 * P5_N * 8 * 4;  // 32 KB, 16 KB
constexpr unsigned long long P5_WAIT_NS = 1000000000ull;

struct P5Stage {
  uint32_t A[4][2][P5_M * 8];
  uint32_t B[4][2][P5_N * 8];
};
struct P5Smem {
  P5Stage st[P5_STAGES];
  unsigned long long full[P5_STAGES], empty[P5_STAGES];
  uint32_t tmem_slot;
  int ok;
};

__device__ unsigned long long g_p5_timeouts;

__device__ __forceinline__ uint32_t p5_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ int p5_off(int row, int k) { return (row >> 3) * 64 + (k >> 2) * 32 + (row & 7) * 4 + (k & 3); }

__device__ __forceinline__ uint64_t p5_desc(const void* p) {
  uint64_t d = (uint64_t)((p5_smem(p) >> 4) & 0x3FFF);
  d |= (uint64_t)(128 >> 4) << 16;  // LBO: K-adjacent core matrices
  d |= (uint64_t)(256 >> 4) << 32;  // SBO: 8-row groups
  d |= (uint64_t)1 << 46;           // descriptor version
  return d;
}
__host__ __device__ constexpr uint32_t p5_idesc(bool negB) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((negB ? 1u : 0u) << 14) | ((uint32_t)(P5_N >> 3) << 17) |
         ((uint32_t)(P5_M >> 4) << 24);
}
__device__ __forceinline__ void p5_mma(uint32_t d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ unsigned long long p5_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool p5_wait(unsigned long long* bar, uint32_t parity,
                                        unsigned long long limit = P5_WAIT_NS) {
  const uint32_t a = p5_smem(bar);
  const unsigned long long t0 = p5_now();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (p5_now() - t0 > limit) return false;
  }
}
// Bounded wait until *flag != 0 (the wait test's hold flag).
__device__ __forceinline__ bool p5_hold(const int* flag, unsigned long long limit) {
  const unsigned long long t0 = p5_now();
  while (*(const volatile int*)flag == 0)
    if (p5_now() - t0 > limit) return false;
  return true;
}
// Bulk copies of slice `it` into ring slot s, completing on full[s].
__device__ __forceinline__ void p5_load(P5Smem& S, int s, const uint32_t* ga, const uint32_t* gb) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(p5_smem(&S.full[s])),
               "r"(P5_A_BYTES + P5_B_BYTES)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          p5_smem(&S.st[s].A[0][0][0])),
      "l"(ga), "r"(P5_A_BYTES), "r"(p5_smem(&S.full[s]))
      : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          p5_smem(&S.st[s].B[0][0][0])),
      "l"(gb), "r"(P5_B_BYTES), "r"(p5_smem(&S.full[s]))
      : "memory");
}

// ---------------------------------------------------------------- conversion
struct P5Operand {
  const zd* src;
  uint32_t* dst;
  int rows, k, ld, op, isB;  // logical rows (M of op(A), N of op(B)) x k
  int nks;                   // k slices of 16
};

__device__ __forceinline__ uint32_t p5_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// One thread per padded element (row, k) of every operand; consecutive
// threads walk the operand's contiguous dimension.
__global__ void p5_convert_kernel(const P5Operand* __restrict__ ops, const long* __restrict__ start, int nops,
                                  long total) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nops - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (start[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    const P5Operand& O = ops[lo];
    const long u = t - start[lo];
    const int tileRows = O.isB ? P5_N : P5_M;
    const int prow = ((O.rows + tileRows - 1) / tileRows) * tileRows, pk = O.nks * P5_KS;
    // row-fastest when the storage is contiguous along rows (op(A) = A, op(B) = B^H), else k-fastest
    const bool rowFast = O.isB ? (O.op == OP_C) : (O.op == OP_N);
    int r, k;
    if (rowFast) { r = (int)(u % prow); k = (int)(u / prow); }
    else { k = (int)(u % pk); r = (int)(u / pk); }
    zd v = zmk(0, 0);
    if (r < O.rows && k < O.k) {
      if (!O.isB) v = (O.op == OP_N) ? O.src[(size_t)k * O.ld + r] : zconj(O.src[(size_t)r * O.ld + k]);
      else v = (O.op == OP_N) ? O.src[(size_t)r * O.ld + k] : zconj(O.src[(size_t)k * O.ld + r]);
    }
    const int tr = r / tileRows, ks = k / P5_KS, kk = k % P5_KS;
    const size_t chunkWords = (size_t)4 * 2 * tileRows * 8;
    uint32_t* c = O.dst + ((size_t)tr * O.nks + ks) * chunkWords;
    const size_t planeWords = (size_t)2 * tileRows * 8;
    const int off = (kk >> 3) * tileRows * 8 + p5_off(r % tileRows, kk & 7);
    const float fr = (float)v.x, fi = (float)v.y;
    const uint32_t hr = p5_tf32(fr), hi2 = p5_tf32(fi);
    c[off] = hr;
    c[planeWords + off] = p5_tf32(fr - __uint_as_float(hr));
    c[2 * planeWords + off] = hi2;
    c[3 * planeWords + off] = p5_tf32(fi - __uint_as_float(hi2));
  }
}

// ---------------------------------------------------------------- GEMM
template <bool INLINE>
__global__ void __launch_bounds__(P5_THREADS, 1) zgemm_tc5p_kernel(const __grid_constant__ GemmArgs a) {
  extern __shared__ unsigned char p5_raw[];
  P5Smem& S = *reinterpret_cast<P5Smem*>((reinterpret_cast<uintptr_t>(p5_raw) + 1023) & ~uintptr_t(1023));
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
  const int tm = local / g.tilesN, tn = local % g.tilesN;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(p5_smem(&S.tmem_slot)),
                 "r"(P5_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < P5_STAGES; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(p5_smem(&S.full[s])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(p5_smem(&S.empty[s])) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    S.ok = 1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = S.tmem_slot;

  // slices of the whole chain: problem q contributes nks(q) slices
  int total = 0;
  for (int q = 0; q < g.nchain; ++q) total += (probs[g.head + q].k + P5_KS - 1) / P5_KS;

  if (tid == 0 && total > 0) {
    auto src = [&](int it, const uint32_t*& pa, const uint32_t*& pb) {
      int q = 0, base = 0;
      for (;; ++q) {
        const int n = (probs[g.head + q].k + P5_KS - 1) / P5_KS;
        if (it < base + n) break;
        base += n;
      }
      const GemmProblem& P = probs[g.head + q];
      const int nks = (P.k + P5_KS - 1) / P5_KS, ks = it - base;
      pa = P.pa + ((size_t)tm * nks + ks) * (P5_A_BYTES / 4);
      pb = P.pb + ((size_t)tn * nks + ks) * (P5_B_BYTES / 4);
    };
    uint32_t fph[P5_STAGES] = {0, 0, 0, 0}, eph[P5_STAGES] = {0, 0, 0, 0};
    bool loaded[P5_STAGES] = {false, false, false, false};  // a copy whose full phase is not consumed yet
    const unsigned long long lim = a.waitNs;
    // the wait test's hold comes before any copy, so nothing is in flight if it runs out
    bool ok = !(a.hold && !p5_hold(a.hold, lim));
    const int pre = ok ? min(total, P5_STAGES) : 0;
    for (int it = 0; it < pre; ++it) {
      const uint32_t *pa, *pb;
      src(it, pa, pb);
      p5_load(S, it, pa, pb);
      loaded[it] = true;
    }
    constexpr uint32_t ip = p5_idesc(false), in = p5_idesc(true);
    const uint32_t dr = tmem, di = tmem + P5_N;
    int issuedLoads = pre, lastCommit = -1;
    for (int it = 0; it < total && ok; ++it) {
      const int s = it % P5_STAGES;
      if (!p5_wait(&S.full[s], fph[s], lim)) { ok = false; break; }
      fph[s] ^= 1;
      loaded[s] = false;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      P5Stage& st = S.st[s];
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        const uint64_t dA[4] = {p5_desc(st.A[0][ks]), p5_desc(st.A[1][ks]), p5_desc(st.A[2][ks]), p5_desc(st.A[3][ks])};
        const uint64_t dB[4] = {p5_desc(st.B[0][ks]), p5_desc(st.B[1][ks]), p5_desc(st.B[2][ks]), p5_desc(st.B[3][ks])};
        const uint32_t first = (it == 0 && ks == 0) ? 0u : 1u;
        // Cr += Ar Br - Ai Bi ; Ci += Ar Bi + Ai Br (hi*hi + hi*lo + lo*hi each)
        p5_mma(dr, dA[0], dB[0], ip, first);
        p5_mma(dr, dA[0], dB[1], ip, 1u);
        p5_mma(dr, dA[1], dB[0], ip, 1u);
        p5_mma(dr, dA[2], dB[2], in, 1u);
        p5_mma(dr, dA[2], dB[3], in, 1u);
        p5_mma(dr, dA[3], dB[2], in, 1u);
        p5_mma(di, dA[0], dB[2], ip, first);
        p5_mma(di, dA[0], dB[3], ip, 1u);
        p5_mma(di, dA[1], dB[2], ip, 1u);
        p5_mma(di, dA[2], dB[0], ip, 1u);
        p5_mma(di, dA[2], dB[1], ip, 1u);
        p5_mma(di, dA[3], dB[0], ip, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       p5_smem(&S.empty[s]))
                   : "memory");
      lastCommit = it;
      // refill the previous slice's slot once its MMAs are done
      if (it >= 1 && issuedLoads < total) {
        const int sp = (it - 1) % P5_STAGES;
        if (!p5_wait(&S.empty[sp], eph[sp], lim)) { ok = false; break; }
        eph[sp] ^= 1;
        const uint32_t *pa, *pb;
        src(issuedLoads, pa, pb);
        p5_load(S, sp, pa, pb);
        loaded[sp] = true;
        ++issuedLoads;
      }
    }
    if (ok) {  // the last commit covers every MMA
      const int sl = (total - 1) % P5_STAGES;
      // slots whose empty phase was already consumed by a refill wait are not waited again
      ok = p5_wait(&S.empty[sl], eph[sl], lim);
    } else {
      // drain before the tile is abandoned: the MMAs of the last commit (they
      // read shared memory and write tensor memory) and every copy in flight,
      // each wait bounded by the normal limit
      if (lastCommit >= 0) p5_wait(&S.empty[lastCommit % P5_STAGES], eph[lastCommit % P5_STAGES]);
      for (int s = 0; s < P5_STAGES; ++s)
        if (loaded[s]) p5_wait(&S.full[s], fph[s]);
    }
    if (!ok) {
      atomicAdd(&g_p5_timeouts, 1ull);
      S.ok = 0;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const GemmProblem& P = probs[g.head];
  if (S.ok) {
    const int row = tm * P5_M + warp * 32 + lane;
    const bool beta0 = (P.beta.x == 0.0 && P.beta.y == 0.0);
    for (int c0 = 0; c0 < P5_N; c0 += 16) {
      uint32_t vr[16], vi[16];
      if (total > 0) {
        const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
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
            : "r"(ta + P5_N));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) vr[j] = vi[j] = 0u;
      }
      if (row < P.m) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = tn * P5_N + c0 + j;
          if (col >= P.n) break;
          zd* cp = P.C + (size_t)col * P.ldc + row;
          zd v = zmul(P.alpha, zmk((double)__uint_as_float(vr[j]), (double)__uint_as_float(vi[j])));
          if (!beta0) v = zadd(v, zmul(P.beta, *cp));
          *cp = v;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P5_TMEM_COLS) : "memory");
}

namespace {
// An operand as the conversion sees it; problems that read the same matrix
// the same way share its planes.
struct P5Key {
  const zd* src;
  int ld, op, rows, k, isB;
  bool operator<(const P5Key& o) const {
    if (src != o.src) return src < o.src;
    if (ld != o.ld) return ld < o.ld;
    if (op != o.op) return op < o.op;
    if (rows != o.rows) return rows < o.rows;
    if (k != o.k) return k < o.k;
    return isB < o.isB;
  }
};
size_t p5_words(const P5Key& key) {
  const int tr = key.isB ? P5_N : P5_M;
  const int nks = std::max(1, (key.k + P5_KS - 1) / P5_KS);
  return (size_t)((key.rows + tr - 1) / tr) * nks * (key.isB ? P5_B_BYTES : P5_A_BYTES) / 4;
}
constexpr size_t P5_PLANE_BUDGET = (size_t)4 << 30;  // bytes of planes per launch
}  // namespace

// Converts the distinct operands of a run of groups and launches their tiles.
static void p5_launch(aifmm_ctx* ctx, const std::vector<GemmProblem>& all, const std::vector<GemmGroup>& gs, size_t g0,
                      size_t g1) {
  std::map<P5Key, size_t> where;  // operand -> word offset of its planes
  size_t words = 0;
  std::vector<GemmProblem> ps;
  std::vector<GemmGroup> groups;
  long tiles = 0;
  for (size_t gi = g0; gi < g1; ++gi) {
    GemmGroup g = gs[gi];
    const int head = (int)ps.size();
    for (int q = 0; q < g.nchain; ++q) {
      GemmProblem p = all[g.head + q];
      const P5Key ka{p.A, p.lda, p.opA, p.m, p.k, 0}, kb{p.B, p.ldb, p.opB, p.n, p.k, 1};
      for (const P5Key& key : {ka, kb})
        if (!where.count(key)) {
          where[key] = words;
          words += p5_words(key);
        }
      ps.push_back(p);
    }
    const int nrt = (all[g.head].m + P5_M - 1) / P5_M;
    g.head = head;
    g.tileStart = (int)tiles;
    tiles += (long)nrt * g.tilesN;
    groups.push_back(g);
  }
  DevBuf planes(ctx, sizeof(uint32_t) * std::max<size_t>(words, 4));
  uint32_t* base = planes.as<uint32_t>();
  std::vector<P5Operand> ops;
  std::vector<long> start;
  long total = 0;
  for (const auto& kv : where) {
    const P5Key& key = kv.first;
    if (key.k <= 0) continue;
    const int nks = (key.k + P5_KS - 1) / P5_KS, tr = key.isB ? P5_N : P5_M;
    ops.push_back({key.src, base + kv.second, key.rows, key.k, key.ld, key.op, key.isB, nks});
    start.push_back(total);
    total += (long)((key.rows + tr - 1) / tr) * tr * (nks * P5_KS);
  }
  for (GemmProblem& p : ps) {
    p.pa = base + where[P5Key{p.A, p.lda, p.opA, p.m, p.k, 0}];
    p.pb = base + where[P5Key{p.B, p.ldb, p.opB, p.n, p.k, 1}];
  }
  if (total > 0) {
    DevBuf dops = upload(ctx, ops), dst = upload(ctx, start);
    const int grid = (int)std::min<long>((total + 255) / 256, 148L * 32);
    p5_convert_kernel<<<grid, 256, 0, ctx->stream>>>(dops.as<P5Operand>(), dst.as<long>(), (int)ops.size(), total);
    AIFMM_LAUNCHED();
  }
  if (tiles <= 0) return;
  AIFMM_REQUIRE(tiles < (long)INT32_MAX, AIFMM_EOVERFLOW, "too many GEMM tiles");
  GemmArgs a;
  a.ngroups = (int)groups.size();
  a.probs = nullptr;
  a.groups = nullptr;
  tc_wait_args(ctx, a);
  DevBuf dp, dg;
  const bool inl = groups.size() <= (size_t)GEMM_INLINE && ps.size() <= (size_t)GEMM_INLINE;
  if (inl) {
    std::copy(ps.begin(), ps.end(), a.ip);
    std::copy(groups.begin(), groups.end(), a.ig);
  } else {
    dp = upload(ctx, ps);
    dg = upload(ctx, groups);
    a.probs = dp.as<GemmProblem>();
    a.groups = dg.as<GemmGroup>();
  }
  const size_t smem = sizeof(P5Smem) + 1024;
  smem_attr_once((const void*)zgemm_tc5p_kernel<true>, ctx->device, (int)smem);
  smem_attr_once((const void*)zgemm_tc5p_kernel<false>, ctx->device, (int)smem);
  if (inl) zgemm_tc5p_kernel<true><<<(unsigned)tiles, P5_THREADS, smem, ctx->stream>>>(a);
  else zgemm_tc5p_kernel<false><<<(unsigned)tiles, P5_THREADS, smem, ctx->stream>>>(a);
  AIFMM_LAUNCHED();
}

// Groups are launched in runs whose distinct operands fit the plane budget
// (a group larger than the budget runs alone).
void zgemm_tc5p(aifmm_ctx* ctx, std::vector<GemmProblem> ps, const std::vector<GemmGroup>& gs, long) {
  size_t g0 = 0;
  while (g0 < gs.size()) {
    std::map<P5Key, bool> seen;
    size_t bytes = 0, g1 = g0;
    while (g1 < gs.size()) {
      size_t add = 0;
      std::vector<P5Key> fresh;
      for (int q = 0; q < gs[g1].nchain; ++q) {
        const GemmProblem& p = ps[gs[g1].head + q];
        for (const P5Key& key : {P5Key{p.A, p.lda, p.opA, p.m, p.k, 0}, P5Key{p.B, p.ldb, p.opB, p.n, p.k, 1}})
          if (!seen.count(key)) {
            bool dup = false;
            for (const P5Key& f : fresh) dup = dup || !(f < key || key < f);
            if (!dup) {
              fresh.push_back(key);
              add += 4 * p5_words(key);
            }
          }
      }
      if (g1 > g0 && bytes + add > P5_PLANE_BUDGET) break;
      for (const P5Key& f : fresh) seen[f] = true;
      bytes += add;
      ++g1;
    }
    p5_launch(ctx, ps, gs, g0, g1);
    g0 = g1;
  }
}

long zgemm_tc5p_timeouts() {
  unsigned long long v = 0;
  AIFMM_CUDA(cudaMemcpyFromSymbol(&v, g_p5_timeouts, sizeof(v)));
  return (long)v;
}

long tc_timeouts() { return zgemm_tc5_timeouts() + zgemm_tc5p_timeouts() + zgemm_tc6_timeouts(); }

void tc_check(long before, const char* what) {
  const long now = tc_timeouts();
  if (now > before)
    throw Error(AIFMM_ETIMEOUT, std::string(what) + ": " + std::to_string(now - before) +
                                    " tensor-core GEMM tile(s) gave up on a bounded pipeline wait; their output "
                                    "blocks are not written");
}

void tc_wait_args(aifmm_ctx* ctx, GemmArgs& a) {
  a.hold = ctx->gemmHold ? ctx->holdFlag : nullptr;
  a.waitNs = ctx->gemmHold ? 1000000ull : P5_WAIT_NS;
}

}  // namespace aifmm
