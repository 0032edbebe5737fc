// Split-TF32 complex grouped GEMM on the tcgen05 tensor cores: persistent,
// warp-specialised, 128 x 128 complex tiles.
//
// A complex product C = op(A) op(B) is one real product of twice the depth:
//   [Cr | Ci] = [Ar Ai] * [[Br, Bi], [-Bi, Br]]   (depth interleaved: real
// depth 2k is the real part of complex k, 2k+1 the imaginary part), so a
// tile of 128 rows x 128 complex columns is one 128 x 256 real MMA tile whose
// accumulator holds Cr in tensor-memory columns 0..127 and Ci in 128..255.
// Each real operand is split into TF32 high and low planes (x = hi + lo) and
// the product is accumulated as hi*hi + hi*lo + lo*hi in FP32: three
// 128x256x8 MMAs per 8-deep real step, 6 per 16-deep slice (8 complex k).
// Compared with the 128 x 64 complex tiles of zgemm_tc5p.cu (12 MMAs of
// 128x64x8 per complex 8-step) the tensor work per flop is the same, but each
// MMA reads 4 KB of A and 8 KB of B from shared memory for 262,144 MACs
// instead of 6 KB for 65,536, which takes the shared-memory reads off the
// critical path.
//
// A conversion kernel first writes every distinct operand once in the MMA's
// no-swizzle K-major core-matrix layout, chunk by chunk (A: 128 rows x 16
// real depth x {hi, lo} = 16 KB; B: 256 rows x 16 x {hi, lo} = 32 KB), so the
// GEMM only streams bytes.  The GEMM is persistent (one CTA per SM walks the
// tiles blockIdx.x, +gridDim.x, ...) with three roles:
//   warp 0   -- one thread copies each slice's A and B chunks with
//               cp.async.bulk into a four-stage ring (full/empty mbarriers);
//   warp 1   -- one thread issues the MMAs into one of two tensor-memory
//               accumulators (512 columns) and commits each slice to its
//               ring slot's "empty" barrier and each tile to the
//               accumulator's "full" barrier;
//   warps 2-5 -- read the finished accumulator (tcgen05.ld, each warp its
//               32-lane quarter), apply alpha and beta in FP64, store C, and
//               release the accumulator, while the MMAs of the next tile run
//               into the other one.
// Every wait is bounded (one second; one millisecond in the library's wait
// test); a wait that runs out makes the CTA stop, drain what it has in
// flight, leave its remaining tiles unwritten and count the failure
// (zgemm_tc6_timeouts()).
//
// A second operand form (FORM 1, "split planes") keeps the real and imaginary
// parts apart instead: A as four planes (Ar hi, Ar lo, Ai hi, Ai lo) of
// 128 rows, B likewise with 128 rows, and per 8-deep complex step twelve
// 128x128x8 MMAs into two accumulators, Cr += Ar Br - Ai Bi (the minus by the
// instruction's B negation) and Ci += Ar Bi + Ai Br, each as hi*hi + hi*lo +
// lo*hi.  The MMA work is the same; the operand bytes per step drop from 48 KB
// to 32 KB because B is not stored twice, at the price of twice as many
// (half as wide) MMAs.  The ring then holds six 32 KB stages.  On the
// solver's Schur launches (products of 100-1,000 on a side) the split form is
// 5-15 % faster and is the default (aifmm_ctx_set_gemm_tiling, the autotuner
// of GEMM precision 5 picks per launch class); on large square products the
// packed form's wider MMAs win.
#include <algorithm>
#include <map>

#include "dense.cuh"

namespace aifmm {

constexpr int T6_M = 128, T6_NC = 128, T6_N = 2 * T6_NC, T6_KS = 16, T6_THREADS = 192;
constexpr uint32_t T6_TMEM_COLS = 512;
constexpr uint32_t T6_A_WORDS = 2 * 2 * T6_M * 8, T6_B_WORDS = 2 * 2 * T6_N * 8;  // per slice chunk

// per-form chunk sizes (32-bit words) and ring depth
template <int FORM>
struct T6Form;
template <>
struct T6Form<0> {  // packed real: A [hi/lo][k-step][128 x 8], B [hi/lo][k-step][256 x 8]
  static constexpr uint32_t A_WORDS = T6_A_WORDS, B_WORDS = T6_B_WORDS;
  static constexpr int STAGES = 4;
};
template <>
struct T6Form<1> {  // split planes: A [re hi, re lo, im hi, im lo][128 x 8], B the same
  static constexpr uint32_t A_WORDS = 4 * T6_M * 8, B_WORDS = 4 * T6_NC * 8;
  static constexpr int STAGES = 6;
};
template <int FORM>
struct T6Smem {
  static constexpr uint32_t STAGE_WORDS = T6Form<FORM>::A_WORDS + T6Form<FORM>::B_WORDS;
  uint32_t ring[T6Form<FORM>::STAGES][STAGE_WORDS];  // each stage: A chunk, then B chunk
  unsigned long long full[T6Form<FORM>::STAGES], empty[T6Form<FORM>::STAGES], accFull[2], accEmpty[2];
  uint32_t tmem_slot;
  int err;
};

__device__ unsigned long long g_t6_timeouts;

__device__ __forceinline__ uint32_t t6_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
// word offset of (row, k) inside an 8-deep k-step of a K-major no-swizzle
// core-matrix tile: 8-row groups of 256 B, two 4-deep core matrices of 128 B
__device__ __forceinline__ int t6_off(int row, int k) {
  return (row >> 3) * 64 + (k >> 2) * 32 + (row & 7) * 4 + (k & 3);
}
__device__ __forceinline__ uint64_t t6_desc(const void* p) {
  uint64_t d = (uint64_t)((t6_smem(p) >> 4) & 0x3FFF);
  d |= (uint64_t)(128 >> 4) << 16;  // leading byte offset: the K-adjacent core matrix
  d |= (uint64_t)(256 >> 4) << 32;  // stride byte offset: the next 8-row group
  d |= (uint64_t)1 << 46;           // descriptor version
  return d;
}
// kind::tf32, FP32 accumulator, both operands K-major, M = 128, N = 256
// (packed real) or N = 128 with and without B negated (split planes)
constexpr uint32_t T6_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(T6_N >> 3) << 17) |
                              ((uint32_t)(T6_M >> 4) << 24);
constexpr uint32_t T6_IDESC_S = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(T6_NC >> 3) << 17) |
                                ((uint32_t)(T6_M >> 4) << 24);
constexpr uint32_t T6_IDESC_SN = T6_IDESC_S | (1u << 14);

__device__ __forceinline__ void t6_mma(uint32_t d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void t6_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(t6_smem(bar))
               : "memory");
}
__device__ __forceinline__ unsigned long long t6_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool t6_wait(unsigned long long* bar, uint32_t parity, unsigned long long limit) {
  const uint32_t a = t6_smem(bar);
  const unsigned long long t0 = t6_now();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (t6_now() - t0 > limit) return false;
  }
}
__device__ __forceinline__ bool t6_hold(const int* flag, unsigned long long limit) {
  const unsigned long long t0 = t6_now();
  while (*(const volatile int*)flag == 0)
    if (t6_now() - t0 > limit) return false;
  return true;
}
__device__ __forceinline__ void t6_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(t6_smem(bar)) : "memory");
}

// ---------------------------------------------------------------- conversion
struct T6Operand {
  const zd* src;
  uint32_t* dst;
  int rows, k, ld, op, isB;  // rows: M of op(A) / N of op(B); k: complex depth
  int nks;                   // slices (8 complex k each)
  int form;                  // 0 packed real, 1 split planes
};

__device__ __forceinline__ uint32_t t6_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void t6_split4(const float (&x)[4], uint4& hi, uint4& lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    h[q] = t6_tf32(x[q]);
    l[q] = t6_tf32(x[q] - __uint_as_float(h[q]));
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// One thread per (padded row, four consecutive complex k) of every operand:
// it reads the four entries and writes them as 16-byte vectors (the core
// matrix layout keeps four consecutive depths of a row together), so a warp's
// stores cover whole 128-byte lines.  Consecutive threads take consecutive
// rows.
__global__ void t6_convert_kernel(const T6Operand* __restrict__ ops, const long* __restrict__ start, int nops,
                                  long total) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nops - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (start[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    const T6Operand& O = ops[lo];
    const long u = t - start[lo];
    const int tileRows = O.isB ? T6_NC : T6_M;
    const int prow = ((O.rows + tileRows - 1) / tileRows) * tileRows;
    const int r = (int)(u % prow), q = (int)(u / prow);  // row, quad of complex depths 4q..4q+3
    float re[4], im[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int k = 4 * q + i;
      zd v = zmk(0, 0);
      if (r < O.rows && k < O.k) {
        if (!O.isB) v = (O.op == OP_N) ? O.src[(size_t)k * O.ld + r] : zconj(O.src[(size_t)r * O.ld + k]);
        else v = (O.op == OP_N) ? O.src[(size_t)r * O.ld + k] : zconj(O.src[(size_t)k * O.ld + r]);
      }
      re[i] = (float)v.x;
      im[i] = (float)v.y;
    }
    const int tr = r / tileRows, rr = r % tileRows;
    const int rowOff = (rr >> 3) * 64 + (rr & 7) * 4;
    uint4 h, l;
    if (O.form == 1) {  // planes re hi, re lo, im hi, im lo; slice = 8 complex k
      const int ks = q >> 1, half = q & 1;
      const uint32_t words = O.isB ? T6Form<1>::B_WORDS : T6Form<1>::A_WORDS;
      uint32_t* c = O.dst + ((size_t)tr * O.nks + ks) * words + rowOff + half * 32;
      t6_split4(re, h, l);
      *reinterpret_cast<uint4*>(c) = h;
      *reinterpret_cast<uint4*>(c + 1024) = l;
      t6_split4(im, h, l);
      *reinterpret_cast<uint4*>(c + 2048) = h;
      *reinterpret_cast<uint4*>(c + 3072) = l;
      continue;
    }
    // packed real: real depths 8q..8q+7 = one k-step of the slice q / 2
    const int ks = q >> 1, step = q & 1;
    if (!O.isB) {
      uint32_t* c = O.dst + ((size_t)tr * O.nks + ks) * T6_A_WORDS + (size_t)step * (T6_M * 8) + rowOff;
      const int pw = 2 * T6_M * 8;  // hi plane -> lo plane
      const float a0[4] = {re[0], im[0], re[1], im[1]}, a1[4] = {re[2], im[2], re[3], im[3]};
      t6_split4(a0, h, l);
      *reinterpret_cast<uint4*>(c) = h;
      *reinterpret_cast<uint4*>(c + pw) = l;
      t6_split4(a1, h, l);
      *reinterpret_cast<uint4*>(c + 32) = h;
      *reinterpret_cast<uint4*>(c + pw + 32) = l;
    } else {
      uint32_t* c = O.dst + ((size_t)tr * O.nks + ks) * T6_B_WORDS + (size_t)step * (T6_N * 8);
      const int pw = 2 * T6_N * 8;
      // rows rr (Cr): [Br, -Bi]; rows 128 + rr (Ci): [Bi, Br] along the depth
      const int offR = rowOff, offI = ((T6_NC + rr) >> 3) * 64 + (rr & 7) * 4;
      const float r0[4] = {re[0], -im[0], re[1], -im[1]}, r1[4] = {re[2], -im[2], re[3], -im[3]};
      const float i0[4] = {im[0], re[0], im[1], re[1]}, i1[4] = {im[2], re[2], im[3], re[3]};
      t6_split4(r0, h, l);
      *reinterpret_cast<uint4*>(c + offR) = h;
      *reinterpret_cast<uint4*>(c + pw + offR) = l;
      t6_split4(r1, h, l);
      *reinterpret_cast<uint4*>(c + offR + 32) = h;
      *reinterpret_cast<uint4*>(c + pw + offR + 32) = l;
      t6_split4(i0, h, l);
      *reinterpret_cast<uint4*>(c + offI) = h;
      *reinterpret_cast<uint4*>(c + pw + offI) = l;
      t6_split4(i1, h, l);
      *reinterpret_cast<uint4*>(c + offI + 32) = h;
      *reinterpret_cast<uint4*>(c + pw + offI + 32) = l;
    }
  }
}

// ---------------------------------------------------------------- GEMM
__device__ __forceinline__ int t6_group(const GemmGroup* G, int ngroups, int tile) {
  int lo = 0, hi = ngroups - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (G[mid].tileStart <= tile) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
// tile -> (row tile, column tile) of its group, in the launch's raster order
__device__ __forceinline__ void t6_coords(const GemmProblem* probs, const GemmGroup& g, int raster, int tile,
                                          int& tm, int& tn) {
  const int local = tile - g.tileStart;
  if (raster == 0) {
    tm = local / g.tilesN;
    tn = local % g.tilesN;
  } else {
    const int tilesM = (probs[g.head].m + T6_M - 1) / T6_M;
    tn = local / tilesM;
    tm = local % tilesM;
  }
}
__device__ __forceinline__ int t6_slices(const GemmProblem* probs, const GemmGroup& g) {
  int total = 0;
  for (int q = 0; q < g.nchain; ++q) total += (probs[g.head + q].k + 7) / 8;
  return total;
}

template <int FORM, bool INLINE>
__global__ void __launch_bounds__(T6_THREADS, 1) zgemm_tc6_kernel(const __grid_constant__ GemmArgs a, int nTiles) {
  using F = T6Form<FORM>;
  constexpr int STAGES = F::STAGES;
  constexpr uint32_t A_WORDS = F::A_WORDS, B_WORDS = F::B_WORDS;
  extern __shared__ unsigned char t6_raw[];
  T6Smem<FORM>& S =
      *reinterpret_cast<T6Smem<FORM>*>((reinterpret_cast<uintptr_t>(t6_raw) + 1023) & ~uintptr_t(1023));
  const GemmGroup* G = INLINE ? a.ig : a.groups;
  const GemmProblem* probs = INLINE ? a.ip : a.probs;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned long long lim = a.waitNs;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(t6_smem(&S.tmem_slot)),
                 "r"(T6_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    for (int s = 0; s < STAGES; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(t6_smem(&S.full[s])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(t6_smem(&S.empty[s])) : "memory");
    }
    for (int b = 0; b < 2; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(t6_smem(&S.accFull[b])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(t6_smem(&S.accEmpty[b])) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    S.err = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = S.tmem_slot;

  if (warp == 0) {
    if (lane == 0) {  // ---- producer: slice chunks into the ring
      bool ok = !(a.hold && !t6_hold(a.hold, lim));
      uint32_t it = 0;
      for (int tile = blockIdx.x; tile < nTiles && ok; tile += gridDim.x) {
        const GemmGroup g = G[t6_group(G, a.ngroups, tile)];
        int tm, tn;
        t6_coords(probs, g, a.raster, tile, tm, tn);
        for (int q = 0; q < g.nchain && ok; ++q) {
          const GemmProblem& P = probs[g.head + q];
          const int nks = (P.k + 7) / 8;
          for (int ks = 0; ks < nks; ++ks, ++it) {
            const int s = it % STAGES;
            const uint32_t ph = (it / STAGES) & 1u;
            if (!t6_wait(&S.empty[s], ph ^ 1u, lim) || *(volatile int*)&S.err) {
              ok = false;
              break;
            }
            const uint32_t* ga = P.pa + ((size_t)tm * nks + ks) * A_WORDS;
            const uint32_t* gb = P.pb + ((size_t)tn * nks + ks) * B_WORDS;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(t6_smem(&S.full[s])),
                         "r"((A_WORDS + B_WORDS) * 4)
                         : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    t6_smem(&S.ring[s][0])),
                "l"(ga), "r"(A_WORDS * 4), "r"(t6_smem(&S.full[s]))
                : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    t6_smem(&S.ring[s][A_WORDS])),
                "l"(gb), "r"(B_WORDS * 4), "r"(t6_smem(&S.full[s]))
                : "memory");
          }
        }
      }
      if (!ok) S.err = 1;
      // drain: every slot's last copy has landed before the CTA may exit
      for (int q = 0; q < STAGES && it > 0; ++q) {
        const int back = (int)it - 1 - q;
        if (back < 0) break;
        t6_wait(&S.full[back % STAGES], (uint32_t)(back / STAGES) & 1u, lim);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // ---- MMA issuer
      bool ok = true;
      uint32_t it = 0;
      int lastSlot = -1;
      uint32_t lastPh = 0;
      int local = 0;
      for (int tile = blockIdx.x; tile < nTiles && ok; tile += gridDim.x, ++local) {
        const int b = local & 1;
        const uint32_t aph = (uint32_t)(local >> 1) & 1u;
        if (!t6_wait(&S.accEmpty[b], aph ^ 1u, lim) || *(volatile int*)&S.err) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)(b * T6_N);
        const GemmGroup g = G[t6_group(G, a.ngroups, tile)];
        const int total = t6_slices(probs, g);
        for (int j = 0; j < total; ++j, ++it) {
          const int s = it % STAGES;
          const uint32_t ph = (it / STAGES) & 1u;
          if (!t6_wait(&S.full[s], ph, lim)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t* sa = &S.ring[s][0];
          const uint32_t* sb = &S.ring[s][A_WORDS];
          if (FORM == 0) {
#pragma unroll
            for (int step = 0; step < 2; ++step) {  // [plane][step][rows x 8]
              const uint64_t ah = t6_desc(sa + step * T6_M * 8), al = t6_desc(sa + (2 + step) * T6_M * 8);
              const uint64_t bh = t6_desc(sb + step * T6_N * 8), bl = t6_desc(sb + (2 + step) * T6_N * 8);
              t6_mma(d, ah, bh, T6_IDESC, (j | step) ? 1u : 0u);
              t6_mma(d, ah, bl, T6_IDESC, 1u);
              t6_mma(d, al, bh, T6_IDESC, 1u);
            }
          } else {  // [re hi, re lo, im hi, im lo][128 x 8]
            const uint64_t arh = t6_desc(sa), arl = t6_desc(sa + 1024), aih = t6_desc(sa + 2048),
                           ail = t6_desc(sa + 3072);
            const uint64_t brh = t6_desc(sb), brl = t6_desc(sb + 1024), bih = t6_desc(sb + 2048),
                           bil = t6_desc(sb + 3072);
            const uint32_t first = j ? 1u : 0u, dr = d, di = d + T6_NC;
            // Cr += Ar Br - Ai Bi ; Ci += Ar Bi + Ai Br (hi*hi + hi*lo + lo*hi each)
            t6_mma(dr, arh, brh, T6_IDESC_S, first);
            t6_mma(dr, arh, brl, T6_IDESC_S, 1u);
            t6_mma(dr, arl, brh, T6_IDESC_S, 1u);
            t6_mma(dr, aih, bih, T6_IDESC_SN, 1u);
            t6_mma(dr, aih, bil, T6_IDESC_SN, 1u);
            t6_mma(dr, ail, bih, T6_IDESC_SN, 1u);
            t6_mma(di, arh, bih, T6_IDESC_S, first);
            t6_mma(di, arh, bil, T6_IDESC_S, 1u);
            t6_mma(di, arl, bih, T6_IDESC_S, 1u);
            t6_mma(di, aih, brh, T6_IDESC_S, 1u);
            t6_mma(di, aih, brl, T6_IDESC_S, 1u);
            t6_mma(di, ail, brh, T6_IDESC_S, 1u);
          }
          t6_commit(&S.empty[s]);
          lastSlot = s;
          lastPh = ph;
        }
        if (!ok) break;
        t6_commit(&S.accFull[b]);  // arrives once this tile's MMAs are complete
      }
      if (!ok) {
        S.err = 1;
        if (lastSlot >= 0) t6_wait(&S.empty[lastSlot], lastPh, lim);  // the MMAs in flight have finished
      }
    }
  } else {  // ---- epilogue: warps 2..5, lane quarter warp % 4
    const int quarter = warp & 3;
    int local = 0;
    for (int tile = blockIdx.x; tile < nTiles; tile += gridDim.x, ++local) {
      const int b = local & 1;
      const uint32_t aph = (uint32_t)(local >> 1) & 1u;
      // warp-uniform outcome: the loads below are .sync.aligned
      if (!__all_sync(0xffffffffu, t6_wait(&S.accFull[b], aph, lim))) {
        if (lane == 0) S.err = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const GemmGroup g = G[t6_group(G, a.ngroups, tile)];
      int tm, tn;
      t6_coords(probs, g, a.raster, tile, tm, tn);
      const GemmProblem& P = probs[g.head];
      const bool any = t6_slices(probs, g) > 0;
      const bool beta0 = (P.beta.x == 0.0 && P.beta.y == 0.0);
      const int row = tm * T6_M + quarter * 32 + lane;
      const uint32_t base = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * T6_N);
      for (int c0 = 0; c0 < T6_NC; c0 += 16) {
        // the chunk's 16 C entries of this row are loaded first, all in
        // flight at once (a warp reads 512 contiguous bytes per column), so
        // the accumulating tiles pay one memory latency per chunk instead
        // of one per column
        zd cv[16];
        const int ncol = min(16, P.n - (tn * T6_NC + c0));
        if (!beta0 && row < P.m) {
          const zd* cp0 = P.C + (size_t)(tn * T6_NC + c0) * P.ldc + row;
#pragma unroll
          for (int j = 0; j < 16; ++j)
            if (j < ncol) cv[j] = __ldcg(cp0 + (size_t)j * P.ldc);
        }
        uint32_t vr[16], vi[16];
        if (any) {
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
              "[%16];"
              : "=r"(vr[0]), "=r"(vr[1]), "=r"(vr[2]), "=r"(vr[3]), "=r"(vr[4]), "=r"(vr[5]), "=r"(vr[6]),
                "=r"(vr[7]), "=r"(vr[8]), "=r"(vr[9]), "=r"(vr[10]), "=r"(vr[11]), "=r"(vr[12]), "=r"(vr[13]),
                "=r"(vr[14]), "=r"(vr[15])
              : "r"(base + (uint32_t)c0));
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
              "[%16];"
              : "=r"(vi[0]), "=r"(vi[1]), "=r"(vi[2]), "=r"(vi[3]), "=r"(vi[4]), "=r"(vi[5]), "=r"(vi[6]),
                "=r"(vi[7]), "=r"(vi[8]), "=r"(vi[9]), "=r"(vi[10]), "=r"(vi[11]), "=r"(vi[12]), "=r"(vi[13]),
                "=r"(vi[14]), "=r"(vi[15])
              : "r"(base + (uint32_t)(T6_NC + c0)));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j) vr[j] = vi[j] = 0u;
        }
        if (row < P.m) {
          zd* cp0 = P.C + (size_t)(tn * T6_NC + c0) * P.ldc + row;
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            if (j >= ncol) break;
            zd v = zmul(P.alpha, zmk((double)__uint_as_float(vr[j]), (double)__uint_as_float(vi[j])));
            if (!beta0) v = zadd(v, zmul(P.beta, cv[j]));
            cp0[(size_t)j * P.ldc] = v;
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) t6_arrive(&S.accEmpty[b]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (tid == 0 && S.err) atomicAdd(&g_t6_timeouts, 1ull);
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(T6_TMEM_COLS) : "memory");
}

namespace {
struct T6Key {
  const zd* src;
  int ld, op, rows, k, isB;
  bool operator<(const T6Key& o) const {
    if (src != o.src) return src < o.src;
    if (ld != o.ld) return ld < o.ld;
    if (op != o.op) return op < o.op;
    if (rows != o.rows) return rows < o.rows;
    if (k != o.k) return k < o.k;
    return isB < o.isB;
  }
};
size_t t6_words(const T6Key& key, int form) {
  const int tr = key.isB ? T6_NC : T6_M;
  const int nks = std::max(1, (key.k + 7) / 8);
  const size_t chunk = form == 1 ? (key.isB ? T6Form<1>::B_WORDS : T6Form<1>::A_WORDS)
                                 : (key.isB ? T6_B_WORDS : T6_A_WORDS);
  return (size_t)((key.rows + tr - 1) / tr) * nks * chunk;
}
constexpr size_t T6_PLANE_BUDGET = (size_t)4 << 30;  // bytes of planes per launch
}  // namespace

// Converts the distinct operands of groups [g0, g1) and launches their tiles.
static void t6_launch(aifmm_ctx* ctx, const std::vector<GemmProblem>& all, const std::vector<GemmGroup>& gs, size_t g0,
                      size_t g1) {
  const int form = ctx->gemmForm;
  std::map<T6Key, size_t> where;
  size_t words = 0;
  std::vector<GemmProblem> ps;
  std::vector<GemmGroup> groups;
  long tiles = 0;
  for (size_t gi = g0; gi < g1; ++gi) {
    GemmGroup g = gs[gi];
    const int head = (int)ps.size();
    for (int q = 0; q < g.nchain; ++q) {
      const GemmProblem& p = all[g.head + q];
      for (const T6Key& key : {T6Key{p.A, p.lda, p.opA, p.m, p.k, 0}, T6Key{p.B, p.ldb, p.opB, p.n, p.k, 1}})
        if (!where.count(key)) {
          where[key] = words;
          words += t6_words(key, form);
        }
      ps.push_back(p);
    }
    g.head = head;
    g.tileStart = (int)tiles;
    tiles += (long)((all[gs[gi].head].m + T6_M - 1) / T6_M) * g.tilesN;
    groups.push_back(g);
  }
  DevBuf planes(ctx, sizeof(uint32_t) * std::max<size_t>(words, 4));
  uint32_t* base = planes.as<uint32_t>();
  std::vector<T6Operand> ops;
  std::vector<long> start;
  long total = 0;
  for (const auto& kv : where) {
    const T6Key& key = kv.first;
    if (key.k <= 0) continue;
    const int nks = (key.k + 7) / 8, tr = key.isB ? T6_NC : T6_M;
    ops.push_back({key.src, base + kv.second, key.rows, key.k, key.ld, key.op, key.isB, nks, form});
    start.push_back(total);
    total += (long)((key.rows + tr - 1) / tr) * tr * (nks * 2);  // rows x quads of 4 complex k
  }
  for (GemmProblem& p : ps) {
    p.pa = base + where[T6Key{p.A, p.lda, p.opA, p.m, p.k, 0}];
    p.pb = base + where[T6Key{p.B, p.ldb, p.opB, p.n, p.k, 1}];
  }
  if (total > 0) {
    DevBuf dops = upload(ctx, ops), dst = upload(ctx, start);
    const int grid = (int)std::min<long>((total + 255) / 256, 148L * 32);
    t6_convert_kernel<<<grid, 256, 0, ctx->stream>>>(dops.as<T6Operand>(), dst.as<long>(), (int)ops.size(), total);
    AIFMM_LAUNCHED();
  }
  if (tiles <= 0) return;
  AIFMM_REQUIRE(tiles < (long)INT32_MAX, AIFMM_EOVERFLOW, "too many GEMM tiles");
  GemmArgs a;
  a.ngroups = (int)groups.size();
  a.probs = nullptr;
  a.groups = nullptr;
  a.raster = ctx->gemmRaster;
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
  const unsigned grid = (unsigned)std::min<long>(tiles, ctx->numSMs > 0 ? ctx->numSMs : 148);
  if (form == 1) {
    const size_t smem = sizeof(T6Smem<1>) + 1024;
    smem_attr_once((const void*)zgemm_tc6_kernel<1, true>, ctx->device, (int)smem);
    smem_attr_once((const void*)zgemm_tc6_kernel<1, false>, ctx->device, (int)smem);
    if (inl) zgemm_tc6_kernel<1, true><<<grid, T6_THREADS, smem, ctx->stream>>>(a, (int)tiles);
    else zgemm_tc6_kernel<1, false><<<grid, T6_THREADS, smem, ctx->stream>>>(a, (int)tiles);
  } else {
    const size_t smem = sizeof(T6Smem<0>) + 1024;
    smem_attr_once((const void*)zgemm_tc6_kernel<0, true>, ctx->device, (int)smem);
    smem_attr_once((const void*)zgemm_tc6_kernel<0, false>, ctx->device, (int)smem);
    if (inl) zgemm_tc6_kernel<0, true><<<grid, T6_THREADS, smem, ctx->stream>>>(a, (int)tiles);
    else zgemm_tc6_kernel<0, false><<<grid, T6_THREADS, smem, ctx->stream>>>(a, (int)tiles);
  }
  AIFMM_LAUNCHED();
}

void zgemm_tc6(aifmm_ctx* ctx, const std::vector<GemmProblem>& ps, const std::vector<GemmGroup>& gs) {
  size_t g0 = 0;
  while (g0 < gs.size()) {
    std::map<T6Key, bool> seen;
    size_t bytes = 0, g1 = g0;
    while (g1 < gs.size()) {
      size_t add = 0;
      std::vector<T6Key> fresh;
      for (int q = 0; q < gs[g1].nchain; ++q) {
        const GemmProblem& p = ps[gs[g1].head + q];
        for (const T6Key& key : {T6Key{p.A, p.lda, p.opA, p.m, p.k, 0}, T6Key{p.B, p.ldb, p.opB, p.n, p.k, 1}})
          if (!seen.count(key)) {
            bool dup = false;
            for (const T6Key& f : fresh) dup = dup || !(f < key || key < f);
            if (!dup) {
              fresh.push_back(key);
              add += 4 * t6_words(key, ctx->gemmForm);
            }
          }
      }
      if (g1 > g0 && bytes + add > T6_PLANE_BUDGET) break;
      for (const T6Key& f : fresh) seen[f] = true;
      bytes += add;
      ++g1;
    }
    t6_launch(ctx, ps, gs, g0, g1);
    g0 = g1;
  }
}

long zgemm_tc6_timeouts() {
  unsigned long long v = 0;
  AIFMM_CUDA(cudaMemcpyFromSymbol(&v, g_t6_timeouts, sizeof(v)));
  return (long)v;
}

}  // namespace aifmm
