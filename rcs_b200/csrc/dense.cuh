// Dense complex128 building blocks of the GPU solver: grouped GEMM, blocked
// partial-pivot LU and solves, batched copies and Frobenius norms.  All
// matrices are column-major device arrays; all work is stream-ordered on the
// context stream.
#pragma once
#include <vector>

#include "context.cuh"

namespace aifmm {

enum Op : int { OP_N = 0, OP_C = 1 };  // none / conjugate transpose

struct GemmProblem {
  const zd* A;
  const zd* B;
  zd* C;
  int m, n, k;
  int lda, ldb, ldc;
  int opA, opB;
  zd alpha, beta;
  // split-TF32 planes of op(A) / op(B) in the tcgen05 tile layout (set by
  // the launcher of the pre-tiled tensor-core GEMM; unused elsewhere)
  const uint32_t* pa = nullptr;
  const uint32_t* pb = nullptr;
};

// A group = a chain of problems accumulated into one C (consecutive in the
// problem list); its tiles are numbered from tileStart, tilesN along n.
struct GemmGroup {
  int head, nchain, tilesN, tileStart;
};
// Launch arguments of the grouped GEMM kernels.  Up to GEMM_INLINE groups
// travel in the kernel's parameter space (no upload); larger launches read
// device arrays.
constexpr int GEMM_INLINE = 96;
struct GemmArgs {
  int ngroups;
  const GemmProblem* probs;
  const GemmGroup* groups;
  // tensor-core kernels: limit of each bounded pipeline wait (ns), and an
  // optional device flag that the issuing thread waits on before its first
  // copy (null in normal use; the library's wait test points it at a flag
  // that nothing sets, so that the wait runs out)
  unsigned long long waitNs;
  const int* hold;
  // persistent tensor-core GEMM: tile order inside a group (0: row-major,
  // 1: column-major), picked by the autotuner
  int raster;
  GemmProblem ip[GEMM_INLINE];
  GemmGroup ig[GEMM_INLINE];
};
// Tensor-core (tcgen05) form of the split-TF32 grouped GEMM, 128x64 complex
// tiles (zgemm_tc5.cu); groups must be tiled with tilesN = ceil(n / 64) and
// ceil(m / 128) row tiles.
void zgemm_tc5_launch(aifmm_ctx* ctx, const GemmArgs& a, bool inl, long tiles);
// Number of tcgen05 pipeline waits that ran out (each leaves its tile unwritten).
long zgemm_tc5_timeouts();
// Sum of both tensor-core GEMMs' timeout counters, and a check that throws
// AIFMM_ETIMEOUT when it grew past `before` (call after the stream drained).
long tc_timeouts();
void tc_check(long before, const char* what);
// Fills the wait limit and hold flag of a tensor-core launch from the context.
void tc_wait_args(aifmm_ctx* ctx, GemmArgs& a);
// The tensor-core GEMM over pre-tiled operand planes (zgemm_tc5p.cu): the
// operands of every problem are first converted once into split-TF32 planes
// laid out tile by tile, then each CTA streams its tiles with bulk copies.
// Same tiling as zgemm_tc5_launch.
long zgemm_tc5p_timeouts();
void zgemm_tc5p(aifmm_ctx* ctx, std::vector<GemmProblem> ps, const std::vector<GemmGroup>& gs, long tiles);
// The persistent, warp-specialised tensor-core GEMM (zgemm_tc6.cu): complex
// products as one real product of twice the depth, 128 x 128 complex tiles,
// double-buffered tensor-memory accumulators.  Groups must be tiled with
// tilesN = ceil(n / 128) and ceil(m / 128) row tiles.
long zgemm_tc6_timeouts();
void zgemm_tc6(aifmm_ctx* ctx, const std::vector<GemmProblem>& ps, const std::vector<GemmGroup>& gs);
// GEMM precision 5: the tensor-core kernel and tile order picked per launch
// class by the autotuner (autotune.cu); tune_report lists its trials.
void zgemm_tuned(aifmm_ctx* ctx, const std::vector<GemmProblem>& probs, const std::vector<int>& chain);
std::string tune_report(aifmm_ctx* ctx);

// C = alpha op(A) op(B) + beta C for every problem, one launch; the
// problems must write disjoint C.
void zgemm_grouped(aifmm_ctx* ctx, const std::vector<GemmProblem>& probs);
// Same with chains: chain[i] = L > 0 makes problems i..i+L-1 one
// accumulation C = alpha sum_q op(A_q) op(B_q) + beta_i C (they share C,
// m, n, ldc and alpha; beta is 1 after the first); chain[i+1..i+L-1] are
// ignored.  Distinct chains must write disjoint C.
void zgemm_chained(aifmm_ctx* ctx, const std::vector<GemmProblem>& probs, const std::vector<int>& chain);
// Per-launch CUDA-event timing of zgemm_grouped (process-wide switch).
void gemm_profile_enable(bool on);
void gemm_profile_read(double* ms, double* flops, long* launches);
// Device-time records (events around launches) while the GEMM profiler is
// on: the grouped GEMMs and the RRQR launch chains; a table by tag of
// "tag launches seconds flops" lines.
bool gemm_profile_on();
void device_span_record(cudaEvent_t e0, cudaEvent_t e1, const std::string& tag, double flops);
std::string gemm_profile_table();

struct CopyProblem {
  const zd* src;     // nullptr: dst is zero-filled
  zd* dst;
  int rows, cols;  // of dst
  int lds, ldd;
  int conjTrans;   // dst = conj(src)^T when set
  zd scale;        // dst = scale * src
  int accumulate;  // dst += scale * src when set
};
void zcopy_grouped(aifmm_ctx* ctx, const std::vector<CopyProblem>& probs);
void zfill(aifmm_ctx* ctx, zd* p, size_t n, zd v);
void zset_identity(aifmm_ctx* ctx, zd* p, int rows, int cols, zd diag);

struct NormProblem {
  const zd* p;
  int rows, cols, ld;
};
// Frobenius norms into out_dev[i].
void znorm_grouped(aifmm_ctx* ctx, const std::vector<NormProblem>& probs, double* out_dev);

// In-place partial-pivot LU of an n x n matrix (lda); pivots are row
// transpositions (piv[k] = row swapped with k).  Returns via *info_dev the
// 1-based index of the first exactly-zero pivot (0 if none).
void zgetrf(aifmm_ctx* ctx, zd* A, int n, int lda, int* piv_dev, int* info_dev);
// B <- A^{-1} B for the factors of zgetrf.
void zgetrs(aifmm_ctx* ctx, const zd* LU, int n, int lda, const int* piv_dev, zd* B, int nrhs, int ldb);

}  // namespace aifmm
