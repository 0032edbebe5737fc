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
};

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

struct CopyProblem {
  const zd* src;
  zd* dst;
  int rows, cols;  // of dst
  int lds, ldd;
  int conjTrans;   // dst = conj(src)^T when set
  zd scale;        // dst = scale * src
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
