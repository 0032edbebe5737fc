// FP64 forward operator y = A x of the H^2 representation that the AIFMM
// constructor builds (leaf near field P2P, P2M upward, M2L on every level's
// interaction list, L2P downward), used as the residual operator of the
// iterative refinement around a factorization.  The reference never applies
// its tree as an operator (it factorizes it directly); this operator is built
// with the same assembly code at a tighter ACA tolerance than the
// factorization it refines, so that the residual it measures is that of the
// MoM operator to within that tolerance.
//
// Layout: unknowns are permuted to tree order (leaves in box order, each
// leaf's charges in the reference's chargeLocations order), so a box's slice
// of every level vector is contiguous and the children of box k -- boxes
// 8k..8k+7 -- occupy one contiguous range of the next level.  Each box's
// far-field blocks M2L[k][l], l in IL(k), are packed side by side into one
// matrix, and its leaf near-field blocks P2P[k][nn] likewise, so that a level's
// interactions are one grouped skinny GEMM against a gathered stack of the
// source vectors.
#pragma once
#include <map>
#include <memory>
#include <vector>

#include "solver.cuh"

namespace aifmm {

// C (m x nr) = A (m x k) B (k x nr) (+ C when accumulate), column-major.
struct SkinnyProblem {
  const zd* A;
  const zd* B;
  zd* C;
  int m, k, lda, ldb, ldc, accumulate;
};
struct SkinnyTile {
  int prob, row0;
};
constexpr int SKINNY_ROWS = 32;
constexpr int SKINNY_MAXNR = 16;
// One launch per 8 columns over pre-uploaded problems/tiles; nr <= SKINNY_MAXNR.
void zgemm_skinny(aifmm_ctx* ctx, const SkinnyProblem* probs, const SkinnyTile* tiles, int ntiles, int nr);
// dst[t, c] = src[idx[t], c] (gather) or dst[idx[t], c] = src[t, c] (scatter), c < nr.
void zrows_gather(aifmm_ctx* ctx, const zd* src, int lds, const int* idx, int n, zd* dst, int ldd, int nr);
void zrows_scatter(aifmm_ctx* ctx, const zd* src, int lds, const int* idx, int n, zd* dst, int ldd, int nr);

class H2Operator {
 public:
  // Takes the assembled (unfactorized) blocks of `s`, which is released.
  explicit H2Operator(std::unique_ptr<Solver> s);
  // y = A x for x, y: N x nr device blocks (leading dimensions ldx, ldy);
  // columns go through the skinny GEMMs SKINNY_MAXNR at a time.
  void apply(const zd* x, int ldx, zd* y, int ldy, int nr);
  int N = 0;
  double bytes = 0;           // device bytes of the packed blocks
  double flopsPerColumn = 0;  // complex-counted flops of one matvec column (8 per complex multiply-add)
  long launchesPerApply = 0;
  aifmm_ctx* ctx = nullptr;

 private:
  struct Level {
    std::vector<int> moff, loff;  // per box offsets into the level's multipole / local vectors
    int nm = 0, nl = 0;
    std::vector<DMat> P2M, L2P, Mpack;
    std::vector<int> sidx;        // stacked source rows (into the multipole vector) of every box's IL
    std::vector<int> soff;        // per box offset into the stack
  };
  int L = 0, j0 = 0;
  std::vector<Level> lv;          // indexed by level
  std::vector<int> xoff, nx;      // leaf offsets and sizes in tree order
  std::vector<int> perm;          // tree-order position -> unknown id
  std::vector<DMat> Ppack;        // leaf near field, per box
  std::vector<int> xidx, xsoff;   // stacked near-field source rows (tree order), per box offsets
  DevBuf dperm, dxidx;
  std::vector<DevBuf> dsidx;

  struct Phase {
    DevBuf probs, tiles;
    int ntiles = 0;
  };
  struct Plan {
    int nr = 0;
    DevBuf Xt, Yt, SX;
    std::vector<DevBuf> M, Lc, S;
    std::vector<Phase> up, m2l, down;
    Phase leafL2P, leafP2P;
  };
  std::map<int, std::unique_ptr<Plan>> plans_;  // by column count
  Plan& plan(int nr);
  void applyChunk(const zd* x, int ldx, zd* y, int ldy, int nr);
  Phase phase(const std::vector<SkinnyProblem>& ps);
  void run(const Phase& p, int nr);
};

}  // namespace aifmm

struct aifmm_operator {
  std::unique_ptr<aifmm::H2Operator> op;
};
