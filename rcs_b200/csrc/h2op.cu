// H^2 forward operator: packing of the assembled blocks and the matvec
// (skinny grouped GEMMs over pre-uploaded problem lists, row gathers).
#include <algorithm>

#include "h2op.cuh"

namespace aifmm {

// ------------------------------------------------------------------ kernels
// One CTA = 32 rows of one problem; warp w sums the columns k = w (mod 8) of
// A against B, lane = row, so each A column segment is one coalesced 512-byte
// load; the eight warps' partial sums are added in warp order (deterministic).
template <int NR>
__global__ void __launch_bounds__(256) zgemm_skinny_kernel(const SkinnyProblem* __restrict__ probs,
                                                           const SkinnyTile* __restrict__ tiles, int c0) {
  __shared__ zd red[8][NR][SKINNY_ROWS];
  const SkinnyTile T = tiles[blockIdx.x];
  const SkinnyProblem P = probs[T.prob];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int row = T.row0 + lane;
  const bool live = row < P.m;
  zd acc[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) acc[r] = zmk(0, 0);
  const zd* A = P.A + (live ? row : 0);
  const zd* B = P.B + (size_t)c0 * P.ldb;
#pragma unroll 2
  for (int k = w; k < P.k; k += 8) {
    const zd a = live ? A[(size_t)k * P.lda] : zmk(0, 0);
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      const zd b = __ldg(B + (size_t)r * P.ldb + k);
      acc[r].x = fma(a.x, b.x, acc[r].x);
      acc[r].x = fma(-a.y, b.y, acc[r].x);
      acc[r].y = fma(a.x, b.y, acc[r].y);
      acc[r].y = fma(a.y, b.x, acc[r].y);
    }
  }
#pragma unroll
  for (int r = 0; r < NR; ++r) red[w][r][lane] = acc[r];
  __syncthreads();
  for (int t = threadIdx.x; t < NR * SKINNY_ROWS; t += blockDim.x) {
    const int r = t / SKINNY_ROWS, l = t % SKINNY_ROWS;
    const int rr = T.row0 + l;
    if (rr >= P.m) continue;
    zd s = red[0][r][l];
#pragma unroll
    for (int q = 1; q < 8; ++q) s = zadd(s, red[q][r][l]);
    zd* cp = P.C + (size_t)(c0 + r) * P.ldc + rr;
    *cp = P.accumulate ? zadd(*cp, s) : s;
  }
}

void zgemm_skinny(aifmm_ctx* ctx, const SkinnyProblem* probs, const SkinnyTile* tiles, int ntiles, int nr) {
  if (ntiles <= 0) return;
  AIFMM_REQUIRE(nr >= 1 && nr <= SKINNY_MAXNR, AIFMM_EINVAL, "skinny GEMM column count out of range");
  for (int c0 = 0; c0 < nr; c0 += 8) {
    const int nc = std::min(8, nr - c0);
    switch (nc) {
#define SKINNY_CASE(V) \
  case V: zgemm_skinny_kernel<V><<<ntiles, 256, 0, ctx->stream>>>(probs, tiles, c0); break;
      SKINNY_CASE(1) SKINNY_CASE(2) SKINNY_CASE(3) SKINNY_CASE(4)
      SKINNY_CASE(5) SKINNY_CASE(6) SKINNY_CASE(7) SKINNY_CASE(8)
#undef SKINNY_CASE
    }
    AIFMM_LAUNCHED();
  }
}

__global__ void zrows_kernel(const zd* __restrict__ src, int lds, const int* __restrict__ idx, int n, zd* dst, int ldd,
                             int nr, int scatter) {
  const long total = (long)n * nr;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t % n), c = (int)(t / n);
    if (scatter) dst[(size_t)c * ldd + idx[i]] = src[(size_t)c * lds + i];
    else dst[(size_t)c * ldd + i] = src[(size_t)c * lds + idx[i]];
  }
}

static void zrows(aifmm_ctx* ctx, const zd* src, int lds, const int* idx, int n, zd* dst, int ldd, int nr, int sc) {
  if (n <= 0 || nr <= 0) return;
  const int grid = (int)std::min<long>(((long)n * nr + 255) / 256, 148L * 16);
  zrows_kernel<<<grid, 256, 0, ctx->stream>>>(src, lds, idx, n, dst, ldd, nr, sc);
  AIFMM_LAUNCHED();
}
void zrows_gather(aifmm_ctx* ctx, const zd* src, int lds, const int* idx, int n, zd* dst, int ldd, int nr) {
  zrows(ctx, src, lds, idx, n, dst, ldd, nr, 0);
}
void zrows_scatter(aifmm_ctx* ctx, const zd* src, int lds, const int* idx, int n, zd* dst, int ldd, int nr) {
  zrows(ctx, src, lds, idx, n, dst, ldd, nr, 1);
}

// ------------------------------------------------------------------ packing
H2Operator::H2Operator(std::unique_ptr<Solver> sp) {
  AIFMM_REQUIRE(sp && !sp->factored, AIFMM_ESTATE, "the forward operator needs an assembled, unfactorized tree");
  Solver& s = *sp;
  ctx = s.ctx;
  N = s.N;
  L = s.nLevels;
  j0 = s.startLevel;
  Ops ops(ctx);
  const int nLeaf = s.nBoxesPerLevel[L];
  xoff.resize(nLeaf);
  nx.resize(nLeaf);
  for (int k = 0; k < nLeaf; ++k) {
    xoff[k] = (int)perm.size();
    nx[k] = (int)s.tree[L][k].chargeLocations.size();
    perm.insert(perm.end(), s.tree[L][k].chargeLocations.begin(), s.tree[L][k].chargeLocations.end());
  }
  {
    AIFMM_REQUIRE((int)perm.size() == N, AIFMM_EINVAL, "leaves do not cover every unknown");
    std::vector<char> seen(N, 0);
    for (int id : perm) {
      AIFMM_REQUIRE(id >= 0 && id < N && !seen[id], AIFMM_EINVAL, "leaf charges are not a permutation");
      seen[id] = 1;
    }
  }
  lv.resize(L + 1);
  for (int j = j0; j <= L; ++j) {
    Level& V = lv[j];
    const int nb = s.nBoxesPerLevel[j];
    V.moff.resize(nb);
    V.loff.resize(nb);
    V.P2M.resize(nb);
    V.L2P.resize(nb);
    V.Mpack.resize(nb);
    V.soff.resize(nb);
    for (int k = 0; k < nb; ++k) {
      const DBox& B = s.tree[j][k];
      V.moff[k] = V.nm;
      V.loff[k] = V.nl;
      V.nm += B.P2M.r;
      V.nl += B.L2P.c;
      V.P2M[k] = B.P2M;
      V.L2P[k] = B.L2P;
    }
  }
  // the input of a box's P2M (and output of its L2P) is its leaf slice or its children's range
  for (int j = j0; j <= L; ++j)
    for (int k = 0; k < s.nBoxesPerLevel[j]; ++k) {
      int nin = 0, nout = 0;
      if (j == L) nin = nout = nx[k];
      else
        for (int c = 0; c < 8; ++c) {
          nin += lv[j + 1].P2M[8 * k + c].r;
          nout += lv[j + 1].L2P[8 * k + c].c;
        }
      const DMat& P = lv[j].P2M[k];
      const DMat& Q = lv[j].L2P[k];
      AIFMM_REQUIRE(P.r == 0 || P.c == nin, AIFMM_EINVAL, "P2M input size does not match the level below");
      AIFMM_REQUIRE(Q.c == 0 || Q.r == nout, AIFMM_EINVAL, "L2P output size does not match the level below");
    }
  // far field: M2L[k][l] for l in IL(k), side by side
  for (int j = j0; j <= L; ++j) {
    Level& V = lv[j];
    for (int k = 0; k < s.nBoxesPerLevel[j]; ++k) {
      DBox& B = s.tree[j][k];
      V.soff[k] = (int)V.sidx.size();
      std::vector<DMat> parts;
      for (int l : B.IL) {
        auto it = B.M2L.find(l);
        if (it == B.M2L.end() || it->second.size() == 0) continue;
        const DMat& m = it->second;
        AIFMM_REQUIRE(m.r == V.L2P[k].c && m.c == V.P2M[l].r, AIFMM_EINVAL, "M2L block shape");
        parts.push_back(m);
        for (int i = 0; i < m.c; ++i) V.sidx.push_back(V.moff[l] + i);
      }
      if (!parts.empty()) V.Mpack[k] = ops.hcatv(parts);
      for (auto& kv : B.M2L) kv.second = DMat();
    }
  }
  // near field at the leaves, self block included
  Ppack.resize(nLeaf);
  xsoff.resize(nLeaf);
  for (int k = 0; k < nLeaf; ++k) {
    DBox& B = s.tree[L][k];
    xsoff[k] = (int)xidx.size();
    std::vector<DMat> parts;
    for (int nn : B.NB) {
      auto it = B.P2P.find(nn);
      if (it == B.P2P.end() || it->second.size() == 0) continue;
      const DMat& m = it->second;
      AIFMM_REQUIRE(m.r == nx[k] && m.c == nx[nn], AIFMM_EINVAL, "P2P block shape");
      parts.push_back(m);
      for (int i = 0; i < m.c; ++i) xidx.push_back(xoff[nn] + i);
    }
    if (!parts.empty()) Ppack[k] = ops.hcatv(parts);
    for (auto& kv : B.P2P) kv.second = DMat();
  }
  sp.reset();  // the unpacked blocks go back to the pool
  dperm = upload(ctx, perm);
  dxidx = upload(ctx, xidx);
  dsidx.resize(L + 1);
  for (int j = j0; j <= L; ++j) dsidx[j] = upload(ctx, lv[j].sidx);
  for (int j = j0; j <= L; ++j)
    for (int k = 0; k < (int)lv[j].P2M.size(); ++k) {
      const double e = (double)lv[j].P2M[k].size() + lv[j].L2P[k].size() + lv[j].Mpack[k].size();
      bytes += 16.0 * e;
      flopsPerColumn += 8.0 * e;
    }
  for (const DMat& m : Ppack) {
    bytes += 16.0 * m.size();
    flopsPerColumn += 8.0 * m.size();
  }
  ops.sync();
}

H2Operator::Phase H2Operator::phase(const std::vector<SkinnyProblem>& ps) {
  Phase ph;
  std::vector<SkinnyProblem> kept;
  std::vector<SkinnyTile> tiles;
  for (const SkinnyProblem& p : ps) {
    if (p.m <= 0 || p.k <= 0) continue;
    const int pi = (int)kept.size();
    kept.push_back(p);
    for (int r0 = 0; r0 < p.m; r0 += SKINNY_ROWS) tiles.push_back({pi, r0});
  }
  ph.ntiles = (int)tiles.size();
  ph.probs = upload(ctx, kept);
  ph.tiles = upload(ctx, tiles);
  return ph;
}

static SkinnyProblem skinny(const DMat& a, const zd* b, int ldb, zd* c, int ldc, int accumulate) {
  SkinnyProblem q;
  q.A = a.p;
  q.lda = a.ld();
  q.B = b;
  q.ldb = ldb;
  q.C = c;
  q.ldc = ldc;
  q.m = a.r;
  q.k = a.c;
  q.accumulate = accumulate;
  return q;
}

H2Operator::Plan& H2Operator::plan(int nr) {
  auto it = plans_.find(nr);
  if (it != plans_.end()) return *it->second;
  auto P = std::make_unique<Plan>();
  P->nr = nr;
  const size_t z = sizeof(zd);
  P->Xt = DevBuf(ctx, z * (size_t)N * nr + 16);
  P->Yt = DevBuf(ctx, z * (size_t)N * nr + 16);
  P->SX = DevBuf(ctx, z * xidx.size() * nr + 16);
  P->M.resize(L + 1);
  P->Lc.resize(L + 1);
  P->S.resize(L + 1);
  P->up.resize(L + 1);
  P->m2l.resize(L + 1);
  P->down.resize(L + 1);
  for (int j = j0; j <= L; ++j) {
    P->M[j] = DevBuf(ctx, z * (size_t)lv[j].nm * nr + 16);
    P->Lc[j] = DevBuf(ctx, z * (size_t)lv[j].nl * nr + 16);
    P->S[j] = DevBuf(ctx, z * lv[j].sidx.size() * nr + 16);
  }
  zd* Xt = P->Xt.as<zd>();
  zd* Yt = P->Yt.as<zd>();
  for (int j = j0; j <= L; ++j) {
    const Level& V = lv[j];
    const int nb = (int)V.P2M.size();
    zd* Mj = P->M[j].as<zd>();
    zd* Lj = P->Lc[j].as<zd>();
    const int ldm = std::max(V.nm, 1), ldl = std::max(V.nl, 1), lds = std::max((int)V.sidx.size(), 1);
    std::vector<SkinnyProblem> up, m2l, down;
    for (int k = 0; k < nb; ++k) {
      const DMat& p2m = V.P2M[k];
      if (p2m.r > 0 && p2m.c > 0) {
        if (j == L) up.push_back(skinny(p2m, Xt + xoff[k], N, Mj + V.moff[k], ldm, 0));
        else
          up.push_back(skinny(p2m, P->M[j + 1].as<zd>() + lv[j + 1].moff[8 * k], std::max(lv[j + 1].nm, 1),
                              Mj + V.moff[k], ldm, 0));
      }
      if (V.Mpack[k].size() > 0) m2l.push_back(skinny(V.Mpack[k], P->S[j].as<zd>() + V.soff[k], lds, Lj + V.loff[k], ldl, 1));
      const DMat& l2p = V.L2P[k];
      if (j < L && l2p.r > 0 && l2p.c > 0)
        down.push_back(skinny(l2p, Lj + V.loff[k], ldl, P->Lc[j + 1].as<zd>() + lv[j + 1].loff[8 * k],
                              std::max(lv[j + 1].nl, 1), 1));
    }
    P->up[j] = phase(up);
    P->m2l[j] = phase(m2l);
    P->down[j] = phase(down);
  }
  std::vector<SkinnyProblem> ll, lp;
  const Level& VL = lv[L];
  for (int k = 0; k < (int)nx.size(); ++k) {
    const DMat& l2p = VL.L2P[k];
    if (l2p.r > 0 && l2p.c > 0)
      ll.push_back(skinny(l2p, P->Lc[L].as<zd>() + VL.loff[k], std::max(VL.nl, 1), Yt + xoff[k], N, 1));
    if (Ppack[k].size() > 0)
      lp.push_back(skinny(Ppack[k], P->SX.as<zd>() + xsoff[k], std::max((int)xidx.size(), 1), Yt + xoff[k], N, 1));
  }
  P->leafL2P = phase(ll);
  P->leafP2P = phase(lp);
  Plan& ref = *P;
  plans_[nr] = std::move(P);
  return ref;
}

void H2Operator::run(const Phase& p, int nr) {
  zgemm_skinny(ctx, p.probs.as<SkinnyProblem>(), p.tiles.as<SkinnyTile>(), p.ntiles, nr);
}

void H2Operator::apply(const zd* x, int ldx, zd* y, int ldy, int nr) {
  AIFMM_REQUIRE(nr >= 1, AIFMM_EINVAL, "no columns");
  AIFMM_REQUIRE(ldx >= N && ldy >= N, AIFMM_EINVAL, "leading dimension below N");
  AIFMM_CUDA(cudaSetDevice(ctx->device));
  const long before = thread_launch_count();
  for (int c0 = 0; c0 < nr; c0 += SKINNY_MAXNR)
    applyChunk(x + (size_t)c0 * ldx, ldx, y + (size_t)c0 * ldy, ldy, std::min(SKINNY_MAXNR, nr - c0));
  launchesPerApply = thread_launch_count() - before;
}

// Upward P2M, M2L per level, downward L2P, leaf L2P + near field, all in tree order.
void H2Operator::applyChunk(const zd* x, int ldx, zd* y, int ldy, int nr) {
  Plan& P = plan(nr);
  for (int j = j0; j <= L; ++j) zfill(ctx, P.Lc[j].as<zd>(), (size_t)lv[j].nl * nr, zmk(0, 0));
  zfill(ctx, P.Yt.as<zd>(), (size_t)N * nr, zmk(0, 0));
  zrows_gather(ctx, x, ldx, dperm.as<int>(), N, P.Xt.as<zd>(), N, nr);
  for (int j = L; j >= j0; --j) run(P.up[j], nr);
  for (int j = j0; j <= L; ++j) {
    const int ns = (int)lv[j].sidx.size();
    zrows_gather(ctx, P.M[j].as<zd>(), std::max(lv[j].nm, 1), dsidx[j].as<int>(), ns, P.S[j].as<zd>(), std::max(ns, 1),
                 nr);
    run(P.m2l[j], nr);
  }
  for (int j = j0; j < L; ++j) run(P.down[j], nr);
  run(P.leafL2P, nr);
  zrows_gather(ctx, P.Xt.as<zd>(), N, dxidx.as<int>(), (int)xidx.size(), P.SX.as<zd>(), std::max((int)xidx.size(), 1),
               nr);
  run(P.leafP2P, nr);
  zrows_scatter(ctx, P.Yt.as<zd>(), N, dperm.as<int>(), N, y, ldy, nr);
}

}  // namespace aifmm
