// GPU AIFMM solver.  Reference functions are cited as T:line for
// include/AIFMMTree2D_3D_memory_optimized.hpp of vaishna77/RCS.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>

#include "h2op.cuh"
#include "solver.cuh"

namespace aifmm {

static double wall() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
static const zd ONE = {1.0, 0.0}, ZERO = {0.0, 0.0}, MONE = {-1.0, 0.0};

// Grouped GEMMs issued inside the scope use the given precision.
struct GemmPrecisionScope {
  aifmm_ctx* c;
  int saved;
  GemmPrecisionScope(aifmm_ctx* ctx, int p) : c(ctx), saved(ctx->gemmPrecision) { c->gemmPrecision = p; }
  ~GemmPrecisionScope() { c->gemmPrecision = saved; }
};

// Adds the wall time of a scope to a phase counter; with phaseTiming the
// stream is drained on entry and exit so the time is the phase's own.
// Nested scopes (RRQR inside a recompression) count in both.
struct PhaseTimer {
  Solver& s;
  double& acc;
  double t0;
  PhaseTimer(Solver& so, double& a) : s(so), acc(a) {
    if (s.prm.phaseTiming) s.ops.sync();
    t0 = wall();
  }
  ~PhaseTimer() {
    if (s.prm.phaseTiming) cudaStreamSynchronize(s.ctx->stream);
    acc += wall() - t0;
  }
};

// ------------------------------------------------------------ setup, T:52-165
Solver::Solver(aifmm_kernel* k, const SolverParams& p, const double* xyz, const double* dom)
    : K(k), ctx(k->ctx), ops(k->ctx), prm(p) {
  N = k->geom.N;
  particles = xyz ? std::vector<double>(xyz, xyz + 3 * (size_t)N) : k->locations;
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < N; ++i)
    for (int q = 0; q < 3; ++q) {
      mn[q] = std::min(mn[q], particles[3 * i + q]);
      mx[q] = std::max(mx[q], particles[3 * i + q]);
    }
  if (dom)
    for (int q = 0; q < 3; ++q) {
      AIFMM_REQUIRE(dom[2 * q] <= mn[q] && dom[2 * q + 1] >= mx[q], AIFMM_EINVAL,
                    "the domain box does not contain every location");
      mn[q] = dom[2 * q];
      mx[q] = dom[2 * q + 1];
    }
  for (int q = 0; q < 3; ++q) {
    domain[2 * q] = mn[q];
    domain[2 * q + 1] = mx[q];
  }
  fillInTolerance = std::pow(10, -1.0 * prm.tol_pow);
  if (prm.drop_pow > 0) fillInTolerance = std::pow(10, -1.0 * prm.drop_pow);
  if (prm.drop_pow < 0) fillInTolerance = std::numeric_limits<double>::infinity();
  L = std::max({mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]});
  AIFMM_REQUIRE(prm.leafSize > 0, AIFMM_EINVAL, "leaf size must be positive");
  const int q = N / prm.leafSize;
  nLevels = (q <= 0) ? 2 : std::max(2, int(std::floor(std::log(q) / std::log(8))));
  if (prm.nLevelsInput > 0) nLevels = prm.nLevelsInput;
  AIFMM_REQUIRE(nLevels < 9, AIFMM_EINVAL, "too many levels for the dense level arrays");
  eta = std::sqrt(3) * 2;
  nBoxesPerLevel.push_back(1);
  boxSideLength.push_back(L);
  for (int j = 1; j <= nLevels; ++j) {
    nBoxesPerLevel.push_back(nChild * nBoxesPerLevel[j - 1]);
    boxSideLength.push_back(0.5 * boxSideLength[j - 1]);
  }
  for (int j = 0; j < 64; ++j) fillin_rankVec[j] = 0;
  int temp = 5, i = 0;
  for (int j = nLevels; j >= 2; --j) {
    fillin_rankVec[j] = temp;
    if (++i % 3 == 0) temp += 5;
  }
}

void Solver::createTree() {
  tree.assign(nLevels + 1, {});
  for (int j = 0; j <= nLevels; ++j) tree[j].resize(nBoxesPerLevel[j]);
}

void Solver::assignCenters() {  // T:425-463
  DBox& r = tree[0][0];
  for (int q = 0; q < 3; ++q) r.center[q] = (domain[2 * q] + domain[2 * q + 1]) / 2.0;
  static const int sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
  static const int sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
  static const int sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
  for (int j = 0; j < nLevels; ++j) {
    const double shift = 0.5 * boxSideLength[j + 1];
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
      const double* c = tree[j][k].center;
      for (int ch = 0; ch < 8; ++ch) {
        double* cc = tree[j + 1][8 * k + ch].center;
        cc[0] = sx[ch] < 0 ? c[0] - shift : c[0] + shift;
        cc[1] = sy[ch] < 0 ? c[1] - shift : c[1] + shift;
        cc[2] = sz[ch] < 0 ? c[2] - shift : c[2] + shift;
      }
    }
  }
}

void Solver::assignInteractions() {  // T:266-331
  tree[0][0].NB.push_back(0);
  for (int j = 0; j < nLevels; ++j)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k)
      for (int c = 0; c < nChild; ++c) {
        const int child = nChild * k + c;
        for (int nn : tree[j][k].NB)
          for (int cc = 0; cc < nChild; ++cc) {
            const int other = nn * nChild + cc;
            const double* a = tree[j + 1][child].center;
            const double* b = tree[j + 1][other].center;
            const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
            const double d = std::sqrt(dx * dx + dy * dy + dz * dz);
            const double etaLocal = (j + 1 == nLevels) ? eta / 2.0 : eta;
            if (d > etaLocal * boxSideLength[j + 1] + boxSideLength[nLevels] / 2.0) tree[j + 1][child].IL.push_back(other);
            else tree[j + 1][child].NB.push_back(other);
          }
      }
  bool found = false;
  for (int j = 0; j <= nLevels && !found; ++j)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k)
      if (!tree[j][k].IL.empty()) {
        startLevel = j;
        found = true;
        break;
      }
}

void Solver::assignCharges() {  // T:576-668, the binning on the GPU
  std::vector<double> centers;
  for (int j = 0; j < nLevels; ++j)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) centers.insert(centers.end(), tree[j][k].center, tree[j][k].center + 3);
  std::vector<int> start;
  const std::vector<int> order = bin_points_gpu(ctx, particles, centers, nLevels, start);
  for (int k = 0; k < nBoxesPerLevel[nLevels]; ++k)
    tree[nLevels][k].chargeLocations.assign(order.begin() + start[k], order.begin() + start[k + 1]);
  for (int j = nLevels - 1; j >= 0; j--)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
      auto& cl = tree[j][k].chargeLocations;
      cl.clear();
      for (int c = 0; c < nChild; ++c) {
        auto& v = tree[j + 1][nChild * k + c].chargeLocations;
        cl.insert(cl.end(), v.begin(), v.end());
      }
    }
}

// Dense tiles K(rows, cols) for many (rows, cols) pairs in one launch.
void Solver::gatherBlocks(const std::vector<std::vector<int>*>& rows, const std::vector<std::vector<int>*>& cols,
                          std::vector<DMat*>& outs) {
  std::vector<int> ids;
  std::vector<std::pair<size_t, size_t>> off;
  for (size_t b = 0; b < rows.size(); ++b) {
    *outs[b] = ops.alloc((int)rows[b]->size(), (int)cols[b]->size());
    off.push_back({ids.size(), ids.size() + rows[b]->size()});
    ids.insert(ids.end(), rows[b]->begin(), rows[b]->end());
    ids.insert(ids.end(), cols[b]->begin(), cols[b]->end());
  }
  if (ids.empty()) return;
  DevBuf dids = upload(ctx, ids);
  std::vector<GatherBlock> blocks;
  std::vector<long> start;
  long total = 0;
  for (size_t b = 0; b < rows.size(); ++b) {
    if (outs[b]->size() == 0) continue;
    GatherBlock g;
    g.rows = dids.as<int>() + off[b].first;
    g.cols = dids.as<int>() + off[b].second;
    g.out = outs[b]->p;
    g.nr = outs[b]->r;
    g.nc = outs[b]->c;
    g.ld = outs[b]->ld();
    g.pad = 0;
    blocks.push_back(g);
    start.push_back(total);
    total += (long)g.nr * g.nc;
  }
  if (blocks.empty()) return;
  DevBuf db = upload(ctx, blocks), ds = upload(ctx, start);
  launch_batched_gather(K->geom, db.as<GatherBlock>(), ds.as<long>(), (int)blocks.size(), total, 0, ctx->stream);
  stats.kernels++;
}

// ------------------------------------------------------------ skeletons, T:917-1256
RankFeatures Solver::rankFeatures(int j, int k, int nr, int nc) const {
  const DBox& B = tree[j][k];
  double d = 0.0;
  for (int kIL : B.IL) {
    const double* a = B.center;
    const double* b = tree[j][kIL].center;
    d += std::sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
  }
  RankFeatures f;
  f.f[0] = B.IL.empty() ? 0.0f : (float)(d / B.IL.size() / boxSideLength[j]);
  f.f[1] = K->geom.efie ? (float)(K->geom.ge.kappa * boxSideLength[j]) : 0.0f;
  f.f[2] = (float)std::log2(1.0 + nr);
  f.f[3] = (float)std::log2(1.0 + nc);
  f.f[4] = (float)j;
  f.f[5] = (j == nLevels) ? 1.0f : 0.0f;
  return f;
}

void Solver::runACA(int j, bool incoming) {
  struct Item {
    int k;
    std::vector<int> boxA, ILn;
    int nr, nc, rmax, rmax0;
    RankFeatures feat;
  };
  const double tAca0 = wall();
  std::vector<Item> items;
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    DBox& B = tree[j][k];
    Item it;
    it.k = k;
    // own points: leaf charges, or the children's skeletons
    if (j == nLevels) it.boxA = B.chargeLocations;
    else
      for (int c = 0; c < nChild; ++c) {
        auto& v = incoming ? tree[j + 1][nChild * k + c].in_check : tree[j + 1][nChild * k + c].out_charge;
        it.boxA.insert(it.boxA.end(), v.begin(), v.end());
      }
    for (int kIL : B.IL) {
      if (j == nLevels) {
        auto& v = tree[j][kIL].chargeLocations;
        it.ILn.insert(it.ILn.end(), v.begin(), v.end());
      } else
        for (int c = 0; c < nChild; ++c) {
          auto& v = incoming ? tree[j + 1][nChild * kIL + c].out_charge : tree[j + 1][nChild * kIL + c].in_check;
          it.ILn.insert(it.ILn.end(), v.begin(), v.end());
        }
    }
    // incoming: rows = box, cols = IL;  outgoing: rows = IL, cols = box
    const int nr = (int)(incoming ? it.boxA.size() : it.ILn.size());
    const int nc = (int)(incoming ? it.ILn.size() : it.boxA.size());
    if (nr > 0 && nc > 0) {
      it.nr = nr;
      it.nc = nc;
      it.rmax = std::min(std::min(nr, nc), 128);
      items.push_back(std::move(it));
    } else if (incoming && nc == 0) {
      B.ILActive = false;
      B.in_check = it.boxA;
    } else if (!incoming && nr == 0) {
      B.ILActive = false;
      B.out_charge = it.boxA;
    }
  }
  // The workspace of a problem holds rmax rank-1 terms.  With a rank model on
  // the context, its prediction (with a margin) sizes rmax instead of the
  // fixed bound; either way a problem whose adaptive ACA needs more terms is
  // rerun with twice the bound (the plain ACA decides the rank).
  {
    std::vector<RankFeatures> feats(items.size());
    for (size_t q = 0; q < items.size(); ++q) feats[q] = rankFeatures(j, items[q].k, items[q].nr, items[q].nc);
    if (ctx->rankModel && !items.empty()) {
      std::vector<float> y;
      mlp_infer(ctx->rankModel.get(), feats, y);
      for (size_t q = 0; q < items.size(); ++q) {
        const double pred = std::max(0.0, std::exp2((double)y[q]) - 1.0);
        const int r = std::max(16, (int)std::ceil(pred * ctx->rankMargin) + 8);
        items[q].rmax = std::min({r, std::min(items[q].nr, items[q].nc), 1024});
      }
    }
    for (size_t q = 0; q < items.size(); ++q) {
      items[q].feat = feats[q];
      items[q].rmax0 = items[q].rmax;
    }
  }
  const double tol = std::pow(10, -prm.tol_pow);
  std::vector<Item*> pending;
  for (auto& it : items) pending.push_back(&it);
  while (!pending.empty()) {
    // one launch per chunk that fits the workspace budget
    std::vector<Item*> chunk;
    size_t bytes = 0;
    while (!pending.empty()) {
      Item* it = pending.front();
      const size_t need = (size_t)it->rmax * (it->nr + it->nc) * sizeof(zd) * 2 + (it->nr + it->nc) * 9 + 4096;
      if (!chunk.empty() && bytes + need > prm.aca_budget) break;
      chunk.push_back(it);
      bytes += need;
      pending.erase(pending.begin());
    }
    std::vector<int> ids;
    std::vector<size_t> offs;
    for (Item* it : chunk) {
      offs.push_back(ids.size());
      const auto& rows = incoming ? it->boxA : it->ILn;
      const auto& cols = incoming ? it->ILn : it->boxA;
      ids.insert(ids.end(), rows.begin(), rows.end());
      ids.insert(ids.end(), cols.begin(), cols.end());
    }
    DevBuf dids = upload(ctx, ids);
    std::vector<DevBuf> ws;
    std::vector<ACAProblem> probs;
    const int nq = (int)chunk.size();
    DevBuf dint(ctx, sizeof(int) * 2 * nq);
    for (int q = 0; q < nq; ++q) {
      Item* it = chunk[q];
      const int nP = (it->nr < it->nc) ? it->nr : it->nc, nS = (it->nr < it->nc) ? it->nc : it->nr;
      const size_t zU = (size_t)it->rmax * nP, zV = (size_t)it->rmax * nS;
      const size_t zAc = (size_t)it->nr * it->rmax, zAr = (size_t)it->rmax * it->nc;
      ws.emplace_back(ctx, sizeof(zd) * (zU + zV + zAc + zAr) + (it->nr + it->nc) + sizeof(int) * 2 * it->rmax + 64);
      stats.aca_ws_bytes += (double)ws.back().bytes;
      char* base = (char*)ws.back().p;
      ACAProblem P;
      P.rows = dids.as<int>() + offs[q];
      P.cols = dids.as<int>() + offs[q] + it->nr;
      P.nr = it->nr;
      P.nc = it->nc;
      P.rmax = it->rmax;
      P.U = (zd*)base;
      P.V = P.U + zU;
      P.Ac = P.V + zV;
      P.Ar = P.Ac + zAc;
      P.rowBases = (int*)(P.Ar + zAr);
      P.colBases = P.rowBases + it->rmax;
      P.used = (unsigned char*)(P.colBases + it->rmax);
      P.rank = dint.as<int>() + 2 * q;
      P.status = dint.as<int>() + 2 * q + 1;
      probs.push_back(P);
    }
    launch_aca(ctx, K->geom, probs, tol);
    stats.kernels++;
    stats.nACA += nq;
    stats.nACALaunches++;
    std::vector<int> rs(2 * nq);
    AIFMM_CUDA(cudaMemcpyAsync(rs.data(), dint.p, sizeof(int) * 2 * nq, cudaMemcpyDeviceToHost, ctx->stream));
    ops.sync();
    for (int q = 0; q < nq; ++q) {
      Item* it = chunk[q];
      const int rank = rs[2 * q], status = rs[2 * q + 1];
      if (status != 0) {  // workspace rank bound reached: rerun this box with twice the bound
        AIFMM_REQUIRE(it->rmax < std::min(it->nr, it->nc) && it->rmax < 1024, AIFMM_EOVERFLOW,
                      "ACA rank exceeds the workspace bound");
        it->rmax = std::min(std::min(it->nr, it->nc), std::min(2 * it->rmax, 1024));
        stats.nACARetry++;
        pending.push_back(it);
        continue;
      }
      acaLog.push_back({it->feat, it->rmax0, rank});
      DBox& B = tree[j][it->k];
      std::vector<int> rb(rank), cb(rank);
      if (rank > 0) {
        AIFMM_CUDA(cudaMemcpyAsync(rb.data(), probs[q].rowBases, sizeof(int) * rank, cudaMemcpyDeviceToHost, ctx->stream));
        AIFMM_CUDA(cudaMemcpyAsync(cb.data(), probs[q].colBases, sizeof(int) * rank, cudaMemcpyDeviceToHost, ctx->stream));
      }
      if (incoming) {
        // Ac = nr x rank original columns
        DMat Ac = ops.alloc(it->nr, rank);
        if (Ac.size())
          zcopy_grouped(ctx, {{probs[q].Ac, Ac.p, it->nr, rank, it->nr, Ac.ld(), 0, ONE}});
        B.Ac = Ac;
      } else {
        DMat Ar = ops.alloc(rank, it->nc);
        if (Ar.size())
          zcopy_grouped(ctx, {{probs[q].Ar, Ar.p, rank, it->nc, it->rmax, Ar.ld(), 0, ONE}});
        B.Ar = Ar;
      }
      ops.sync();
      if (rank > 0) {
        const auto& rows = incoming ? it->boxA : it->ILn;
        const auto& cols = incoming ? it->ILn : it->boxA;
        auto& chk = incoming ? B.in_check : B.out_check;
        auto& chg = incoming ? B.in_charge : B.out_charge;
        for (int r = 0; r < rank; ++r) chk.push_back(rows[rb[r]]);
        for (int c = 0; c < rank; ++c) chg.push_back(cols[cb[c]]);
      }
    }
  }
  stats.t_aca += wall() - tAca0;
}

static void truncateTo(std::vector<int>& v, size_t n) {
  if (v.size() > n) v.resize(n);
}

void Solver::getL2PP2MBox(int j, int k) {  // T:681-732
  DBox& B = tree[j][k];
  if (B.in_check.size() < B.out_charge.size()) {
    truncateTo(B.out_check, B.in_check.size());
    truncateTo(B.out_charge, B.in_check.size());
  } else {
    truncateTo(B.in_check, B.out_charge.size());
    truncateTo(B.in_charge, B.out_charge.size());
  }
  const int nin = (int)B.in_check.size(), nout = (int)B.out_check.size();
  if (B.ILActive) {
    DMat temp1 = ops.block(B.Ac, 0, 0, B.Ac.r, nin);
    B.L2P = ops.zeros(B.Ac.r, nin);
    if (nin > 0) {
      DMat D1;
      std::vector<DMat*> o{&D1};
      gatherBlocks({&B.in_check}, {&B.in_charge}, o);
      DLU f = ops.factor(ops.adj(D1));
      B.L2P = ops.adj(ops.solve(f, ops.adj(temp1)));
    }
    DMat temp2 = ops.block(B.Ar, 0, 0, nout, B.Ar.c);
    B.P2M = ops.alloc(nout, B.Ar.c);
    if (nout > 0) {
      DMat D2;
      std::vector<DMat*> o{&D2};
      gatherBlocks({&B.out_check}, {&B.out_charge}, o);
      DLU f = ops.factor(D2);
      B.P2M = ops.solve(f, temp2);
    }
  } else {
    B.L2P = ops.ident(nin, ONE);
    const int no = (int)B.out_charge.size();
    B.P2M = ops.ident(no, ONE);
  }
  if (B.Ac.size() > 0) B.maxPivot_L2P = ops.maxColNorm(ops.block(B.Ac, 0, 0, B.Ac.r, nin));
  if (B.Ar.size() > 0) B.maxPivot_P2M = ops.maxColNorm(ops.adj(ops.block(B.Ar, 0, 0, nout, B.Ar.c)));
}

void Solver::getNodesLevel(int j) {
  runACA(j, true);
  runACA(j, false);
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) getL2PP2MBox(j, k);
}

void Solver::assembleM2L() {  // T:1258-1273
  std::vector<std::vector<int>*> R, C;
  std::vector<DMat*> O;
  for (int j = startLevel; j <= nLevels; ++j)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k)
      for (int kIL : tree[j][k].IL) {
        R.push_back(&tree[j][k].in_check);
        C.push_back(&tree[j][kIL].out_charge);
        O.push_back(&tree[j][k].M2L[kIL]);
      }
  gatherBlocks(R, C, O);
}

void Solver::initP2PLeaf() {  // T:3372-3386
  const int j = nLevels;
  std::vector<std::vector<int>*> R, C;
  std::vector<DMat*> O;
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    for (int nn : tree[j][k].NB)
      if (nn != k) {
        R.push_back(&tree[j][k].chargeLocations);
        C.push_back(&tree[j][nn].chargeLocations);
        O.push_back(&tree[j][k].P2P[nn]);
      }
    R.push_back(&tree[j][k].chargeLocations);
    C.push_back(&tree[j][k].chargeLocations);
    O.push_back(&tree[j][k].P2P[k]);
  }
  gatherBlocks(R, C, O);
}

void Solver::build() {  // AIFMM.cpp:7-93
  const double t0 = wall();
  AIFMM_CUDA(cudaSetDevice(ctx->device));
  createTree();
  assignCenters();
  assignInteractions();
  assignCharges();
  for (int j = nLevels; j >= startLevel; --j) getNodesLevel(j);
  assembleM2L();
  for (int j = startLevel; j <= nLevels; ++j)
    for (DBox& B : tree[j]) {  // free_charge_and_checkPoints, T:1275-1284
      B.out_charge.clear();
      B.in_check.clear();
      B.Ar = DMat();
      B.Ac = DMat();
    }
  for (int j = startLevel; j <= nLevels; ++j)  // initialise_phase, T:3354-3370
    for (DBox& B : tree[j]) {
      B.NumMultipoles = B.P2M.r;
      B.NumLocals = B.L2P.c;
    }
  initP2PLeaf();
  ops.sync();
  stats.t_assemble = wall() - t0;
}

// ------------------------------------------------------------ non-leaf P2P, T:3413-3504
void Solver::initP2PNonLeaf(int j) {
  opprof::Scope prof_fn_("nonleaf_p2p", ctx->stream);
  PhaseTimer pt(*this, stats.t_nonleaf);
  std::vector<CopyProblem> cps;
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    DBox& B = tree[j][k];
    for (int nn : B.NB) {
      if (nn == k) continue;
      int n_rows = 0, n_cols = 0;
      for (int a = 0; a < nChild; ++a) {
        int t = 0;
        for (int b = 0; b < nChild; ++b) t += tree[j + 1][nChild * k + a].M2L[nChild * nn + b].c;
        n_cols = std::max(n_cols, t);
      }
      for (int b = 0; b < nChild; ++b) {
        int t = 0;
        for (int a = 0; a < nChild; ++a) t += tree[j + 1][nChild * k + a].M2L[nChild * nn + b].r;
        n_rows = std::max(n_rows, t);
      }
      DMat P = ops.zeros(n_rows, n_cols);
      int ri = 0, ci = 0;
      for (int a = 0; a < nChild; ++a) {
        for (int b = 0; b < nChild; ++b) {
          const DMat& m = tree[j + 1][nChild * k + a].M2L[nChild * nn + b];
          if (m.size() > 0) {
            AIFMM_REQUIRE(ri + m.r <= P.r && ci + m.c <= P.c, AIFMM_EINVAL, "non-leaf P2P placement");
            cps.push_back({m.p, P.p + (size_t)ci * P.ld() + ri, m.r, m.c, m.ld(), P.ld(), 0, ONE});
            ci += m.c;
          }
        }
        ri += tree[j + 1][nChild * k + a].M2L[nChild * nn + 0].r;
        ci = 0;
      }
      B.P2P[nn] = P;
    }
    int n_rows = 0, n_cols = 0;
    for (int a = 0; a < nChild; ++a) n_rows += tree[j + 1][nChild * k + a].NumLocals;
    for (int b = 0; b < nChild; ++b) n_cols += tree[j + 1][nChild * k + b].NumMultipoles;
    DMat P = ops.zeros(n_rows, n_cols);
    int ri = 0, ci = 0;
    for (int a = 0; a < nChild; ++a) {
      for (int b = 0; b < nChild; ++b) {
        const DBox& ca = tree[j + 1][nChild * k + a];
        const DBox& cb = tree[j + 1][nChild * k + b];
        const DMat& m = tree[j + 1][nChild * k + a].M2L[nChild * k + b];
        AIFMM_REQUIRE(m.r == ca.NumLocals && m.c == cb.NumMultipoles, AIFMM_EINVAL, "non-leaf self P2P block shape");
        if (m.size()) cps.push_back({m.p, P.p + (size_t)ci * P.ld() + ri, m.r, m.c, m.ld(), P.ld(), 0, ONE});
        ci += cb.NumMultipoles;
      }
      ri += tree[j + 1][nChild * k + a].NumLocals;
      ci = 0;
    }
    B.P2P[k] = P;
  }
  zcopy_grouped(ctx, cps);
}

void Solver::deleteM2L(int j) {
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    for (int nn : tree[j][k].NB) {
      if (nn == k) continue;
      for (int a = 0; a < nChild; ++a)
        for (int b = 0; b < nChild; ++b)
          if (tree[j + 1][nChild * k + a].M2L[nChild * nn + b].size() > 0)
            tree[j + 1][nChild * k + a].M2L[nChild * nn + b] = DMat();
    }
    for (int a = 0; a < nChild; ++a)
      for (int b = 0; b < nChild; ++b) tree[j + 1][nChild * k + a].M2L[nChild * k + b] = DMat();
  }
}

// ------------------------------------------------------------ recompression
bool Solver::wellSeparated(int j, int k, int l) const {  // T:4044-4055
  if (k == l) return false;
  for (int nn : tree[j][k].NB)
    if (l == nn) return false;
  return true;
}

// RRQR of A = [old basis (partition columns) | fill-in] (rrqr.cpp:98-182),
// for several independent matrices at once: one launch of the column-pivoted
// QR kernels for all of them and one read-back of their ranks, where one
// call each would pay a launch chain and a host round trip apiece.  Each
// matrix's arithmetic is that of a call on its own, bit for bit.
//
// When the old basis has orthonormal columns (orthoPanel), partition 1 of the
// reference keeps every one of them -- each pivot is the unit norm of a
// column orthogonal to the ones before, never below tol1 <= 1 -- so its
// Householder pass only re-expresses the same span.  The shortcut keeps the
// old basis as it is, projects the fill-in onto its orthogonal complement
// (classical Gram-Schmidt, twice) and runs partition 2 on the projection with
// the reference's step bound min(m - partition, fill-in columns); ranks,
// pivots and spans are those of the full pass, the basis of the old span is
// the identity instead of a Householder rotation of it, and maxPivot of an
// empty partition 2 is the unit norm of the first old column.
void Solver::rrqrBatch(const std::vector<RRQRJob*>& jobs) {
  opprof::Scope prof_fn_("rrqr_total", ctx->stream);
  PhaseTimer pt(*this, stats.t_rrqr);
  struct Run {
    RRQRJob* job;
    DMat R;       // working copy, destroyed
    int partition, p2cap;
    DMat Q1;      // shortcut: view of the old basis
    bool shortcut;
  };
  std::vector<Run> runs;
  for (RRQRJob* J : jobs) {
    const int m = J->A.r, n = J->A.c;
    stats.nRRQR++;
    J->prefix = false;
    if (!(J->orthoPanel && prm.orthoShortcut && J->partition > 0 && J->partition <= m)) {
      runs.push_back({J, ops.copy(J->A), J->partition, -1, DMat(), false});
      continue;
    }
    stats.nRRQRShort++;
    J->prefix = true;  // Q_trunc = [old basis | new columns]
    const int r = J->partition, nf = n - r;
    DMat Q1;
    Q1.buf = J->A.buf;
    Q1.p = J->A.p;
    Q1.r = m;
    Q1.c = r;
    if (nf == 0 || m == r) {
      J->maxPivot = 1.0;
      J->Q = ops.copy(Q1);
      continue;
    }
    DMat F = ops.block(J->A, 0, r, m, nf);
    // classical Gram-Schmidt twice: the second pass restores orthogonality to
    // rounding.  One pass is not enough even for the mixed path's
    // preconditioner: a fill-in mostly inside the old span leaves a small
    // remainder whose non-orthogonal part the normalisation amplifies, and
    // the partial-identity basis changes assume orthonormal columns.
    for (int pass = 0; pass < 2; ++pass) {
      const DMat C = ops.mul(Q1, OP_C, F, OP_N);
      GemmBatch g;
      g.add(F, Q1, OP_N, C, OP_N, MONE, ONE);
      g.flush(ctx);
    }
    runs.push_back({J, F, 0, m - r, Q1, true});
  }
  if (runs.empty()) return;
  opprof::Scope prof_("rrqr_kernels", ctx->stream);
  constexpr size_t kOut = 64;  // rank, maxPivot, istate[8], dstate[2] of one problem
  DevBuf out(ctx, kOut * runs.size());
  std::vector<DevBuf> H(runs.size()), Q(runs.size()), nsq(runs.size()), perm(runs.size());
  std::vector<RRQRProblem> probs(runs.size());
  for (size_t i = 0; i < runs.size(); ++i) {
    const Run& u = runs[i];
    const int m = u.R.r, n = u.R.c;
    const int hs = std::min(m, n) + 1;
    H[i].alloc(ctx, sizeof(zd) * (size_t)m * hs + 16);
    Q[i].alloc(ctx, sizeof(zd) * (size_t)m * hs + 16);
    nsq[i].alloc(ctx, sizeof(double) * n + 8);
    perm[i].alloc(ctx, sizeof(int) * n + 8);
    char* o = (char*)out.p + kOut * i;
    RRQRProblem& P = probs[i];
    P.R = u.R.p;
    P.m = m;
    P.n = n;
    P.partition = u.partition;
    P.tol1 = std::pow(10.0, -prm.tol_pow);
    P.tol2 = std::pow(10.0, -prm.fillin_tol);
    P.inputPivot = u.job->inputPivot;
    P.fillInRank = u.job->fillRank;
    P.realMode = prm.realMode;
    P.H = H[i].as<zd>();
    P.nsq = nsq[i].as<double>();
    P.perm = perm[i].as<int>();
    P.Q = Q[i].as<zd>();
    P.rank = (int*)o;
    P.maxPivot = (double*)(o + 8);
    P.istate = (int*)(o + 16);
    P.dstate = (double*)(o + 48);  // after the 8 ints of istate
    P.p2cap = u.p2cap;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (gemm_profile_on()) {
    AIFMM_CUDA(cudaEventCreate(&e0));
    AIFMM_CUDA(cudaEventCreate(&e1));
    AIFMM_CUDA(cudaEventRecord(e0, ctx->stream));
  }
  launch_rrqr_split(ctx, probs);
  if (gemm_profile_on()) {
    AIFMM_CUDA(cudaEventRecord(e1, ctx->stream));
    device_span_record(e0, e1, "rrqr:" + opprof::path(), 0.0);
  }
  stats.kernels += 4 * (long)runs.size();
  std::vector<char> h(kOut * runs.size());
  AIFMM_CUDA(cudaMemcpyAsync(h.data(), out.p, h.size(), cudaMemcpyDeviceToHost, ctx->stream));
  ops.sync();
  std::vector<CopyProblem> cps;
  for (size_t i = 0; i < runs.size(); ++i) {
    const Run& u = runs[i];
    RRQRJob* J = u.job;
    const int m = u.R.r, n = u.R.c;
    int rank;
    double mp;
    std::memcpy(&rank, h.data() + kOut * i, sizeof(int));
    std::memcpy(&mp, h.data() + kOut * i + 8, sizeof(double));
    AIFMM_REQUIRE(rank != -2, AIFMM_ETIMEOUT, "RRQR: a bounded grid-barrier wait ran out");
    AIFMM_REQUIRE(rank >= 0 && rank <= std::min(m, n), AIFMM_EINVAL, "RRQR rank out of range");
    J->maxPivot = mp;
    if (!u.shortcut) {
      J->Q = ops.alloc(m, rank);
      if (rank > 0) cps.push_back({Q[i].as<zd>(), J->Q.p, m, rank, m, J->Q.ld(), 0, ONE});
    } else {
      const int r = u.Q1.c;
      J->Q = ops.alloc(m, r + rank);
      cps.push_back({u.Q1.p, J->Q.p, m, r, u.Q1.ld(), J->Q.ld(), 0, ONE});
      if (rank > 0) cps.push_back({Q[i].as<zd>(), J->Q.p + (size_t)r * J->Q.ld(), m, rank, m, J->Q.ld(), 0, ONE});
    }
  }
  zcopy_grouped(ctx, cps);
}

void Solver::resizeRows(const std::vector<DMat*>& blocks, int rows) {
  std::vector<CopyProblem> cps;
  std::vector<DMat> keep;  // the old blocks stay alive until the copy is enqueued
  std::vector<std::pair<int, int>> shapes;
  for (DMat* b : blocks) shapes.push_back({rows, b->c});
  std::vector<DMat> fresh = ops.allocMany(shapes);
  for (size_t q = 0; q < blocks.size(); ++q) {
    DMat* b = blocks[q];
    DMat nw = fresh[q];
    const int kept = std::min(rows, b->r);
    if (kept > 0 && b->c > 0) cps.push_back({b->p, nw.p, kept, b->c, b->ld(), nw.ld(), 0, ONE});
    if (rows > kept && b->c > 0) cps.push_back({nullptr, nw.p + kept, rows - kept, b->c, 1, nw.ld(), 0, ONE});
    keep.push_back(*b);
    *b = nw;
  }
  zcopy_grouped(ctx, cps);
}

void Solver::resizeCols(const std::vector<DMat*>& blocks, int cols) {
  std::vector<CopyProblem> cps;
  std::vector<DMat> keep;
  std::vector<std::pair<int, int>> shapes;
  for (DMat* b : blocks) shapes.push_back({b->r, cols});
  std::vector<DMat> fresh = ops.allocMany(shapes);
  for (size_t q = 0; q < blocks.size(); ++q) {
    DMat* b = blocks[q];
    DMat nw = fresh[q];
    const int kept = std::min(cols, b->c);
    if (kept > 0 && b->r > 0) cps.push_back({b->p, nw.p, b->r, kept, b->ld(), nw.ld(), 0, ONE});
    if (cols > kept && b->r > 0)
      cps.push_back({nullptr, nw.p + (size_t)kept * nw.ld(), b->r, cols - kept, 1, nw.ld(), 0, ONE});
    keep.push_back(*b);
    *b = nw;
  }
  zcopy_grouped(ctx, cps);
}

void Solver::updateOtherM2LsAtK(int j, int k, int b, const DMat& nL2P, bool prefix) {  // T:3159-3188
  opprof::Scope prof_("upd_m2l_k", ctx->stream);
  DBox& B = tree[j][k];
  std::vector<DMat*> blocks;
  for (auto& kv : B.P2L) blocks.push_back(&B.P2L[kv.first]);
  for (int kIL : B.IL)
    if (kIL != b) blocks.push_back(&B.M2L[kIL]);
  for (int kN : B.NB)
    if (kN != k && tree[j][kN].Eliminated && B.Eliminated) blocks.push_back(&B.M2L[kN]);
  if (B.Eliminated) blocks.push_back(&B.M2L[k]);
  if (prefix) {  // nL2P^H L2P = [I; 0] (or its first rows): keep rows, pad with zeros
    resizeRows(blocks, nL2P.c);
    return;
  }
  const DMat T = ops.mul(nL2P, OP_C, B.L2P, OP_N);
  GemmBatch g;
  std::vector<DMat> keep;  // old blocks stay alive until the batched GEMM that reads them is launched
  std::vector<std::pair<int, int>> shapes;
  for (DMat* old : blocks) shapes.push_back({T.r, old->c});
  std::vector<DMat> fresh = ops.allocMany(shapes);
  for (size_t q = 0; q < blocks.size(); ++q) {
    DMat* old = blocks[q];
    keep.push_back(*old);
    DMat nw = fresh[q];
    if (T.c == 0) nw = ops.zeros(T.r, old->c);
    else g.add(nw, T, OP_N, *old, OP_N, ONE, ZERO);
    *old = nw;
  }
  g.flush(ctx);
}

void Solver::updateOtherM2LsAtB(int j, int k, int b, const DMat& nP2Mt, bool prefix) {  // T:3252-3288
  opprof::Scope prof_("upd_m2l_b", ctx->stream);
  DBox& Bb = tree[j][b];
  std::vector<DMat*> blocks;
  for (auto& kv : Bb.P2L) blocks.push_back(&tree[j][kv.first].M2P[b]);
  for (int kIL : Bb.IL)
    if (kIL != k) blocks.push_back(&tree[j][kIL].M2L[b]);
  for (int kN : Bb.NB)
    if (kN != b && tree[j][kN].Eliminated && Bb.Eliminated) blocks.push_back(&tree[j][kN].M2L[b]);
  if (Bb.Eliminated) blocks.push_back(&Bb.M2L[b]);
  if (prefix) {  // P2M nP2Mt = [I | 0] (or its first columns): keep columns, pad with zeros
    resizeCols(blocks, nP2Mt.c);
    return;
  }
  const DMat S = ops.mul(Bb.P2M, OP_N, nP2Mt, OP_N);
  GemmBatch g;
  std::vector<DMat> keep;
  std::vector<std::pair<int, int>> shapes;
  for (DMat* old : blocks) shapes.push_back({old->r, S.c});
  std::vector<DMat> fresh = ops.allocMany(shapes);
  for (size_t q = 0; q < blocks.size(); ++q) {
    DMat* old = blocks[q];
    keep.push_back(*old);
    DMat nw = fresh[q];
    if (S.r == 0) nw = ops.zeros(old->r, S.c);
    else g.add(nw, *old, OP_N, S, OP_N, ONE, ZERO);
    *old = nw;
  }
  g.flush(ctx);
}

void Solver::updateParentL2P(int j, int k, const DMat& nL2P, bool prefix) {  // T:3290-3314
  opprof::Scope prof_("upd_parent_l2p", ctx->stream);
  const int kP = k / nChild, c_k = k % nChild;
  DMat& PL = tree[j - 1][kP].L2P;
  std::vector<DMat> U(nChild);
  int ri = 0;
  for (int c = 0; c < nChild; ++c) {
    U[c] = ops.block(PL, ri, 0, tree[j][kP * nChild + c].NumLocals, PL.c);
    ri += tree[j][kP * nChild + c].NumLocals;
  }
  if (prefix) resizeRows({&U[c_k]}, nL2P.c);
  else U[c_k] = ops.mul(ops.mul(nL2P, OP_C, tree[j][k].L2P, OP_N), OP_N, U[c_k], OP_N);
  PL = ops.vcat(U);
  tree[j - 1][kP].l2pOrtho = false;
}

void Solver::updateParentP2M(int j, int b, const DMat& nP2Mt, bool prefix) {  // T:3316-3340
  opprof::Scope prof_("upd_parent_p2m", ctx->stream);
  const int bP = b / nChild, c_b = b % nChild;
  DMat& PM = tree[j - 1][bP].P2M;
  std::vector<DMat> V(nChild);
  int ci = 0;
  for (int c = 0; c < nChild; ++c) {
    V[c] = ops.block(PM, 0, ci, PM.r, tree[j][bP * nChild + c].NumMultipoles);
    ci += tree[j][bP * nChild + c].NumMultipoles;
  }
  if (prefix) resizeCols({&V[c_b]}, nP2Mt.c);
  else V[c_b] = ops.mul(ops.mul(V[c_b], OP_N, tree[j][b].P2M, OP_N), OP_N, nP2Mt, OP_N);
  PM = ops.hcatv(V);
  tree[j - 1][bP].p2mOrtho = false;
}

// The new M2L block of compressP2P_myRRQR (T:1573-1656) once its two RRQRs
// gave the new bases: Rnp^H from the projected fill-in Rkp = nL2P^H P2Pt,
// plus the old M2L block carried into the new bases.
void Solver::compressP2PM2L(int j, int k, int b, const DMat& oldL2P, const DMat& oldP2M, const DMat& nL2P,
                            const DMat& nP2Mt, const DMat& Rkp, DMat& newM2L, bool prefixL, bool prefixM) {
  const DMat Rnp = ops.mul(nP2Mt, OP_C, Rkp, OP_C);
  newM2L = ops.adj(Rnp);
  DMat& M = tree[j][k].M2L[b];
  if (M.size() == 0) return;
  // newM2L += Rk M Rn^H with Rk = nL2P^H oldL2P, Rn = nP2Mt^H oldP2M^H; a
  // prefix basis makes its factor the partial identity [I; 0]
  if (prefixL && prefixM) {  // M lands in the top-left block
    const int r = std::min(M.r, newM2L.r), c = std::min(M.c, newM2L.c);
    zcopy_grouped(ctx, {{M.p, newM2L.p, r, c, M.ld(), newM2L.ld(), 0, ONE, 1}});
    return;
  }
  DMat RkM;
  if (prefixL) {
    RkM = M;
    resizeRows({&RkM}, nL2P.c);
  } else {
    RkM = ops.mul(ops.mul(nL2P, OP_C, oldL2P, OP_N), OP_N, M, OP_N);
  }
  if (prefixM) {  // (Rk M) [I 0]: add Rk M into the leading columns
    const int r = std::min(RkM.r, newM2L.r), c = std::min(RkM.c, newM2L.c);
    zcopy_grouped(ctx, {{RkM.p, newM2L.p, r, c, RkM.ld(), newM2L.ld(), 0, ONE, 1}});
    return;
  }
  GemmBatch g;
  const DMat Rn = ops.mul(nP2Mt, OP_C, oldP2M, OP_C);
  g.add(newM2L, RkM, OP_N, Rn, OP_C, ONE, ONE);
  g.flush(ctx);
}

static void equalise(Ops& ops, const DMat& L2P, const DMat& P2Mt, DMat& L2Pm, DMat& P2Mtm) {
  if (L2P.c < P2Mt.c) {
    P2Mtm = ops.block(P2Mt, 0, 0, P2Mt.r, L2P.c);
    L2Pm = L2P;
  } else {
    L2Pm = ops.block(L2P, 0, 0, L2P.r, P2Mt.c);
    P2Mtm = P2Mt;
  }
}

void Solver::compressP2PTwoWays(int j, int k, int b) {  // T:2116-2306
  if (tree[j][b].M2L[k].size() == 0 || tree[j][k].M2L[b].size() == 0) return;
  PhaseTimer pt(*this, stats.t_compress);
  stats.nCompressP2P++;
  DMat nL2P_k, nP2Mt_b, M2L_k_b, nL2P_b, nP2Mt_k, M2L_b_k;
  bool pkL, pbM, pbL, pkM;  // which new bases start with the old ones
  {
    opprof::Scope prof_fn_("compress_p2p", ctx->stream);
    // compressP2P_myRRQR(j, k, b) and (j, b, k) side by side: the two
    // directions read disjoint bases and blocks, so their row-basis RRQRs run
    // as one batch, then their column-basis RRQRs
    const DMat Lk = tree[j][k].L2P, Mb = tree[j][b].P2M, Pkb = tree[j][k].P2P[b];
    const DMat Lb = tree[j][b].L2P, Mk = tree[j][k].P2M, Pbk = tree[j][b].P2P[k];
    RRQRJob r1, r3;
    r1.A = ops.hcat(Lk, Pkb);
    r1.partition = Lk.c;
    r1.inputPivot = tree[j][k].maxPivot_L2P;
    r1.fillRank = fillin_rankVec[j];
    r1.orthoPanel = tree[j][k].l2pOrtho;
    r3.A = ops.hcat(Lb, Pbk);
    r3.partition = Lb.c;
    r3.inputPivot = tree[j][b].maxPivot_L2P;
    r3.fillRank = fillin_rankVec[j];
    r3.orthoPanel = tree[j][b].l2pOrtho;
    rrqrBatch({&r1, &r3});
    nL2P_k = r1.Q;
    pkL = r1.prefix;
    tree[j][k].maxPivot_L2P = std::max(tree[j][k].maxPivot_L2P, r1.maxPivot);
    nL2P_b = r3.Q;
    pbL = r3.prefix;
    tree[j][b].maxPivot_L2P = std::max(tree[j][b].maxPivot_L2P, r3.maxPivot);
    const DMat Rkp = ops.mul(nL2P_k, OP_C, Pkb, OP_N), Rbp = ops.mul(nL2P_b, OP_C, Pbk, OP_N);
    RRQRJob r2, r4;
    r2.A = ops.hcat(ops.adj(Mb), ops.adj(Rkp));
    r2.partition = Mb.r;
    r2.inputPivot = tree[j][b].maxPivot_P2M;
    r2.fillRank = fillin_rankVec[j];
    r2.orthoPanel = tree[j][b].p2mOrtho;
    r4.A = ops.hcat(ops.adj(Mk), ops.adj(Rbp));
    r4.partition = Mk.r;
    r4.inputPivot = tree[j][k].maxPivot_P2M;
    r4.fillRank = fillin_rankVec[j];
    r4.orthoPanel = tree[j][k].p2mOrtho;
    rrqrBatch({&r2, &r4});
    nP2Mt_b = r2.Q;
    pbM = r2.prefix;
    tree[j][b].maxPivot_P2M = std::max(tree[j][b].maxPivot_P2M, r2.maxPivot);
    nP2Mt_k = r4.Q;
    pkM = r4.prefix;
    tree[j][k].maxPivot_P2M = std::max(tree[j][k].maxPivot_P2M, r4.maxPivot);
    compressP2PM2L(j, k, b, Lk, Mb, nL2P_k, nP2Mt_b, Rkp, M2L_k_b, pkL, pbM);
    compressP2PM2L(j, b, k, Lb, Mk, nL2P_b, nP2Mt_k, Rbp, M2L_b_k, pbL, pkM);
  }
  DMat kL, kM, bL, bM;
  equalise(ops, nL2P_k, nP2Mt_k, kL, kM);
  equalise(ops, nL2P_b, nP2Mt_b, bL, bM);
  tree[j][k].M2L[b] = ops.block(M2L_k_b, 0, 0, kL.c, bM.c);
  updateOtherM2LsAtK(j, k, b, kL, pkL);
  updateOtherM2LsAtB(j, k, b, bM, pbM);
  if (j > startLevel) {
    updateParentL2P(j, k, kL, pkL);
    updateParentP2M(j, b, bM, pbM);
  }
  tree[j][k].L2P = kL;
  tree[j][b].P2M = ops.adj(bM);
  tree[j][k].l2pOrtho = tree[j][b].p2mOrtho = true;
  tree[j][k].NumLocals = tree[j][k].L2P.c;
  tree[j][b].NumMultipoles = tree[j][b].P2M.r;
  tree[j][b].M2L[k] = ops.block(M2L_b_k, 0, 0, bL.c, kM.c);
  updateOtherM2LsAtK(j, b, k, bL, pbL);
  updateOtherM2LsAtB(j, b, k, kM, pkM);
  if (j > startLevel) {
    updateParentL2P(j, b, bL, pbL);
    updateParentP2M(j, k, kM, pkM);
  }
  tree[j][b].L2P = bL;
  tree[j][k].P2M = ops.adj(kM);
  tree[j][b].l2pOrtho = tree[j][k].p2mOrtho = true;
  tree[j][b].NumLocals = tree[j][b].L2P.c;
  tree[j][k].NumMultipoles = tree[j][k].P2M.r;
}

void Solver::compressM2PP2L(int j, int k, int b) {  // T:2454-2596, :2878-2959
  if (tree[j][b].M2L[k].size() == 0 || tree[j][k].M2L[b].size() == 0) return;
  PhaseTimer pt(*this, stats.t_compress);
  stats.nCompressP2L++;
  DBox& Bk = tree[j][k];
  DBox& Bb = tree[j][b];
  // the RRQRs of compress_M2P_myRRQR(j, k, b) (A = [L2P_k | M2P[b]]) and of
  // compress_P2L_myRRQR(j, b, k) (A_row = [P2M_k^H | P2L[b][k]^H]) read
  // disjoint blocks: one batch
  RRQRJob rl, rm;
  rl.A = ops.hcat(Bk.L2P, Bk.M2P[b]);
  rl.partition = Bk.L2P.c;
  rl.inputPivot = Bk.maxPivot_L2P;
  rl.fillRank = fillin_rankVec[j];
  rl.orthoPanel = Bk.l2pOrtho;
  rm.A = ops.hcat(ops.adj(Bk.P2M), ops.adj(Bb.P2L[k]));
  rm.partition = Bk.P2M.r;
  rm.inputPivot = Bk.maxPivot_P2M;
  rm.fillRank = fillin_rankVec[j];
  rm.orthoPanel = Bk.p2mOrtho;
  rrqrBatch({&rl, &rm});
  const bool pL = rl.prefix, pM = rm.prefix;  // the new bases start with the old ones
  DMat nL2P_k = rl.Q;
  Bk.maxPivot_L2P = std::max(Bk.maxPivot_L2P, rl.maxPivot);
  DMat nP2Mt_k = rm.Q;
  Bk.maxPivot_P2M = std::max(Bk.maxPivot_P2M, rm.maxPivot);
  // compress_M2P_myRRQR(j, k, b)
  DMat M2L_k_b = ops.mul(nL2P_k, OP_C, Bk.M2P[b], OP_N);  // Rk'
  {
  opprof::Scope prof_fn_("compress_p2l", ctx->stream);
    const DMat& M = Bk.M2L[b];
    if (pL) {  // Rk = [I; 0]: M2L[b] adds into the leading rows
      if (M.size() > 0)
        zcopy_grouped(ctx, {{M.p, M2L_k_b.p, std::min(M.r, M2L_k_b.r), std::min(M.c, M2L_k_b.c), M.ld(),
                             M2L_k_b.ld(), 0, ONE, 1}});
    } else {
      const DMat Rk = ops.mul(nL2P_k, OP_C, Bk.L2P, OP_N);
      GemmBatch g;
      g.add(M2L_k_b, Rk, OP_N, M, OP_N, ONE, ONE);
      g.flush(ctx);
    }
  }
  // compress_P2L_myRRQR(j, b, k)
  DMat M2L_b_k;
  {
    const DMat Rnp = ops.mul(nP2Mt_k, OP_C, Bb.P2L[k], OP_C);
    M2L_b_k = ops.adj(Rnp);
    const DMat& M = Bb.M2L[k];
    if (pM) {  // Rn^H = [I 0]: M2L[k] adds into the leading columns
      if (M.size() > 0)
        zcopy_grouped(ctx, {{M.p, M2L_b_k.p, std::min(M.r, M2L_b_k.r), std::min(M.c, M2L_b_k.c), M.ld(),
                             M2L_b_k.ld(), 0, ONE, 1}});
    } else {
      const DMat Rn = ops.mul(nP2Mt_k, OP_C, Bk.P2M, OP_C);
      GemmBatch g;
      g.add(M2L_b_k, M, OP_N, Rn, OP_C, ONE, ONE);
      g.flush(ctx);
    }
  }
  DMat kL, kM;
  equalise(ops, nL2P_k, nP2Mt_k, kL, kM);
  Bk.M2L[b] = ops.block(M2L_k_b, 0, 0, kL.c, M2L_k_b.c);
  updateOtherM2LsAtK(j, k, b, kL, pL);
  if (j > startLevel) updateParentL2P(j, k, kL, pL);
  Bk.L2P = kL;
  Bk.l2pOrtho = true;
  Bk.NumLocals = Bk.L2P.c;
  Bb.M2L[k] = ops.block(M2L_b_k, 0, 0, M2L_b_k.r, kM.c);
  updateOtherM2LsAtB(j, b, k, kM, pM);
  if (j > startLevel) updateParentP2M(j, k, kM, pM);
  Bk.P2M = ops.adj(kM);
  Bk.p2mOrtho = true;
  Bk.NumMultipoles = Bk.P2M.r;
}

// ------------------------------------------------------------ elimination
// eliminate_x, T:3561-3611 with :3656-3791 (empty box) and :3800-4042.
void Solver::eliminateX(int j, int k) {
  opprof::Scope prof_fn_("elim_x", ctx->stream);
  PhaseTimer pt(*this, stats.t_elim_x);
  DBox& B = tree[j][k];
  auto E = [&](int x) { return tree[j][x].Eliminated; };
  std::vector<int> nbs;
  for (int nn : B.NB)
    if (nn != k) nbs.push_back(nn);
  if (B.P2P[k].size() != 0) {
    {
      PhaseTimer t(*this, stats.t_lu);
      B.luP2P = ops.factor(B.P2P[k]);
    }
    B.hasLuP2P = true;
    const int m = B.P2P[k].r;
    stats.flops_factor += 8.0 / 3.0 * m * (double)m * m;
    // one multi-RHS solve for [L2P | X_k,pp for every neighbour pp]
    std::vector<DMat> parts{B.L2P};
    std::vector<int> coff{0};
    int tot = B.L2P.c;
    for (int pp : nbs) {
      const DMat& X = E(pp) ? B.M2P[pp] : B.P2P[pp];
      AIFMM_REQUIRE(X.r == m, AIFMM_EINVAL, "eliminate_x: neighbour block rows");
      parts.push_back(X);
      coff.push_back(tot);
      tot += X.c;
    }
    // W = P2P[k]^{-1} [L2P | X...]: the inverse from the LU (m columns), then
    // one GEMM over all the neighbour columns instead of a triangular solve
    // with thousands of right-hand sides; the inverse also serves the sweeps.
    DMat W;
    {
      PhaseTimer t(*this, stats.t_msolve);
      B.invP2P = ops.solve(B.luP2P, ops.ident(m, ONE));
      const DMat X = ops.hcatv(parts);  // alive until the product is enqueued
      W = ops.alloc(m, tot);
      GemmBatch gw;
      gw.add(W, B.invP2P, OP_N, X, OP_N, ONE, ZERO);
      GemmPrecisionScope gp(ctx, prm.precision);  // the mixed path's tensor-core products
      gw.flush(ctx);
    }
    stats.flops_factor += 4.0 * m * (double)m * m + 8.0 * m * (double)m * tot;
    B.luP2P = DLU();
    auto Wb = [&](int idx, int cols) {  // column slice view of W
      DMat v;
      v.buf = W.buf;
      v.p = W.p + (size_t)coff[idx] * W.ld();
      v.r = W.r;
      v.c = cols;
      return v;
    };
    const DMat WL = Wb(0, B.L2P.c);
    GemmBatch g;
    auto addg = [&](DMat& C, const DMat& A, const DMat& Bm, zd alpha, zd beta) {
      g.add(C, A, OP_N, Bm, OP_N, alpha, beta);
      stats.flops_factor += 8.0 * C.r * (double)C.c * A.c;
    };
    B.L2M_f = ops.alloc(B.P2M.r, B.L2P.c);
    if (B.P2M.c == 0) B.L2M_f = ops.zeros(B.P2M.r, B.L2P.c);
    else addg(B.L2M_f, B.P2M, WL, MONE, ZERO);
    for (size_t q = 0; q < nbs.size(); ++q) {
      const int nn = nbs[q];
      const DMat Wn = Wb((int)q + 1, parts[q + 1].c);
      DMat& T = E(nn) ? B.M2M_f[nn] : B.P2M_f[nn];
      T = ops.alloc(B.P2M.r, Wn.c);
      if (B.P2M.c == 0) T = ops.zeros(B.P2M.r, Wn.c);
      else addg(T, B.P2M, Wn, MONE, ZERO);
    }
    for (size_t qn = 0; qn < nbs.size(); ++qn) {
      const int nn = nbs[qn];
      DBox& Bn = tree[j][nn];
      const DMat& Y = E(nn) ? Bn.P2L[k] : Bn.P2P[k];
      DMat& Lf = Bn.L2P_f[k];
      Lf = ops.alloc(Y.r, B.L2P.c);
      if (Y.c == 0) Lf = ops.zeros(Y.r, B.L2P.c);
      else addg(Lf, Y, WL, MONE, ZERO);
      for (size_t qp = 0; qp < nbs.size(); ++qp) {
        const int pp = nbs[qp];
        const DMat Wp = Wb((int)qp + 1, parts[qp + 1].c);
        DMat* Z;
        bool create;
        if (!E(nn)) {
          Z = E(pp) ? &Bn.M2P[pp] : &Bn.P2P[pp];
          create = Z->size() == 0;
        } else {
          Z = E(pp) ? &Bn.M2L[pp] : &Bn.P2L[pp];
          create = Z->size() == 0;
        }
        if (create) {
          *Z = ops.alloc(Y.r, Wp.c);
          if (Y.c == 0) *Z = ops.zeros(Y.r, Wp.c);
          else addg(*Z, Y, Wp, MONE, ZERO);
        } else if (Y.c > 0) {
          addg(*Z, Y, Wp, MONE, ONE);
        }
      }
    }
    {
      PhaseTimer t(*this, stats.t_schur);
      GemmPrecisionScope gp(ctx, prm.precision);  // the mixed path's tensor-core products
      g.flush(ctx);
    }
  } else {
    B.L2M_f = ops.zeros(B.P2M.r, B.L2P.c);
    for (int nn : nbs) {
      if (!E(nn)) B.P2M_f[nn] = ops.zeros(B.P2M.r, B.P2P[nn].c);
      else B.M2M_f[nn] = ops.zeros(B.P2M.r, B.M2P[nn].c);
    }
    for (int nn : nbs) {
      DBox& Bn = tree[j][nn];
      if (!E(nn)) Bn.L2P_f[k] = ops.zeros(Bn.P2P[k].r, B.L2P.c);
      else Bn.L2P_f[k] = ops.zeros(Bn.P2L[k].r, B.L2P.c);
      for (int pp : nbs) {
        if (!E(nn)) {
          if (!E(pp)) {
            if (Bn.P2P[pp].size() == 0) Bn.P2P[pp] = ops.zeros(Bn.P2P[k].r, B.P2P[pp].c);
          } else {
            if (Bn.M2P[pp].size() == 0) Bn.M2P[pp] = ops.zeros(Bn.P2P[k].r, B.M2P[pp].c);
          }
        } else {
          if (!E(pp)) {
            if (Bn.P2L[pp].size() == 0) Bn.P2L[pp] = ops.zeros(Bn.P2L[k].r, B.P2P[pp].c);
          } else {
            Bn.M2L[pp];
          }
        }
      }
    }
  }
}

// eliminate_z, T:4081-4113 with :4151-4296 (empty) and :4304-4509.
void Solver::eliminateZ(int j, int k) {
  opprof::Scope prof_fn_("elim_z", ctx->stream);
  PhaseTimer pt(*this, stats.t_elim_z);
  DBox& B = tree[j][k];
  auto E = [&](int x) { return tree[j][x].Eliminated; };
  std::vector<int> nbs;
  for (int nn : B.NB)
    if (nn != k) nbs.push_back(nn);
  if (B.L2M_f.size() > 0) {
    AIFMM_REQUIRE(B.L2M_f.r == B.L2M_f.c, AIFMM_EINVAL, "L2M_f is not square");
    {
      PhaseTimer t(*this, stats.t_lu);
      B.luL2M = ops.factor(B.L2M_f);
    }
    B.hasLuL2M = true;
    const int r = B.L2M_f.r;
    stats.flops_factor += 8.0 / 3.0 * r * (double)r * r;
    // [ -I | P2M_f[nn] or M2M_f[nn] ] in one solve
    std::vector<DMat> parts{ops.ident(B.NumMultipoles, MONE)};
    std::vector<int> coff{0};
    int tot = B.NumMultipoles;
    for (int nn : nbs) {
      const DMat& X = E(nn) ? B.M2M_f[nn] : B.P2M_f[nn];
      parts.push_back(X);
      coff.push_back(tot);
      tot += X.c;
    }
    DMat W;
    {
      PhaseTimer t(*this, stats.t_msolve);
      W = ops.solve(B.luL2M, ops.hcatv(parts));
    }
    stats.flops_factor += 4.0 * r * (double)r * tot;
    auto Wb = [&](int idx, int cols) {
      DMat v;
      v.buf = W.buf;
      v.p = W.p + (size_t)coff[idx] * W.ld();
      v.r = W.r;
      v.c = cols;
      return v;
    };
    const DMat Xy = Wb(0, B.NumMultipoles);  // -L2M_f^{-1}
    B.M2L[k] = ops.copy(Xy);
    B.negInvL2M = ops.copy(Xy);  // kept for the sweeps (M2L[k] is updated in place later)
    B.luL2M = DLU();
    std::vector<DMat> T(nbs.size());
    for (size_t q = 0; q < nbs.size(); ++q) {
      const int nn = nbs[q];
      T[q] = ops.copy(Wb((int)q + 1, parts[q + 1].c));
      if (!E(nn)) B.P2L[nn] = T[q];
      else B.M2L[nn] = T[q];
      // the P2L_M2P push of T:4340-4347 needs is_well_separated(j,k,nn), which
      // is false for every neighbour nn of k, so it never fires.
    }
    GemmBatch g;
    auto addg = [&](DMat& C, const DMat& A, const DMat& Bm, zd alpha, zd beta) {
      g.add(C, A, OP_N, Bm, OP_N, alpha, beta);
      stats.flops_factor += 8.0 * C.r * (double)C.c * A.c;
    };
    struct Check {
      int nn, pp;
      bool p2p;
    };
    // a preconditioner that drops every fill-in needs no queue decisions (and
    // no norm read-back)
    const bool dropAll = std::isinf(fillInTolerance);
    std::vector<Check> checks;
    for (size_t qn = 0; qn < nbs.size(); ++qn) {
      const int nn = nbs[qn];
      DBox& Bn = tree[j][nn];
      const DMat& Y = Bn.L2P_f[k];
      DMat& Z = E(nn) ? Bn.M2L[k] : Bn.M2P[k];
      if (Z.size() == 0) {
        Z = ops.alloc(Y.r, Xy.c);
        if (Y.c == 0) Z = ops.zeros(Y.r, Xy.c);
        else addg(Z, Y, Xy, MONE, ZERO);
      } else if (Y.c > 0) {
        addg(Z, Y, Xy, MONE, ONE);
      }
      for (size_t qp = 0; qp < nbs.size(); ++qp) {
        const int pp = nbs[qp];
        DMat* D;
        if (!E(nn)) D = E(pp) ? &Bn.M2P[pp] : &Bn.P2P[pp];
        else D = E(pp) ? &Bn.M2L[pp] : &Bn.P2L[pp];
        AIFMM_REQUIRE(D->r == Y.r && D->c == T[qp].c, AIFMM_EINVAL, "eliminate_z: fill-in block shape");
        if (Y.c > 0) addg(*D, Y, T[qp], MONE, ONE);
        if (!E(pp) && !dropAll && wellSeparated(j, nn, pp)) {
          if (!E(nn) && nn < pp) checks.push_back({nn, pp, true});
          if (E(nn)) checks.push_back({nn, pp, false});
        }
      }
    }
    {
      PhaseTimer t(*this, stats.t_schur);
      GemmPrecisionScope gp(ctx, prm.precision);  // the mixed path's tensor-core products
      g.flush(ctx);
    }
    if (!checks.empty()) {  // queue decisions need the norms of the updated blocks (T:4409-4418, :4448-4455)
      std::vector<const DMat*> ms;
      for (auto& c : checks) {
        DBox& Bn = tree[j][c.nn];
        ms.push_back(c.p2p ? &Bn.P2P[c.pp] : &Bn.P2L[c.pp]);
        ms.push_back(&Bn.M2L[c.pp]);
      }
      std::vector<double> nv = ops.norms(ms);
      for (size_t q = 0; q < checks.size(); ++q) {
        const double nf = nv[2 * q], nm = nv[2 * q + 1];
        if (nm > 0 && nf / nm > fillInTolerance) {
          if (checks[q].p2p) P2Pq.push_back({checks[q].nn, checks[q].pp});
          else P2L_M2P.push_back({checks[q].nn, checks[q].pp});
        }
      }
    }
  } else {
    B.M2L[k] = ops.zeros(0, B.NumMultipoles);
    for (int nn : nbs) {
      if (!E(nn)) B.P2L[nn] = ops.zeros(0, B.P2M_f[nn].c);
      else B.M2L[nn] = ops.zeros(0, B.M2M_f[nn].c);
    }
    for (int nn : nbs) {
      DBox& Bn = tree[j][nn];
      if (!E(nn)) {
        if (Bn.M2P[k].size() == 0) Bn.M2P[k] = ops.zeros(Bn.L2P_f[k].r, B.NumMultipoles);
      } else {
        if (Bn.M2L[k].size() == 0) Bn.M2L[k] = ops.zeros(Bn.L2P_f[k].r, B.NumMultipoles);
      }
      for (int pp : nbs) {
        if (!E(nn)) {
          if (!E(pp)) Bn.P2P[pp];
          else Bn.M2P[pp];
        } else {
          if (!E(pp)) Bn.P2L[pp];
          else Bn.M2L[pp];
        }
      }
    }
  }
}

void Solver::factorize() {  // eliminate_phase_efficient, T:4599-4747
  const double t0 = wall();
  AIFMM_CUDA(cudaSetDevice(ctx->device));
  const long tc0 = prm.precision >= 2 ? tc_timeouts() : 0;
  dropPlan();  // its graph reads the blocks this factorization replaces
  stats.nRRQR = stats.nRRQRShort = stats.nCompressP2P = stats.nCompressP2L = 0;
  // A fresh tree's fill-in queues are empty.  The reference does not clear
  // them between levels, and pairs queued late at one level can still be
  // waiting when its elimination ends; a refactorization after rewind() must
  // not inherit them from the previous factorization.
  P2Pq.clear();
  P2L_M2P.clear();
  stats.flops_factor = 0;
  baseLU_ = DLU();
  baseReady_ = false;
  stats.t_rrqr = stats.t_compress = stats.t_elim_x = stats.t_elim_z = stats.t_nonleaf = 0;
  stats.t_lu = stats.t_msolve = stats.t_schur = 0;
  for (int j = nLevels; j >= startLevel; --j) {
    if (j != nLevels) {
      initP2PNonLeaf(j);
      deleteM2L(j);
    }
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
      for (int i = 0; i < (int)P2Pq.size(); i++) {
        const int nn = P2Pq[i].first, pp = P2Pq[i].second;
        if (k == nn || k == pp) {
          P2Pq.erase(P2Pq.begin() + i);
          i--;
          if (tree[j][nn].P2P[pp].size() != 0) {
            compressP2PTwoWays(j, nn, pp);
            tree[j][nn].P2P[pp] = DMat();
            tree[j][pp].P2P[nn] = DMat();
          }
        }
      }
      for (int i = 0; i < (int)P2L_M2P.size(); i++) {
        const int nn = P2L_M2P[i].first, pp = P2L_M2P[i].second;
        if (k == nn || k == pp) {
          P2L_M2P.erase(P2L_M2P.begin() + i);
          i--;
          if (tree[j][nn].P2L[pp].size() != 0) {
            compressM2PP2L(j, pp, nn);
            tree[j][nn].P2L[pp] = DMat();
            tree[j][pp].M2P[nn] = DMat();
          }
        }
      }
      tree[j][k].Eliminated = true;
      eliminateX(j, k);
      eliminateZ(j, k);
    }
  }
  factorBase(startLevel);
  ops.sync();
  // a tensor-core tile that gave up on a bounded wait left its Schur block unwritten
  if (prm.precision >= 2) tc_check(tc0, "factorize");
  factored = true;
  stats.t_factor = wall() - t0;
}

// ------------------------------------------------------------ solve sweeps
// Tree order of the unknowns: leaves in box order, each leaf's
// chargeLocations in order; built once, used by the gathers of the sweeps.
void Solver::treeOrder() {
  if (leafPermReady_) return;
  std::vector<int> perm;
  leafOff_.assign(nBoxesPerLevel[nLevels] + 1, 0);
  for (int k = 0; k < nBoxesPerLevel[nLevels]; ++k) {
    leafOff_[k] = (int)perm.size();
    const auto& cl = tree[nLevels][k].chargeLocations;
    perm.insert(perm.end(), cl.begin(), cl.end());
  }
  leafOff_.back() = (int)perm.size();
  AIFMM_REQUIRE((int)perm.size() == N, AIFMM_EINVAL, "leaves do not cover every unknown");
  leafPerm_ = std::make_shared<DevBuf>(upload(ctx, perm));
  leafPermReady_ = true;
}

void Solver::assignLeafRhs(const DMat& rhs) {  // T:670-678 (a gather of rows)
  const int j = nLevels;
  treeOrder();
  // rows of rhs in tree order, then one block copy per leaf
  DMat Xt = ops.alloc(N, nrhs_);
  zrows_gather(ctx, rhs.p, rhs.ld(), leafPerm_->as<int>(), N, Xt.p, Xt.ld(), nrhs_);
  std::vector<CopyProblem> cps;
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    DBox& B = tree[j][k];
    const int n = leafOff_[k + 1] - leafOff_[k];
    B.particle_rhs = ops.alloc(n, nrhs_);
    if (n > 0) cps.push_back({Xt.p + leafOff_[k], B.particle_rhs.p, n, nrhs_, Xt.ld(), B.particle_rhs.ld(), 0, ONE});
  }
  zcopy_grouped(ctx, cps);
}

void Solver::rhsEliminateX(int j, int k) {  // T:3613-3653, :3795-3886
  DBox& B = tree[j][k];
  if (B.P2P[k].size() != 0) {
    const DMat y = ops.mul(B.invP2P, OP_N, B.particle_rhs, OP_N);
    // local_rhs = -P2M y rides in the same launch as the neighbour updates
    B.local_rhs = ops.alloc(B.P2M.r, nrhs_);
    GemmBatch g;
    g.add(B.local_rhs, B.P2M, OP_N, y, OP_N, MONE, ZERO);
    for (int nn : B.NB) {
      if (nn == k) continue;
      DBox& Bn = tree[j][nn];
      if (!Bn.Eliminated) g.add(Bn.particle_rhs, Bn.P2P[k], OP_N, y, OP_N, MONE, ONE);
      else g.add(Bn.multipole_rhs, Bn.P2L[k], OP_N, y, OP_N, MONE, ONE);
    }
    g.flush(ctx);
  } else {
    B.local_rhs = ops.zeros(B.P2M.r, nrhs_);
  }
}

void Solver::rhsEliminateZ(int j, int k) {  // T:4115-4148, :4313-4397
  DBox& B = tree[j][k];
  if (B.L2M_f.size() > 0) {
    B.multipole_rhs = ops.mul(B.negInvL2M, OP_N, B.local_rhs, OP_N, MONE);
    GemmBatch g;
    for (int nn : B.NB) {
      if (nn == k) continue;
      DBox& Bn = tree[j][nn];
      DMat& t = Bn.Eliminated ? Bn.multipole_rhs : Bn.particle_rhs;
      g.add(t, Bn.L2P_f[k], OP_N, B.multipole_rhs, OP_N, MONE, ONE);
    }
    g.flush(ctx);
  } else {
    B.multipole_rhs = ops.alloc(0, nrhs_);
  }
}

// The base-level system of solve_particles_at_base_level (T:4772-4810): the
// M2L blocks of the start level, fixed once the factorization is done.  The
// reference assembles and factorizes it in every solve; here it is factorized
// once, at the end of factorize(), and each solve only applies the factors.
void Solver::factorBase(int j) {
  opprof::Scope prof_fn_("base_lu", ctx->stream);
  int NM = 0, NL = 0;
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    NM += tree[j][k].NumMultipoles;
    NL += tree[j][k].NumLocals;
  }
  baseLU_ = DLU();
  baseReady_ = true;
  if (NL == 0 || NM == 0) return;
  AIFMM_REQUIRE(NL == NM, AIFMM_EINVAL, "base-level system is not square");
  DMat A = ops.zeros(NL, NM);
  std::vector<CopyProblem> cps;
  int ri = 0;
  for (int r = 0; r < nBoxesPerLevel[j]; ++r) {
    int si = 0;
    for (int s = 0; s < nBoxesPerLevel[j]; ++s) {
      const DMat& m = tree[j][r].M2L[s];
      AIFMM_REQUIRE(m.r == tree[j][r].NumLocals && m.c == tree[j][s].NumMultipoles, AIFMM_EINVAL,
                    "base-level M2L block shape");
      if (m.size()) cps.push_back({m.p, A.p + (size_t)si * A.ld() + ri, m.r, m.c, m.ld(), A.ld(), 0, ONE});
      si += tree[j][s].NumMultipoles;
    }
    ri += tree[j][r].NumLocals;
  }
  zcopy_grouped(ctx, cps);
  baseLU_ = ops.factor(A);
  stats.flops_factor += 8.0 / 3.0 * NL * (double)NL * NL;
}

void Solver::baseSolve(int j) {  // solve_particles_at_base_level, T:4772-4810
  int NM = 0, NL = 0;
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    NM += tree[j][k].NumMultipoles;
    NL += tree[j][k].NumLocals;
  }
  if (NL == 0 || NM == 0) return;
  AIFMM_REQUIRE(NL == NM, AIFMM_EINVAL, "base-level system is not square");
  if (!baseReady_) factorBase(j);
  AIFMM_REQUIRE(baseLU_.n == NL, AIFMM_EINVAL, "base-level factors do not match the system");
  DMat b = ops.zeros(NL, nrhs_);
  std::vector<CopyProblem> cps;
  int ri = 0;
  for (int r = 0; r < nBoxesPerLevel[j]; ++r) {
    const DMat& mr = tree[j][r].multipole_rhs;
    if (mr.size()) cps.push_back({mr.p, b.p + ri, mr.r, mr.c, mr.ld(), b.ld(), 0, ONE});
    ri += tree[j][r].NumLocals;
  }
  zcopy_grouped(ctx, cps);
  DMat mp = ops.solve(baseLU_, b);
  int idx = 0;
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    tree[j][k].multipoles = ops.block(mp, idx, 0, tree[j][k].NumMultipoles, nrhs_);
    idx += tree[j][k].NumMultipoles;
  }
}

void Solver::backSubstitute() {  // back_substitution_phase, T:4812-4865
  baseSolve(startLevel);
  for (int j = startLevel; j <= nLevels; j++)
    for (int k = nBoxesPerLevel[j] - 1; k >= 0; k--) {
      DBox& B = tree[j][k];
      if (B.P2P[k].size() != 0) {
        DMat rhs1 = ops.copy(B.particle_rhs);
        GemmBatch g;
        for (int nn : B.NB) {
          if (nn == k) continue;
          if (!tree[j][nn].Eliminated) g.add(rhs1, B.P2P[nn], OP_N, tree[j][nn].particles, OP_N, MONE, ONE);
          else g.add(rhs1, B.M2P[nn], OP_N, tree[j][nn].multipoles, OP_N, MONE, ONE);
        }
        g.flush(ctx);
        // rhs2 = multipoles - P2M P2P_kk^{-1} rhs1 ; Atemp = -P2M P2P_kk^{-1} L2P = L2M_f
        DMat rhs2 = ops.copy(B.multipoles);
        const DMat y = ops.mul(B.invP2P, OP_N, rhs1, OP_N);
        GemmBatch g2;
        if (B.P2M.c > 0) g2.add(rhs2, B.P2M, OP_N, y, OP_N, MONE, ONE);
        g2.flush(ctx);
        if (B.L2M_f.size() != 0) B.locals = ops.mul(B.negInvL2M, OP_N, rhs2, OP_N, MONE);
        else B.locals = ops.alloc(0, nrhs_);
        DMat t = rhs1;
        GemmBatch g3;
        if (B.L2P.c > 0) g3.add(t, B.L2P, OP_N, B.locals, OP_N, MONE, ONE);
        g3.flush(ctx);
        B.particles = ops.mul(B.invP2P, OP_N, t, OP_N);
      } else {
        B.particles = ops.alloc(0, nrhs_);
      }
      B.Eliminated = false;
      if (nLevels != j) {
        int idx = 0;
        for (int c = 0; c < nChild; ++c) {
          DBox& C = tree[j + 1][nChild * k + c];
          C.multipoles = ops.block(B.particles, idx, 0, C.NumMultipoles, nrhs_);
          idx += C.NumMultipoles;
        }
      }
    }
}

SolvePlan::~SolvePlan() {
  if (ctx) cudaStreamSynchronize(ctx->stream);  // no replay in flight
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  if (hold) hold->releaseAll();
}

// Captures solveSweeps(in) -> out on the context stream.  During the capture
// the context allocates and uploads outside it (aifmm_ctx::capture), so the
// graph holds only kernels, memsets and device-to-device copies; the kernel
// launches counted while capturing are not launches and are taken back.
void Solver::capturePlan(int nrhs) {
  opprof::Scope prof_fn_("solve_capture", ctx->stream);
  plan_.reset();
  treeOrder();
  std::unique_ptr<SolvePlan> pl(new SolvePlan);
  pl->ctx = ctx;
  pl->nrhs = nrhs;
  pl->in = ops.alloc(N, nrhs);
  pl->out = ops.alloc(N, nrhs);
  pl->hold = std::make_shared<CaptureHold>();
  pl->hold->ctx = ctx;
  if (!ctx->sideStream) AIFMM_CUDA(cudaStreamCreateWithFlags(&ctx->sideStream, cudaStreamNonBlocking));
  AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
  const long l0 = thread_launch_count();
  AIFMM_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
  ctx->capture = pl->hold;
  try {
    const DMat x = solveSweeps(pl->in);
    AIFMM_CUDA(cudaMemcpyAsync(pl->out.p, x.p, sizeof(zd) * x.size(), cudaMemcpyDeviceToDevice, ctx->stream));
  } catch (...) {
    ctx->capture.reset();
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(ctx->stream, &g);
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    count_launch(l0 - thread_launch_count());
    throw;
  }
  ctx->capture.reset();
  const cudaError_t e = cudaStreamEndCapture(ctx->stream, &pl->graph);
  pl->launches = thread_launch_count() - l0;
  count_launch(-pl->launches);
  AIFMM_CUDA(e);
  AIFMM_CUDA(cudaGraphInstantiate(&pl->exec, pl->graph, 0));
  stats.nSolveCapture++;
  plan_ = std::move(pl);
}

DMat Solver::solve(const DMat& rhs) {
  AIFMM_REQUIRE(factored, AIFMM_ESTATE, "solve before factorize");
  AIFMM_REQUIRE(rhs.r == N && rhs.c >= 1, AIFMM_EINVAL, "rhs must be N x nrhs");
  const double t0 = wall();
  // the per-launch profilers time each launch with host synchronisation: eager sweeps
  if (graphSolve && !opprof::enabled() && !gemm_profile_on()) {
    if (!plan_ || plan_->nrhs != rhs.c) capturePlan(rhs.c);
    AIFMM_CUDA(cudaMemcpyAsync(plan_->in.p, rhs.p, sizeof(zd) * rhs.size(), cudaMemcpyDeviceToDevice, ctx->stream));
    AIFMM_CUDA(cudaGraphLaunch(plan_->exec, ctx->stream));
    count_launch(plan_->launches);
    DMat x = ops.copy(plan_->out);
    ops.sync();
    stats.nSolveGraph++;
    stats.t_solve = wall() - t0;
    return x;
  }
  DMat x = solveSweeps(rhs);
  ops.sync();
  stats.t_solve = wall() - t0;
  return x;
}

DMat Solver::solveSweeps(const DMat& rhs) {
  nrhs_ = rhs.c;
  assignLeafRhs(rhs);
  // rhs_eliminate_phase_efficient, T:4749-4770
  for (int j = nLevels; j >= startLevel; --j)
    for (DBox& B : tree[j]) B.Eliminated = false;
  for (int j = startLevel; j <= nLevels; ++j)  // multipole_rhs starts at zero (initialise_rhs, T:3343-3352)
    for (DBox& B : tree[j]) B.multipole_rhs = ops.zeros(B.NumLocals, nrhs_);
  for (int j = nLevels; j >= startLevel; --j) {
    if (j != nLevels)
      for (int k = 0; k < nBoxesPerLevel[j]; ++k) {  // T:3506-3523
        std::vector<DMat> parts;
        for (int c = 0; c < nChild; ++c) parts.push_back(tree[j + 1][nChild * k + c].multipole_rhs);
        tree[j][k].particle_rhs = ops.vcat(parts);
      }
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
      tree[j][k].Eliminated = true;
      rhsEliminateX(j, k);
      rhsEliminateZ(j, k);
    }
  }
  backSubstitute();
  // getx + reorder (T:4874-4907, :466-476): x[chargeLocations[i]] = particles_i
  DMat Yt = ops.zeros(N, nrhs_);
  std::vector<CopyProblem> cps;
  for (int k = 0; k < nBoxesPerLevel[nLevels]; ++k) {
    DBox& B = tree[nLevels][k];
    const int n = std::min(leafOff_[k + 1] - leafOff_[k], B.particles.r);
    if (n > 0) cps.push_back({B.particles.p, Yt.p + leafOff_[k], n, nrhs_, B.particles.ld(), Yt.ld(), 0, ONE});
  }
  zcopy_grouped(ctx, cps);
  DMat x = ops.alloc(N, nrhs_);
  zrows_scatter(ctx, Yt.p, Yt.ld(), leafPerm_->as<int>(), N, x.p, x.ld(), nrhs_);
  return x;
}

// ------------------------------------------------------------ checkpoint
std::vector<std::vector<DBox>> Solver::deepCopy(std::vector<std::vector<DBox>>& src) {
  std::vector<std::vector<DBox>> dst = src;  // host metadata; device handles still shared
  std::vector<CopyProblem> cps;
  auto dup = [&](DMat& m) {
    if (m.size() == 0) return;
    DMat n = ops.alloc(m.r, m.c);
    cps.push_back({m.p, n.p, m.r, m.c, m.ld(), n.ld(), 0, ONE});
    m = n;
  };
  for (auto& lvl : dst)
    for (DBox& B : lvl) {
      for (auto* mp : {&B.M2L, &B.P2P, &B.M2P, &B.P2L, &B.L2P_f, &B.P2M_f, &B.M2M_f})
        for (auto& kv : *mp) dup(kv.second);
      dup(B.L2M_f);
      dup(B.L2P);
      dup(B.P2M);
      B.luP2P = DLU();
      B.luL2M = DLU();
      B.invP2P = B.negInvL2M = DMat();
      B.hasLuP2P = B.hasLuL2M = false;
      B.particles = B.multipoles = B.locals = B.particle_rhs = B.multipole_rhs = B.local_rhs = DMat();
    }
  zcopy_grouped(ctx, cps);
  return dst;
}

void Solver::checkpoint() {
  AIFMM_REQUIRE(!factored, AIFMM_ESTATE, "checkpoint must be taken before factorize");
  saved_ = deepCopy(tree);
  hasSaved_ = true;
  ops.sync();
}

void Solver::rewind() {
  AIFMM_REQUIRE(hasSaved_, AIFMM_ESTATE, "no checkpoint to rewind to");
  dropPlan();
  tree.clear();  // the factorized blocks go before the copy is made: one tree's memory less at the peak
  tree = deepCopy(saved_);
  P2Pq.clear();
  P2L_M2P.clear();
  baseLU_ = DLU();
  baseReady_ = false;
  factored = false;
}

// ------------------------------------------------------------ diagnostics
int Solver::avgLeafSize() const {
  int avg = 0, n = 0;
  for (const DBox& B : tree[nLevels])
    if (!B.chargeLocations.empty()) {
      n++;
      avg += (int)B.chargeLocations.size();
    }
  return n ? avg / n : 0;
}
int Solver::avgMultipoles() const {
  int avg = 0, n = 0;
  for (int j = nLevels; j >= startLevel; j--)
    for (const DBox& B : tree[j])
      if (B.P2M.r > 0 && !B.IL.empty()) {
        n++;
        avg += B.P2M.r;
      }
  return n ? avg / n : 0;
}
int Solver::maxRank() const {
  int mx = 0;
  for (int j = nLevels; j >= startLevel; j--)
    for (const DBox& B : tree[j]) mx = std::max(mx, B.P2M.r);
  return mx;
}
double Solver::memoryGB(bool after) {  // findMemory / findMemoryAfterFactorize, T:4511-4571
  double sum = 0.0;
  for (int j = nLevels; j >= startLevel; --j)
    for (DBox& B : tree[j]) sum += B.L2P.size() + B.P2M.size();
  if (!after)
    for (int j = nLevels; j >= startLevel; --j)
      for (DBox& B : tree[j])
        for (int n : B.IL) sum += B.M2L[n].size();
  const int jlo = after ? startLevel : nLevels;
  for (int j = nLevels; j >= jlo; --j)
    for (DBox& B : tree[j])
      for (int n : B.NB) sum += B.P2P[n].size();
  return sum * 8 * 1e-9;
}

}  // namespace aifmm
