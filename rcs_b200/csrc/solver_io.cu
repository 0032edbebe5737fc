// Factorization checkpoint file: the factored solver written to disk and read
// back into a new solver, so that later processes solve without rebuilding or
// refactorizing.  The reference keeps its factors only in memory
// (FMM2DTree's per-box std::map blocks, include/AIFMMTree2D_3D_memory_optimized.hpp
// AIFMMBox.hpp:13-71); the file holds the same state: the tree geometry, every
// box's index lists and blocks, and the factors of the base-level system.
//
// Layout (little-endian): 8-byte magic "AIFMMFC1"; the solver parameters and
// tree scalars; per level and box the box's scalars, index lists and blocks
// (each block: int32 rows, int32 cols, then rows x cols complex128 in column
// order); the base-level LU (block, pivots).  Blocks are staged through one
// pinned host buffer of 64 MB (several blocks per device-to-host round trip).
#include <cstdio>
#include <cstring>
#include <memory>

#include "capi_guard.cuh"
#include "solver.cuh"

namespace aifmm {

namespace {

const char kMagic[8] = {'A', 'I', 'F', 'M', 'M', 'F', 'C', '1'};
const size_t kStage = (size_t)64 << 20;

struct PinnedStage {
  void* p = nullptr;
  PinnedStage() { AIFMM_CUDA(cudaMallocHost(&p, kStage)); }
  ~PinnedStage() {
    if (p) cudaFreeHost(p);
  }
};

class Writer {
 public:
  Writer(const std::string& path, aifmm_ctx* ctx) : ctx_(ctx) {
    f_ = std::fopen(path.c_str(), "wb");
    AIFMM_REQUIRE(f_ != nullptr, AIFMM_EINVAL, "cannot open the checkpoint file for writing");
  }
  ~Writer() {
    if (f_) std::fclose(f_);
  }
  void raw(const void* p, size_t n) {
    flushBlocks();
    put(p, n);
  }
  template <typename T>
  void val(const T& v) {
    raw(&v, sizeof(T));
  }
  template <typename T>
  void vec(const std::vector<T>& v) {
    const long long n = (long long)v.size();
    val(n);
    if (n) raw(v.data(), sizeof(T) * v.size());
  }
  // a block: shape now, entries staged (written in enqueue order)
  void mat(const DMat& m) {
    const int32_t rc[2] = {m.r, m.c};
    const size_t bytes = sizeof(zd) * (size_t)m.size();
    if (pendBytes_ + 8 + bytes > kStage) flushBlocks();
    if (8 + bytes > kStage) {  // larger than the stage: on its own, in stage-sized pieces
      put(rc, 8);
      for (size_t off = 0; off < bytes; off += kStage) {
        const size_t n = std::min(kStage, bytes - off);
        AIFMM_CUDA(cudaMemcpyAsync(stage_.p, (const char*)m.p + off, n, cudaMemcpyDeviceToHost, ctx_->stream));
        AIFMM_CUDA(cudaStreamSynchronize(ctx_->stream));
        put(stage_.p, n);
      }
      return;
    }
    char* dst = (char*)stage_.p + pendBytes_;
    std::memcpy(dst, rc, 8);
    if (bytes)
      AIFMM_CUDA(cudaMemcpyAsync(dst + 8, m.p, bytes, cudaMemcpyDeviceToHost, ctx_->stream));
    pendBytes_ += 8 + bytes;
  }
  void finish() {
    flushBlocks();
    AIFMM_REQUIRE(std::fflush(f_) == 0, AIFMM_EINVAL, "checkpoint write failed");
  }

 private:
  void put(const void* p, size_t n) {
    AIFMM_REQUIRE(std::fwrite(p, 1, n, f_) == n, AIFMM_EINVAL, "checkpoint write failed");
  }
  void flushBlocks() {
    if (!pendBytes_) return;
    AIFMM_CUDA(cudaStreamSynchronize(ctx_->stream));
    put(stage_.p, pendBytes_);
    pendBytes_ = 0;
  }
  aifmm_ctx* ctx_;
  std::FILE* f_ = nullptr;
  PinnedStage stage_;
  size_t pendBytes_ = 0;
};

class Reader {
 public:
  Reader(const std::string& path, aifmm_ctx* ctx, Ops& ops) : ctx_(ctx), ops_(ops) {
    f_ = std::fopen(path.c_str(), "rb");
    AIFMM_REQUIRE(f_ != nullptr, AIFMM_EINVAL, "cannot open the checkpoint file");
  }
  ~Reader() {
    if (f_) std::fclose(f_);
  }
  void raw(void* p, size_t n) {
    AIFMM_REQUIRE(std::fread(p, 1, n, f_) == n, AIFMM_EINVAL, "checkpoint file is truncated");
  }
  template <typename T>
  T val() {
    T v;
    raw(&v, sizeof(T));
    return v;
  }
  template <typename T>
  std::vector<T> vec() {
    const long long n = val<long long>();
    AIFMM_REQUIRE(n >= 0 && n < (1LL << 40), AIFMM_EINVAL, "checkpoint file is corrupt");
    std::vector<T> v((size_t)n);
    if (n) raw(v.data(), sizeof(T) * v.size());
    return v;
  }
  DMat mat() {
    int32_t rc[2];
    raw(rc, 8);
    AIFMM_REQUIRE(rc[0] >= 0 && rc[1] >= 0, AIFMM_EINVAL, "checkpoint file is corrupt");
    DMat m = ops_.alloc(rc[0], rc[1]);
    const size_t bytes = sizeof(zd) * (size_t)m.size();
    for (size_t off = 0; off < bytes; off += kStage) {
      const size_t n = std::min(kStage, bytes - off);
      AIFMM_CUDA(cudaStreamSynchronize(ctx_->stream));  // the stage is free again
      raw(stage_.p, n);
      AIFMM_CUDA(cudaMemcpyAsync((char*)m.p + off, stage_.p, n, cudaMemcpyHostToDevice, ctx_->stream));
    }
    return m;
  }

 private:
  aifmm_ctx* ctx_;
  Ops& ops_;
  std::FILE* f_ = nullptr;
  PinnedStage stage_;
};

std::map<int, DMat> DBox::* const kMaps[] = {&DBox::M2L, &DBox::P2P, &DBox::M2P, &DBox::P2L,
                                                   &DBox::L2P_f, &DBox::P2M_f, &DBox::M2M_f};
DMat DBox::* const kMats[] = {&DBox::particles, &DBox::multipoles, &DBox::locals, &DBox::particle_rhs,
                              &DBox::multipole_rhs, &DBox::local_rhs, &DBox::L2M_f, &DBox::L2P, &DBox::P2M,
                              &DBox::Ac, &DBox::Ar, &DBox::invP2P, &DBox::negInvL2M};
std::vector<int> DBox::* const kLists[] = {&DBox::IL, &DBox::NB, &DBox::chargeLocations, &DBox::in_charge,
                                           &DBox::in_check, &DBox::out_charge, &DBox::out_check};

}  // namespace

void Solver::save(const std::string& path) {
  AIFMM_REQUIRE(factored, AIFMM_EINVAL, "save needs a factorized solver");
  AIFMM_CUDA(cudaSetDevice(ctx->device));
  Writer w(path, ctx);
  w.raw(kMagic, 8);
  const int32_t ip[] = {prm.leafSize, prm.tol_pow, prm.nLevelsInput, prm.fillin_rank, prm.fillin_tol, prm.realMode,
                        (int32_t)prm.orthoShortcut, prm.precision, prm.drop_pow, N, nLevels, startLevel, nChild,
                        (int32_t)baseReady_};
  w.raw(ip, sizeof(ip));
  w.val(L);
  w.val(eta);
  w.val(fillInTolerance);
  w.raw(domain, sizeof(domain));
  w.vec(nBoxesPerLevel);
  w.vec(boxSideLength);
  w.vec(particles);
  for (int j = 0; j <= nLevels; ++j) {
    w.val((long long)tree[j].size());
    for (const DBox& B : tree[j]) {
      const double dv[] = {B.maxPivot_L2P, B.maxPivot_P2M, B.center[0], B.center[1], B.center[2]};
      const int32_t iv[] = {(int32_t)B.ILActive, (int32_t)B.Eliminated, B.NumMultipoles, B.NumLocals,
                            (int32_t)B.l2pOrtho, (int32_t)B.p2mOrtho};
      w.raw(dv, sizeof(dv));
      w.raw(iv, sizeof(iv));
      for (auto l : kLists) w.vec(B.*l);
      for (auto m : kMats) w.mat(B.*m);
      for (auto mp : kMaps) {
        const std::map<int, DMat>& M = B.*mp;
        w.val((long long)M.size());
        for (const auto& kv : M) {
          w.val((int32_t)kv.first);
          w.mat(kv.second);
        }
      }
    }
  }
  if (baseReady_) {
    w.val((int32_t)baseLU_.n);
    w.mat(baseLU_.lu);
    std::vector<int> piv((size_t)baseLU_.n);
    if (baseLU_.n) {
      w.finish();
      AIFMM_CUDA(cudaMemcpyAsync(piv.data(), baseLU_.piv->p, sizeof(int) * piv.size(), cudaMemcpyDeviceToHost,
                                 ctx->stream));
      AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    w.vec(piv);
  }
  w.finish();
}

void Solver::load(const std::string& path) {
  AIFMM_CUDA(cudaSetDevice(ctx->device));
  dropPlan();
  Reader r(path, ctx, ops);
  char magic[8];
  r.raw(magic, 8);
  AIFMM_REQUIRE(std::memcmp(magic, kMagic, 8) == 0, AIFMM_EINVAL, "not an AIFMM factorization checkpoint");
  int32_t ip[14];
  r.raw(ip, sizeof(ip));
  AIFMM_REQUIRE(ip[9] == N, AIFMM_EINVAL, "the checkpoint was written for a kernel of another size");
  prm.leafSize = ip[0];
  prm.tol_pow = ip[1];
  prm.nLevelsInput = ip[2];
  prm.fillin_rank = ip[3];
  prm.fillin_tol = ip[4];
  prm.realMode = ip[5];
  prm.orthoShortcut = ip[6] != 0;
  prm.precision = ip[7];
  prm.drop_pow = ip[8];
  nLevels = ip[10];
  startLevel = ip[11];
  nChild = ip[12];
  const bool base = ip[13] != 0;
  AIFMM_REQUIRE(nLevels >= 2 && nLevels < 9 && startLevel >= 0 && startLevel <= nLevels, AIFMM_EINVAL,
                "checkpoint file is corrupt");
  for (int j = 0; j < 64; ++j) fillin_rankVec[j] = 0;  // the constructor's rule for the file's depth
  for (int j = nLevels, temp = 5, i = 0; j >= 2; --j) {
    fillin_rankVec[j] = temp;
    if (++i % 3 == 0) temp += 5;
  }
  L = r.val<double>();
  eta = r.val<double>();
  fillInTolerance = r.val<double>();
  r.raw(domain, sizeof(domain));
  nBoxesPerLevel = r.vec<int>();
  boxSideLength = r.vec<double>();
  particles = r.vec<double>();
  tree.assign(nLevels + 1, {});
  for (int j = 0; j <= nLevels; ++j) {
    const long long nb = r.val<long long>();
    AIFMM_REQUIRE(nb >= 0 && nb < (1LL << 30), AIFMM_EINVAL, "checkpoint file is corrupt");
    tree[j].resize((size_t)nb);
    for (DBox& B : tree[j]) {
      double dv[5];
      int32_t iv[6];
      r.raw(dv, sizeof(dv));
      r.raw(iv, sizeof(iv));
      B.maxPivot_L2P = dv[0];
      B.maxPivot_P2M = dv[1];
      for (int q = 0; q < 3; ++q) B.center[q] = dv[2 + q];
      B.ILActive = iv[0] != 0;
      B.Eliminated = iv[1] != 0;
      B.NumMultipoles = iv[2];
      B.NumLocals = iv[3];
      B.l2pOrtho = iv[4] != 0;
      B.p2mOrtho = iv[5] != 0;
      for (auto l : kLists) B.*l = r.vec<int>();
      for (auto m : kMats) B.*m = r.mat();
      for (auto mp : kMaps) {
        std::map<int, DMat>& M = B.*mp;
        const long long n = r.val<long long>();
        AIFMM_REQUIRE(n >= 0 && n < (1LL << 30), AIFMM_EINVAL, "checkpoint file is corrupt");
        for (long long q = 0; q < n; ++q) {
          const int key = r.val<int32_t>();
          M[key] = r.mat();
        }
      }
    }
  }
  baseLU_ = DLU();
  baseReady_ = false;
  if (base) {
    baseLU_.n = r.val<int32_t>();
    baseLU_.lu = r.mat();
    std::vector<int> piv = r.vec<int>();
    AIFMM_REQUIRE((int)piv.size() == baseLU_.n, AIFMM_EINVAL, "checkpoint file is corrupt");
    baseLU_.piv = std::make_shared<DevBuf>(upload(ctx, piv));
    baseLU_.info = std::make_shared<DevBuf>(ctx, sizeof(int));
    AIFMM_CUDA(cudaMemsetAsync(baseLU_.info->p, 0, sizeof(int), ctx->stream));
    baseReady_ = true;
  }
  P2L_M2P.clear();
  P2Pq.clear();
  leafPermReady_ = false;
  hasSaved_ = false;
  saved_.clear();
  ops.sync();
  factored = true;
}

}  // namespace aifmm

extern "C" {

int aifmm_solver_save(aifmm_solver* s, const char* path) {
  API_BEGIN
  AIFMM_REQUIRE(s && path, AIFMM_EINVAL, "NULL argument");
  s->s->save(path);
  API_END
}

int aifmm_solver_load(aifmm_kernel* k, const char* path, aifmm_solver** out) {
  API_BEGIN
  AIFMM_REQUIRE(k && path && out, AIFMM_EINVAL, "NULL argument");
  aifmm::SolverParams sp;
  sp.realMode = k->geom.efie ? 0 : 1;
  std::unique_ptr<aifmm_solver> s(new aifmm_solver);
  s->s.reset(new aifmm::Solver(k, sp));
  s->s->load(path);
  aifmm::ctx_retain(k->ctx);
  *out = s.release();
  API_END
}

}  // extern "C"
