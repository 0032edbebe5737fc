// Autotuner of the tensor-core GEMM (GEMM precision 5).
//
// The solver's grouped GEMMs come in a few recurring shapes per tree level:
// the Schur-complement products of a leaf box (hundreds of products of about
// m x m x m), those of a non-leaf box, the rank-sized products of
// eliminate_z.  Which kernel and tile order is fastest depends on that
// shape: the 128 x 64 tiles of zgemm_tc5p waste less on narrow products, the
// persistent 128 x 128 kernel of zgemm_tc6 moves fewer bytes per flop on wide
// ones, and the order in which a persistent CTA walks a group's tiles decides
// which operand panel stays in L2.  Each launch is classified by total flops
// and number of output chains (log4 scale) and median n and k (log2 scale); the
// first launch of a class is timed on synthetic operands of exactly its
// shapes (a copy of the launch with scratch buffers, sampled down to 1 GB of
// operands) for each candidate -- tc5p; tc6 in its packed-real and
// split-planes operand forms, each with row-major and column-major tile
// order -- and the fastest is kept for the class on this context.  With the
// environment variable AIFMM_TUNE_FILE set, choices are read from and
// appended to that file, so that later runs make the same choices (the
// candidates round differently, so the choice fixes the bits of the result).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>

#include "dense.cuh"

namespace aifmm {

namespace {

struct Candidate {
  int precision, raster, form;
  const char* name;
};
const Candidate kCandidates[] = {{3, 0, 0, "tc5p 128x64"},
                                 {4, 0, 0, "tc6 packed-real row-major"},
                                 {4, 1, 0, "tc6 packed-real column-major"},
                                 {4, 0, 1, "tc6 split-planes row-major"},
                                 {4, 1, 1, "tc6 split-planes column-major"}};

int lg2(double x) { return x <= 1.0 ? 0 : (int)std::floor(std::log2(x)); }

long long classify(const std::vector<GemmProblem>& probs, const std::vector<int>& chain) {
  double flops = 0;
  int chains = 0;
  std::vector<int> ns, ks;
  for (size_t i = 0; i < probs.size();) {
    const int len = std::max(1, chain[i]);
    chains++;
    for (int q = 0; q < len && i + q < probs.size(); ++q) {
      const GemmProblem& p = probs[i + q];
      flops += 8.0 * p.m * (double)p.n * std::max(p.k, 0);
      ns.push_back(p.n);
      ks.push_back(p.k);
    }
    i += len;
  }
  if (ns.empty()) return 0;
  std::nth_element(ns.begin(), ns.begin() + ns.size() / 2, ns.end());
  std::nth_element(ks.begin(), ks.begin() + ks.size() / 2, ks.end());
  // flops and chain counts on a log4 scale, median n and k on a log2 scale:
  // few enough classes that the trials stay a small share of a factorization
  const long long a = lg2(flops) / 2, b = lg2(chains) / 2, c = lg2(ns[ns.size() / 2]), d = lg2(ks[ks.size() / 2]);
  return (a << 24) | (b << 16) | (c << 8) | d;
}

__global__ void tune_fill_kernel(zd* p, size_t n, unsigned seed) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned h = (unsigned)i * 2654435761u ^ seed;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    p[i] = zmk((double)(h & 0xFFFF) / 65536.0 - 0.5, (double)(h >> 16) / 65536.0 - 0.5);
  }
}

void load_file(aifmm_ctx* ctx) {
  const char* f = std::getenv("AIFMM_TUNE_FILE");
  if (!f) return;
  std::ifstream in(f);
  long long key;
  int choice;
  while (in >> key >> choice)
    if (choice >= 0 && choice < (int)(sizeof(kCandidates) / sizeof(kCandidates[0]))) ctx->tuneCache[key] = choice;
}

void append_file(long long key, int choice) {
  const char* f = std::getenv("AIFMM_TUNE_FILE");
  if (!f) return;
  std::ofstream out(f, std::ios::app);
  out << key << " " << choice << "\n";
}

// Times every candidate on scratch operands with the launch's shapes.
int tune(aifmm_ctx* ctx, const std::vector<GemmProblem>& probs, const std::vector<int>& chain, long long key) {
  // scratch copies of the distinct operands and outputs, chain by chain, up to the budget
  const size_t budget = (size_t)1 << 30;
  std::map<const void*, size_t> extent;  // real buffer -> the largest extent any sampled product reads (elements)
  size_t elems = 0;
  std::vector<GemmProblem> ps;
  std::vector<int> ch;
  for (size_t i = 0; i < probs.size();) {
    const int len = std::max(1, chain[i]);
    std::map<const void*, size_t> ext = extent;
    for (int q = 0; q < len; ++q) {
      const GemmProblem& p = probs[i + q];
      const std::pair<const void*, size_t> uses[3] = {{p.A, (size_t)p.lda * (p.opA == OP_N ? p.k : p.m)},
                                                      {p.B, (size_t)p.ldb * (p.opB == OP_N ? p.n : p.k)},
                                                      {(const void*)p.C, (size_t)p.ldc * p.n}};
      for (const auto& u : uses) ext[u.first] = std::max(ext[u.first], u.second);
    }
    size_t total = 0;
    for (const auto& kv : ext) total += kv.second;
    if (!ps.empty() && total * sizeof(zd) > budget) break;  // sample the launch up to the budget
    extent.swap(ext);
    elems = total;
    for (int q = 0; q < len; ++q) {
      ps.push_back(probs[i + q]);
      ch.push_back(q == 0 ? len : 0);
    }
    i += len;
  }
  std::map<const void*, size_t> where;  // real buffer -> scratch offset (elements)
  {
    size_t off = 0;
    for (const auto& kv : extent) {
      where[kv.first] = off;
      off += kv.second;
    }
  }
  DevBuf scratch(ctx, sizeof(zd) * std::max<size_t>(elems, 1));
  tune_fill_kernel<<<148 * 8, 256, 0, ctx->stream>>>(scratch.as<zd>(), elems, 12345u);
  AIFMM_LAUNCHED();
  zd* base = scratch.as<zd>();
  for (GemmProblem& p : ps) {
    p.A = base + where[p.A];
    p.B = base + where[p.B];
    p.C = base + where[p.C];
  }
  const int saved = ctx->gemmPrecision, savedRaster = ctx->gemmRaster, savedForm = ctx->gemmForm;
  cudaEvent_t e0, e1;
  AIFMM_CUDA(cudaEventCreate(&e0));
  AIFMM_CUDA(cudaEventCreate(&e1));
  int best = 0;
  float bestMs = 1e30f;
  std::ostringstream log;
  log << "class " << key << " (" << ps.size() << " of " << probs.size() << " products timed):";
  const int nc = (int)(sizeof(kCandidates) / sizeof(kCandidates[0]));
  struct Restore {  // the context's GEMM mode after the trials, whatever happens
    aifmm_ctx* c;
    int p, r, f;
    ~Restore() {
      c->gemmPrecision = p;
      c->gemmRaster = r;
      c->gemmForm = f;
    }
  } restore{ctx, saved, savedRaster, savedForm};
  for (int c = 0; c < nc; ++c) {
    ctx->gemmPrecision = kCandidates[c].precision;
    ctx->gemmRaster = kCandidates[c].raster;
    ctx->gemmForm = kCandidates[c].form;
    zgemm_chained(ctx, ps, ch);  // warm-up (plane buffers, first-touch)
    float ms = 1e30f;
    for (int rep = 0; rep < 2; ++rep) {
      AIFMM_CUDA(cudaEventRecord(e0, ctx->stream));
      zgemm_chained(ctx, ps, ch);
      AIFMM_CUDA(cudaEventRecord(e1, ctx->stream));
      AIFMM_CUDA(cudaEventSynchronize(e1));
      float t = 0;
      AIFMM_CUDA(cudaEventElapsedTime(&t, e0, e1));
      ms = std::min(ms, t);
    }
    log << " " << kCandidates[c].name << " " << ms << " ms;";
    if (ms < bestMs) {
      bestMs = ms;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  log << " -> " << kCandidates[best].name;
  std::lock_guard<std::mutex> l(ctx->tuneMu);
  ctx->tuneLog.push_back(log.str());
  return best;
}

}  // namespace

void zgemm_tuned(aifmm_ctx* ctx, const std::vector<GemmProblem>& probs, const std::vector<int>& chain) {
  const long long key = classify(probs, chain);
  int choice = -1;
  {
    std::lock_guard<std::mutex> l(ctx->tuneMu);
    if (ctx->tuneCache.empty()) load_file(ctx);
    auto it = ctx->tuneCache.find(key);
    if (it != ctx->tuneCache.end()) choice = it->second;
  }
  if (choice < 0) {
    choice = tune(ctx, probs, chain, key);
    std::lock_guard<std::mutex> l(ctx->tuneMu);
    ctx->tuneCache[key] = choice;
    append_file(key, choice);
  }
  const int saved = ctx->gemmPrecision, savedRaster = ctx->gemmRaster, savedForm = ctx->gemmForm;
  ctx->gemmPrecision = kCandidates[choice].precision;
  ctx->gemmRaster = kCandidates[choice].raster;
  ctx->gemmForm = kCandidates[choice].form;
  try {
    zgemm_chained(ctx, probs, chain);
  } catch (...) {
    ctx->gemmPrecision = saved;
    ctx->gemmRaster = savedRaster;
    ctx->gemmForm = savedForm;
    throw;
  }
  ctx->gemmPrecision = saved;
  ctx->gemmRaster = savedRaster;
  ctx->gemmForm = savedForm;
}

std::string tune_report(aifmm_ctx* ctx) {
  std::lock_guard<std::mutex> l(ctx->tuneMu);
  std::string out;
  for (const std::string& s : ctx->tuneLog) out += s + "\n";
  return out;
}

}  // namespace aifmm
