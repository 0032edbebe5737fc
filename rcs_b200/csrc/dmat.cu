#include "dmat.cuh"

#include <chrono>
#include <cstdio>
#include <map>
#include <mutex>

namespace aifmm {

namespace opprof {
static int g_mode = 0;
static bool g_on = false;
static std::mutex g_mu;
static std::map<std::string, std::pair<long, double>> g_table;
double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
void enable(int mode) {
  std::lock_guard<std::mutex> l(g_mu);
  g_mode = mode;
  g_on = mode != 0;
  g_table.clear();
}
bool enabled() { return g_on; }
int mode() { return g_mode; }
cudaError_t sync(cudaStream_t s) {
  if (!g_on) return cudaStreamSynchronize(s);
  const double t0 = now();
  const cudaError_t e = cudaStreamSynchronize(s);
  add("sync_wait", now() - t0);
  return e;
}
void add(const char* name, double seconds) {
  std::lock_guard<std::mutex> l(g_mu);
  auto& e = g_table[name];
  e.first++;
  e.second += seconds;
}
std::string report() {
  std::lock_guard<std::mutex> l(g_mu);
  std::string out;
  char line[160];
  for (auto& kv : g_table) {
    snprintf(line, sizeof(line), "%-24s %10ld %12.6f\n", kv.first.c_str(), kv.second.first, kv.second.second);
    out += line;
  }
  return out;
}
static thread_local std::vector<const char*> g_stack;
std::string path() {
  std::string out;
  for (const char* n : g_stack) {
    if (!out.empty()) out += '/';
    out += n;
  }
  return out;
}
Scope::Scope(const char* n, cudaStream_t s) : name(n), stream(s), t0(g_on ? now() : 0.0) { g_stack.push_back(n); }
Scope::~Scope() {
  g_stack.pop_back();
  if (!g_on) return;
  if (g_mode == 1) cudaStreamSynchronize(stream);
  add(name, now() - t0);
}
}  // namespace opprof

void GemmBatch::add(DMat& C, const DMat& A, int opA, const DMat& B, int opB, zd alpha, zd beta) {
  const int m = opA == OP_N ? A.r : A.c;
  const int k = opA == OP_N ? A.c : A.r;
  const int kb = opB == OP_N ? B.r : B.c;
  const int n = opB == OP_N ? B.c : B.r;
  AIFMM_REQUIRE(k == kb && C.r == m && C.c == n, AIFMM_EINVAL,
                "GEMM shape mismatch " + std::to_string(m) + "x" + std::to_string(k) + " * " + std::to_string(kb) +
                    "x" + std::to_string(n) + " -> " + std::to_string(C.r) + "x" + std::to_string(C.c));
  if (m == 0 || n == 0) return;
  probs.push_back({A.p, B.p, C.p, m, n, k, A.ld(), B.ld(), C.ld(), opA, opB, alpha, beta});
}

// Problems that write the same output must not run in one launch (their
// read-modify-write of C would race): problem q goes to wave w = number of
// earlier problems with the same C, and waves run in order, which also keeps
// the accumulation order of each output equal to the insertion order.
// Problems with the same C become one chain when they share shape and alpha
// and every later one has beta 1 (the accumulations the solver issues);
// otherwise the repeats go to later launches, one wave per repeat.
void GemmBatch::flush(aifmm_ctx* ctx) {
  opprof::Scope prof_("gemm_flush", ctx->stream);
  if (probs.empty()) return;
  std::map<const zd*, std::vector<int>> byC;
  std::vector<const zd*> order;
  for (int i = 0; i < (int)probs.size(); ++i) {
    auto& v = byC[probs[i].C];
    if (v.empty()) order.push_back(probs[i].C);
    v.push_back(i);
  }
  std::vector<GemmProblem> ps;
  std::vector<int> chain;
  std::vector<std::vector<GemmProblem>> waves;
  for (const zd* c : order) {
    const std::vector<int>& ids = byC[c];
    const GemmProblem& h = probs[ids[0]];
    bool ok = true;
    for (size_t q = 1; q < ids.size() && ok; ++q) {
      const GemmProblem& p = probs[ids[q]];
      ok = p.m == h.m && p.n == h.n && p.ldc == h.ldc && p.alpha.x == h.alpha.x && p.alpha.y == h.alpha.y &&
           p.beta.x == 1.0 && p.beta.y == 0.0;
    }
    if (ok) {
      chain.push_back((int)ids.size());
      for (size_t q = 1; q < ids.size(); ++q) chain.push_back(0);
      for (int i : ids) ps.push_back(probs[i]);
    } else {
      ps.push_back(h);
      chain.push_back(1);
      for (size_t q = 1; q < ids.size(); ++q) {
        if (waves.size() < q) waves.resize(q);
        waves[q - 1].push_back(probs[ids[q]]);
      }
    }
  }
  zgemm_chained(ctx, ps, chain);
  for (auto& w : waves) zgemm_grouped(ctx, w);
  probs.clear();
}

DMat Ops::alloc(int r, int c) const {
  opprof::Scope prof_("alloc", ctx->stream);
  AIFMM_REQUIRE(r >= 0 && c >= 0, AIFMM_EINVAL, "negative matrix size");
  DMat m;
  m.r = r;
  m.c = c;
  if ((long)r * c > 0) {
    m.buf = std::make_shared<DevBuf>(ctx, sizeof(zd) * (size_t)r * c);
    m.p = m.buf->as<zd>();
  }
  return m;
}
std::vector<DMat> Ops::allocMany(const std::vector<std::pair<int, int>>& shapes) const {
  opprof::Scope prof_("alloc_many", ctx->stream);
  constexpr size_t kAlign = 512 / sizeof(zd), kSlab = ((size_t)16 << 20) / sizeof(zd);
  std::vector<DMat> out(shapes.size());
  size_t i = 0;
  while (i < shapes.size()) {
    // the matrices [i, j) share one slab
    size_t j = i, words = 0;
    for (; j < shapes.size(); ++j) {
      AIFMM_REQUIRE(shapes[j].first >= 0 && shapes[j].second >= 0, AIFMM_EINVAL, "negative matrix size");
      const size_t w = ((size_t)shapes[j].first * shapes[j].second + kAlign - 1) / kAlign * kAlign;
      if (j > i && words + w > kSlab) break;
      words += w;
    }
    std::shared_ptr<DevBuf> slab;
    if (words > 0) slab = std::make_shared<DevBuf>(ctx, sizeof(zd) * words);
    size_t off = 0;
    for (size_t q = i; q < j; ++q) {
      DMat& m = out[q];
      m.r = shapes[q].first;
      m.c = shapes[q].second;
      if (m.size() > 0) {
        m.buf = slab;
        m.p = slab->as<zd>() + off;
        off += ((size_t)m.size() + kAlign - 1) / kAlign * kAlign;
      }
    }
    i = j;
  }
  return out;
}
DMat Ops::zeros(int r, int c) const {
  opprof::Scope prof_("zeros", ctx->stream);
  DMat m = alloc(r, c);
  if (m.size()) AIFMM_CUDA(cudaMemsetAsync(m.p, 0, sizeof(zd) * m.size(), ctx->stream));
  return m;
}
DMat Ops::ident(int n, zd d) const {
  DMat m = alloc(n, n);
  if (m.size()) zset_identity(ctx, m.p, n, n, d);
  return m;
}
DMat Ops::copy(const DMat& a) const {
  opprof::Scope prof_("copy", ctx->stream);
  DMat m = alloc(a.r, a.c);
  if (m.size()) AIFMM_CUDA(cudaMemcpyAsync(m.p, a.p, sizeof(zd) * m.size(), cudaMemcpyDeviceToDevice, ctx->stream));
  return m;
}
DMat Ops::block(const DMat& a, int i0, int j0, int nr, int nc) const {
  opprof::Scope prof_("block", ctx->stream);
  AIFMM_REQUIRE(i0 >= 0 && j0 >= 0 && nr >= 0 && nc >= 0 && i0 + nr <= a.r && j0 + nc <= a.c, AIFMM_EINVAL,
                "block out of range");
  DMat m = alloc(nr, nc);
  if (m.size()) zcopy_grouped(ctx, {{a.p + (size_t)j0 * a.ld() + i0, m.p, nr, nc, a.ld(), m.ld(), 0, zmk(1, 0)}});
  return m;
}
DMat Ops::adj(const DMat& a) const {
  opprof::Scope prof_("adj", ctx->stream);
  DMat m = alloc(a.c, a.r);
  if (m.size()) zcopy_grouped(ctx, {{a.p, m.p, a.c, a.r, a.ld(), m.ld(), 1, zmk(1, 0)}});
  return m;
}
DMat Ops::neg(const DMat& a) const {
  DMat m = alloc(a.r, a.c);
  if (m.size()) zcopy_grouped(ctx, {{a.p, m.p, a.r, a.c, a.ld(), m.ld(), 0, zmk(-1, 0)}});
  return m;
}
void Ops::setBlock(DMat& dst, int i0, int j0, const DMat& src) const {
  AIFMM_REQUIRE(i0 >= 0 && j0 >= 0 && i0 + src.r <= dst.r && j0 + src.c <= dst.c, AIFMM_EINVAL,
                "setBlock out of range");
  if (src.size()) zcopy_grouped(ctx, {{src.p, dst.p + (size_t)j0 * dst.ld() + i0, src.r, src.c, src.ld(), dst.ld(), 0, zmk(1, 0)}});
}
DMat Ops::hcat(const DMat& a, const DMat& b) const { return hcatv({a, b}); }
DMat Ops::hcatv(const std::vector<DMat>& parts) const {
  opprof::Scope prof_("hcat", ctx->stream);
  int r = parts.empty() ? 0 : parts[0].r, c = 0;
  for (const DMat& q : parts) {
    AIFMM_REQUIRE(q.r == r, AIFMM_EINVAL, "hcat rows mismatch");
    c += q.c;
  }
  DMat m = alloc(r, c);
  std::vector<CopyProblem> cp;
  int o = 0;
  for (const DMat& q : parts) {
    if (q.size()) cp.push_back({q.p, m.p + (size_t)o * m.ld(), q.r, q.c, q.ld(), m.ld(), 0, zmk(1, 0)});
    o += q.c;
  }
  zcopy_grouped(ctx, cp);
  return m;
}
DMat Ops::vcat(const std::vector<DMat>& parts) const {
  opprof::Scope prof_("vcat", ctx->stream);
  int r = 0, c = parts.empty() ? 0 : parts[0].c;
  for (const DMat& q : parts) {
    AIFMM_REQUIRE(q.c == c, AIFMM_EINVAL, "vcat cols mismatch");
    r += q.r;
  }
  DMat m = alloc(r, c);
  std::vector<CopyProblem> cp;
  int o = 0;
  for (const DMat& q : parts) {
    if (q.size()) cp.push_back({q.p, m.p + o, q.r, q.c, q.ld(), m.ld(), 0, zmk(1, 0)});
    o += q.r;
  }
  zcopy_grouped(ctx, cp);
  return m;
}
DMat Ops::mul(const DMat& a, int opA, const DMat& b, int opB, zd alpha) const {
  const int m = opA == OP_N ? a.r : a.c;
  const int n = opB == OP_N ? b.c : b.r;
  DMat c = alloc(m, n);
  const int k = opA == OP_N ? a.c : a.r;
  if (k == 0) {
    if (c.size()) AIFMM_CUDA(cudaMemsetAsync(c.p, 0, sizeof(zd) * c.size(), ctx->stream));
    return c;
  }
  GemmBatch g;
  g.add(c, a, opA, b, opB, alpha, zmk(0, 0));
  g.flush(ctx);
  return c;
}
std::vector<double> Ops::norms(const std::vector<const DMat*>& ms) const {
  opprof::Scope prof_("norms", ctx->stream);
  std::vector<double> out(ms.size(), 0.0);
  std::vector<NormProblem> ps;
  std::vector<int> idx;
  for (size_t i = 0; i < ms.size(); ++i)
    if (ms[i]->size() > 0) {
      ps.push_back({ms[i]->p, ms[i]->r, ms[i]->c, ms[i]->ld()});
      idx.push_back((int)i);
    }
  if (ps.empty()) return out;
  DevBuf d(ctx, sizeof(double) * ps.size());
  znorm_grouped(ctx, ps, d.as<double>());
  std::vector<double> h(ps.size());
  AIFMM_CUDA(cudaMemcpyAsync(h.data(), d.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, ctx->stream));
  AIFMM_CUDA(opprof::sync(ctx->stream));
  for (size_t q = 0; q < idx.size(); ++q) out[idx[q]] = h[q];
  return out;
}
double Ops::maxColNorm(const DMat& a) const {
  AIFMM_REQUIRE(a.c > 0, AIFMM_EINVAL, "maxColNorm of empty matrix");
  std::vector<NormProblem> ps;
  for (int j = 0; j < a.c; ++j) ps.push_back({a.p + (size_t)j * a.ld(), a.r, 1, a.ld()});
  DevBuf d(ctx, sizeof(double) * ps.size());
  znorm_grouped(ctx, ps, d.as<double>());
  std::vector<double> h(ps.size());
  AIFMM_CUDA(cudaMemcpyAsync(h.data(), d.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, ctx->stream));
  AIFMM_CUDA(opprof::sync(ctx->stream));
  double best = -1.0;
  for (double v : h) best = std::max(best, v);
  return best;
}
DLU Ops::factor(const DMat& a) const {
  opprof::Scope prof_("lu_factor", ctx->stream);
  AIFMM_REQUIRE(a.r == a.c, AIFMM_EINVAL, "LU of a non-square matrix");
  DLU f;
  f.n = a.r;
  f.lu = copy(a);
  f.piv = std::make_shared<DevBuf>(ctx, sizeof(int) * std::max(1, a.r));
  f.info = std::make_shared<DevBuf>(ctx, sizeof(int));
  if (a.r > 0) zgetrf(ctx, f.lu.p, a.r, a.ld(), f.piv->as<int>(), f.info->as<int>());
  return f;
}
DMat Ops::solve(const DLU& f, const DMat& b) const {
  opprof::Scope prof_("lu_solve", ctx->stream);
  AIFMM_REQUIRE(b.r == f.n, AIFMM_EINVAL, "LU solve size mismatch");
  DMat x = copy(b);
  if (x.size()) zgetrs(ctx, f.lu.p, f.n, f.lu.ld(), f.piv->as<int>(), x.p, x.c, x.ld());
  return x;
}
void Ops::sync() const { AIFMM_CUDA(opprof::sync(ctx->stream)); }
std::vector<zd> Ops::download(const DMat& a) const {
  std::vector<zd> h((size_t)a.size());
  if (a.size())
    AIFMM_CUDA(cudaMemcpyAsync(h.data(), a.p, sizeof(zd) * h.size(), cudaMemcpyDeviceToHost, ctx->stream));
  sync();
  return h;
}
DMat Ops::fromHost(const std::vector<zd>& v, int r, int c) const {
  DMat m = alloc(r, c);
  if (m.size()) AIFMM_CUDA(cudaMemcpyAsync(m.p, v.data(), sizeof(zd) * m.size(), cudaMemcpyHostToDevice, ctx->stream));
  return m;
}

}  // namespace aifmm
