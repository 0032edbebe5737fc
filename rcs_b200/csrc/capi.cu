// C ABI of libaifmm_b200.so: argument checking, error translation and the
// context / kernel objects.  Numerical work happens in the kernels of
// assemble.cu and the solver files; nothing here computes on the host.
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <set>

#include "capi_guard.cuh"
#include "context.cuh"
#include "dense.cuh"
#include "dmat.cuh"

namespace aifmm {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }
static std::atomic<long> g_launches{0};
static thread_local long t_launches = 0;
void count_launch(long n) {
  g_launches += n;
  t_launches += n;
}
long launch_count() { return g_launches.load(); }
long thread_launch_count() { return t_launches; }

static std::mutex g_ctx_mu;

void smem_attr_once(const void* kernel, int device, int bytes) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  std::lock_guard<std::mutex> l(mu);
  if (done.count({kernel, device})) return;
  AIFMM_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done.insert({kernel, device});
}

void ctx_retain(aifmm_ctx* c) {
  std::lock_guard<std::mutex> l(g_ctx_mu);
  c->refs++;
}

void ctx_release(aifmm_ctx* c) {
  bool last;
  {
    std::lock_guard<std::mutex> l(g_ctx_mu);
    last = (--c->refs == 0);
  }
  if (!last) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int i = 0; i < aifmm_ctx::kRingChunks; ++i)
    if (c->ringEvent[i]) cudaEventDestroy(c->ringEvent[i]);
  if (c->ring) cudaFreeHost(c->ring);
  if (c->holdFlag) cudaFree(c->holdFlag);
  if (c->arena) {
    for (auto& ch : c->arena->chunks()) cudaFreeAsync((void*)ch.first, c->stream);
    c->arena.reset();
    if (c->stream) cudaStreamSynchronize(c->stream);
  }
  if (c->pool) cudaMemPoolDestroy(c->pool);
  if (c->sideStream) cudaStreamDestroy(c->sideStream);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

// Returns the arena's chunks that hold no block to the pool.
static void arena_trim(aifmm_ctx* c) {
  if (!c->arena) return;
  std::lock_guard<std::mutex> l(c->arenaMu);
  for (auto& ch : c->arena->takeFreeChunks()) cudaFreeAsync((void*)ch.first, c->stream);
}

void ctx_trim(aifmm_ctx* c) {
  AIFMM_REQUIRE(!c->capture, AIFMM_ESTATE, "trim during a graph capture");
  AIFMM_CUDA(cudaStreamSynchronize(c->stream));
  arena_trim(c);
  AIFMM_CUDA(cudaStreamSynchronize(c->stream));
  AIFMM_CUDA(cudaMemPoolTrimTo(c->pool, 0));
}

void DevBuf::alloc(aifmm_ctx* c, size_t n) {
  release();
  ctx = c;
  bytes = n;
  hold = c->capture;
  if (c->arena && n >= Arena::kMinSize) {
    std::lock_guard<std::mutex> l(c->arenaMu);
    const uint64_t a = c->arena->alloc(n);
    if (a != 0) {
      p = (void*)a;
      fromArena = true;
      c->bytes_live += n;
      return;
    }
  }
  const double t0 = opprof::enabled() ? opprof::now() : 0.0;
  // during a capture the allocation is made outside it, on the side stream
  cudaStream_t s = c->capture ? c->sideStream : c->stream;
  cudaError_t e = cudaMallocFromPoolAsync(&p, n, c->pool, s);
  if (e == cudaSuccess && c->capture) e = cudaStreamSynchronize(s);
  if (opprof::enabled()) {
    const double dt = opprof::now() - t0;
    opprof::add("pool_alloc", dt);
    opprof::add(n < ((size_t)1 << 20) ? "pool_alloc_lt1MB" : n < ((size_t)64 << 20) ? "pool_alloc_lt64MB" : "pool_alloc_ge64MB",
                dt);
  }
  if (e == cudaErrorMemoryAllocation && !c->capture) {  // (a capturing stream cannot be drained)
    // the pool and the arena keep freed blocks; return them to the device and retry once
    cudaGetLastError();
    arena_trim(c);
    cudaStreamSynchronize(c->stream);
    cudaMemPoolTrimTo(c->pool, 0);
    e = cudaMallocFromPoolAsync(&p, n, c->pool, c->stream);
  }
  if (e != cudaSuccess) {
    p = nullptr;
    cudaGetLastError();
    throw Error(AIFMM_ENOMEM, "device allocation of " + std::to_string(n) + " bytes failed: " + cudaGetErrorString(e));
  }
  c->bytes_live += n;
}
void upload_bytes(aifmm_ctx* c, void* dst, const void* src, size_t n) {
  if (n == 0) return;
  if (c->capture) {  // copied now, outside the capture: dst is a buffer the graph holds
    AIFMM_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, c->sideStream));
    AIFMM_CUDA(cudaStreamSynchronize(c->sideStream));
    return;
  }
  if (!c->ring || n > aifmm_ctx::kRingBytes / 4) {
    AIFMM_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, c->stream));
    return;
  }
  size_t head = (c->ringHead + 255) & ~(size_t)255;
  if (head + n > aifmm_ctx::kRingBytes) {
    head = 0;
    c->ringLap++;
  }
  const int c0 = (int)(head / aifmm_ctx::kRingChunk), c1 = (int)((head + n - 1) / aifmm_ctx::kRingChunk);
  for (int q = c0; q <= c1; ++q)  // a chunk from an earlier lap: its last copy must be done
    if (c->ringChunkLap[q] != 0 && c->ringChunkLap[q] != c->ringLap) {
      const double t0 = opprof::enabled() ? opprof::now() : 0.0;
      AIFMM_CUDA(cudaEventSynchronize(c->ringEvent[q]));
      if (opprof::enabled()) opprof::add("ring_wait", opprof::now() - t0);
    }
  std::memcpy(c->ring + head, src, n);
  AIFMM_CUDA(cudaMemcpyAsync(dst, c->ring + head, n, cudaMemcpyHostToDevice, c->stream));
  for (int q = c0; q <= c1; ++q) {
    AIFMM_CUDA(cudaEventRecord(c->ringEvent[q], c->stream));
    c->ringChunkLap[q] = c->ringLap;
  }
  c->ringHead = head + n;
}

void DevBuf::release() {
  if (p && ctx) {
    // A buffer allocated during a capture stays with that graph while the
    // graph lives.  Any other buffer released while a capture is in progress
    // may be read by a node captured before the release, so the capture in
    // progress keeps it (and a free on the capturing stream would be a graph
    // node of memory the graph does not own).
    std::shared_ptr<CaptureHold> own = std::move(hold);
    const std::shared_ptr<CaptureHold> cur = ctx->capture;
    const std::shared_ptr<CaptureHold>* holds[2] = {&own, &cur};
    for (const std::shared_ptr<CaptureHold>* h : holds) {
      if (!*h) continue;
      std::lock_guard<std::mutex> l((*h)->mu);
      if ((*h)->alive) {
        (*h)->held.push_back({p, bytes, fromArena});
        p = nullptr;
        bytes = 0;
        fromArena = false;
        return;
      }
    }
  }
  hold.reset();
  if (p && ctx && fromArena) {
    {
      std::lock_guard<std::mutex> l(ctx->arenaMu);
      ctx->arena->release((uint64_t)p);
    }
    ctx->bytes_live -= bytes;
    p = nullptr;
    bytes = 0;
    fromArena = false;
    return;
  }
  if (p && ctx) {
    const double t0 = opprof::enabled() ? opprof::now() : 0.0;
    cudaFreeAsync(p, ctx->stream);
    if (opprof::enabled()) opprof::add("pool_free", opprof::now() - t0);
    ctx->bytes_live -= bytes;
  }
  p = nullptr;
  bytes = 0;
}

void CaptureHold::releaseAll() {
  std::vector<Rec> recs;
  {
    std::lock_guard<std::mutex> l(mu);
    alive = false;
    recs.swap(held);
  }
  for (const Rec& r : recs) {
    DevBuf b;  // no hold: released at once
    b.ctx = ctx;
    b.p = r.p;
    b.bytes = r.bytes;
    b.fromArena = r.fromArena;
  }
}

}  // namespace aifmm

using namespace aifmm;


extern "C" {

const char* aifmm_last_error(void) { return g_last_error.c_str(); }

int aifmm_profile_ops(int on) {
  API_BEGIN
  AIFMM_REQUIRE(on >= 0 && on <= 2, AIFMM_EINVAL, "mode must be 0 (off), 1 (synchronising) or 2 (host time)");
  opprof::enable(on);
  API_END
}

int aifmm_profile_ops_read(char* buf, int cap) {
  API_BEGIN
  AIFMM_REQUIRE(buf && cap > 0, AIFMM_EINVAL, "bad buffer");
  const std::string r = opprof::report();
  const size_t n = std::min(r.size(), (size_t)cap - 1);
  std::memcpy(buf, r.data(), n);
  buf[n] = 0;
  API_END
}

int aifmm_tc5_timeouts(long* n) {
  API_BEGIN
  AIFMM_REQUIRE(n, AIFMM_EINVAL, "NULL argument");
  *n = tc_timeouts();
  API_END
}

int aifmm_debug_gemm_hold(aifmm_ctx* ctx, int on) {
  API_BEGIN
  AIFMM_REQUIRE(ctx, AIFMM_EINVAL, "ctx is NULL");
  AIFMM_CUDA(cudaSetDevice(ctx->device));
  if (on && !ctx->holdFlag) {
    AIFMM_CUDA(cudaMalloc((void**)&ctx->holdFlag, sizeof(int)));
    AIFMM_CUDA(cudaMemset(ctx->holdFlag, 0, sizeof(int)));
  }
  ctx->gemmHold = on != 0;
  API_END
}

int aifmm_launch_count(long* n) {
  if (!n) return AIFMM_EINVAL;
  *n = launch_count();
  return AIFMM_OK;
}

int aifmm_ctx_create(int device, aifmm_ctx** out) {
  API_BEGIN
  AIFMM_REQUIRE(out, AIFMM_EINVAL, "out is NULL");
  int n = 0;
  AIFMM_CUDA(cudaGetDeviceCount(&n));
  AIFMM_REQUIRE(device >= 0 && device < n, AIFMM_EINVAL, "no such CUDA device");
  AIFMM_CUDA(cudaSetDevice(device));
  std::unique_ptr<aifmm_ctx> c(new aifmm_ctx);
  c->device = device;
  AIFMM_CUDA(cudaDeviceGetAttribute(&c->numSMs, cudaDevAttrMultiProcessorCount, device));
  AIFMM_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  AIFMM_CUDA(cudaMemPoolCreate(&c->pool, &props));
  uint64_t thresh = UINT64_MAX;  // keep freed blocks for reuse
  AIFMM_CUDA(cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &thresh));
  AIFMM_CUDA(cudaMallocHost((void**)&c->ring, aifmm_ctx::kRingBytes));
  {
    aifmm_ctx* cp = c.get();
    c->arena.reset(new Arena([cp](size_t bytes) -> uint64_t {
      void* q = nullptr;
      cudaStream_t s = cp->capture ? cp->sideStream : cp->stream;  // outside a capture in progress
      if (cudaMallocFromPoolAsync(&q, bytes, cp->pool, s) != cudaSuccess ||
          (cp->capture && cudaStreamSynchronize(s) != cudaSuccess)) {
        cudaGetLastError();
        return 0;
      }
      return (uint64_t)q;
    }));
  }
  for (int i = 0; i < aifmm_ctx::kRingChunks; ++i)
    AIFMM_CUDA(cudaEventCreateWithFlags(&c->ringEvent[i], cudaEventDisableTiming));
  *out = c.release();
  API_END
}

int aifmm_ctx_destroy(aifmm_ctx* ctx) {
  API_BEGIN
  if (!ctx) return AIFMM_OK;
  AIFMM_REQUIRE(!ctx->closed, AIFMM_ESTATE, "context destroyed twice");
  ctx->closed = true;
  ctx_release(ctx);
  API_END
}

int aifmm_ctx_synchronize(aifmm_ctx* ctx) {
  API_BEGIN
  AIFMM_REQUIRE(ctx, AIFMM_EINVAL, "ctx is NULL");
  AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
  API_END
}

int aifmm_ctx_stream(aifmm_ctx* ctx, void** stream) {
  API_BEGIN
  AIFMM_REQUIRE(ctx && stream, AIFMM_EINVAL, "NULL argument");
  *stream = (void*)ctx->stream;
  API_END
}

int aifmm_ctx_set_gemm_tiling(aifmm_ctx* ctx, int form, int raster) {
  API_BEGIN
  AIFMM_REQUIRE(ctx && (form == 0 || form == 1) && (raster == 0 || raster == 1), AIFMM_EINVAL,
                "form and raster must be 0 or 1");
  ctx->gemmForm = form;
  ctx->gemmRaster = raster;
  API_END
}

int aifmm_ctx_memory(aifmm_ctx* ctx, size_t* live, size_t* reserved) {
  API_BEGIN
  AIFMM_REQUIRE(ctx, AIFMM_EINVAL, "NULL context");
  if (live) *live = ctx->bytes_live;
  if (reserved) {
    unsigned long long r = 0;  // the attribute is a 64-bit unsigned value
    AIFMM_CUDA(cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReservedMemCurrent, &r));
    *reserved = (size_t)r;
  }
  API_END
}

int aifmm_ctx_trim(aifmm_ctx* ctx) {
  API_BEGIN
  AIFMM_REQUIRE(ctx, AIFMM_EINVAL, "NULL context");
  AIFMM_CUDA(cudaSetDevice(ctx->device));
  ctx_trim(ctx);
  API_END
}

int aifmm_ctx_tune_report(aifmm_ctx* ctx, char* buf, int cap, int* len) {
  API_BEGIN
  AIFMM_REQUIRE(ctx && len, AIFMM_EINVAL, "NULL argument");
  const std::string r = tune_report(ctx);
  *len = (int)r.size();
  if (buf && cap > 0) {
    const int n = std::min((int)r.size(), cap - 1);
    std::memcpy(buf, r.data(), (size_t)n);
    buf[n] = 0;
  }
  API_END
}

int aifmm_kernel_create_efie(aifmm_ctx* ctx, const double* nodes, int n_nodes, const int* tris, int n_tris,
                             double freq, aifmm_kernel** out) {
  API_BEGIN
  AIFMM_REQUIRE(ctx && nodes && tris && out, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(n_nodes > 0 && n_tris > 0, AIFMM_EINVAL, "empty mesh");
  AIFMM_REQUIRE(freq > 0 && std::isfinite(freq), AIFMM_EINVAL, "frequency must be positive");
  AIFMM_CUDA(cudaSetDevice(ctx->device));
  EfieHostTables h;
  build_efie_tables_gpu(ctx, nodes, n_nodes, tris, n_tris, h);
  AIFMM_REQUIRE(!h.len.empty(), AIFMM_EINVAL, "mesh has no RWG (shared) edges");
  std::unique_ptr<aifmm_kernel> k(new aifmm_kernel);
  k->ctx = ctx;
  k->d_tri = upload(ctx, h.tri);
  k->d_node = upload(ctx, h.node);
  k->d_rwg = upload(ctx, h.rwg);
  k->d_len = upload(ctx, h.len);
  k->d_side = upload(ctx, h.side);
  k->locations = h.locations;
  k->rwg_host = h.rwg;
  k->edge_host = h.edge;
  KernelGeom& g = k->geom;
  g.efie = true;
  g.N = (int)h.len.size();
  EfieGeom& e = g.ge;
  e.N = g.N;
  e.nt = n_tris;
  e.tri = k->d_tri.as<double>();
  e.node = k->d_node.as<double>();
  e.rwg = k->d_rwg.as<int4>();
  e.len = k->d_len.as<double>();
  e.side = k->d_side.as<double>();
  // include/includes.hpp:53-63 with a runtime frequency
  const double PI = 4.0 * std::atan(1.0);
  const double c = 3.0e8, lambda = c / freq;
  e.PI = PI;
  e.freq = freq;
  e.eps = 8.854187817e-12;
  e.mu = 4 * PI * 1e-7;
  e.kappa = 2 * PI / lambda;
  e.c4 = -1.0 / 4.0 / PI;
  AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx_retain(ctx);
  *out = k.release();
  API_END
}

int aifmm_kernel_create_es(aifmm_ctx* ctx, const double* nodes, int n_nodes, const int* tris, const int* cond,
                           int n_tris, aifmm_kernel** out) {
  API_BEGIN
  AIFMM_REQUIRE(ctx && nodes && tris && out, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(n_nodes > 0 && n_tris > 0, AIFMM_EINVAL, "empty mesh");
  AIFMM_CUDA(cudaSetDevice(ctx->device));
  std::vector<double> tri, loc;
  build_es_tables(nodes, n_nodes, tris, n_tris, tri, loc);
  std::unique_ptr<aifmm_kernel> k(new aifmm_kernel);
  k->ctx = ctx;
  k->d_tri = upload(ctx, tri);
  k->locations = loc;
  k->cond.assign(n_tris, 1);
  if (cond) k->cond.assign(cond, cond + n_tris);
  KernelGeom& g = k->geom;
  g.efie = false;
  g.N = n_tris;
  g.gs.N = n_tris;
  g.gs.tri = k->d_tri.as<double>();
  const double PI = 4.0 * std::atan(1.0);
  g.gs.C0 = 1.0 / (4 * PI * 8.854187817e-12);
  AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx_retain(ctx);
  *out = k.release();
  API_END
}

int aifmm_kernel_destroy(aifmm_kernel* k) {
  API_BEGIN
  if (!k) return AIFMM_OK;
  aifmm_ctx* c = k->ctx;
  cudaSetDevice(c->device);
  delete k;  // frees the kernel's device tables on the context stream
  ctx_release(c);
  API_END
}

int aifmm_kernel_set_plane_projection(aifmm_kernel* k, int on) {
  API_BEGIN
  AIFMM_REQUIRE(k, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(k->geom.efie, AIFMM_EINVAL, "not an EFIE kernel");
  k->geom.ge.plane_projection = on ? 1 : 0;
  API_END
}

int aifmm_kernel_size(const aifmm_kernel* k, int* n) {
  API_BEGIN
  AIFMM_REQUIRE(k && n, AIFMM_EINVAL, "NULL argument");
  *n = k->geom.N;
  API_END
}

int aifmm_kernel_locations(const aifmm_kernel* k, double* xyz) {
  API_BEGIN
  AIFMM_REQUIRE(k && xyz, AIFMM_EINVAL, "NULL argument");
  std::memcpy(xyz, k->locations.data(), k->locations.size() * sizeof(double));
  API_END
}

static void check_ids(const int* ids, int n, int N, const char* what) {
  for (int i = 0; i < n; ++i)
    AIFMM_REQUIRE(ids[i] >= 0 && ids[i] < N, AIFMM_EINVAL, std::string(what) + " index out of range");
}

int aifmm_kernel_matrix(aifmm_kernel* k, const int* rows, int nr, const int* cols, int nc, int precision, void* out,
                        int ld) {
  API_BEGIN
  AIFMM_REQUIRE(k && rows && cols && out, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(nr >= 0 && nc >= 0 && ld >= nr, AIFMM_EINVAL, "bad sizes");
  AIFMM_REQUIRE(precision == 0 || precision == 1, AIFMM_EINVAL, "precision must be 0 or 1");
  if (nr == 0 || nc == 0) return AIFMM_OK;
  check_ids(rows, nr, k->geom.N, "row");
  check_ids(cols, nc, k->geom.N, "column");
  aifmm_ctx* c = k->ctx;
  AIFMM_CUDA(cudaSetDevice(c->device));
  const size_t esz = precision == 0 ? sizeof(zd) : sizeof(zf);
  DevBuf dr(c, sizeof(int) * nr), dc(c, sizeof(int) * nc), dout(c, esz * (size_t)ld * nc);
  AIFMM_CUDA(cudaMemcpyAsync(dr.p, rows, sizeof(int) * nr, cudaMemcpyHostToDevice, c->stream));
  AIFMM_CUDA(cudaMemcpyAsync(dc.p, cols, sizeof(int) * nc, cudaMemcpyHostToDevice, c->stream));
  launch_gather(k->geom, dr.as<int>(), nr, dc.as<int>(), nc, precision, dout.p, ld, c->stream);
  AIFMM_CUDA(cudaMemcpyAsync(out, dout.p, esz * (size_t)ld * nc, cudaMemcpyDeviceToHost, c->stream));
  AIFMM_CUDA(cudaStreamSynchronize(c->stream));
  API_END
}

int aifmm_kernel_matrix_device(aifmm_kernel* k, const int* rows_device, int nr, const int* cols_device, int nc,
                               int precision, void* out_device, int ld) {
  API_BEGIN
  AIFMM_REQUIRE(k && rows_device && cols_device && out_device, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(nr >= 0 && nc >= 0 && ld >= nr, AIFMM_EINVAL, "bad sizes");
  AIFMM_REQUIRE(precision == 0 || precision == 1, AIFMM_EINVAL, "precision must be 0 or 1");
  AIFMM_CUDA(cudaSetDevice(k->ctx->device));
  launch_gather(k->geom, rows_device, nr, cols_device, nc, precision, out_device, ld, k->ctx->stream);
  API_END
}

int aifmm_kernel_rhs_reference(aifmm_kernel* k, const double einc[3], double* out) {
  API_BEGIN
  AIFMM_REQUIRE(k && einc && out, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(k->geom.efie, AIFMM_EINVAL, "not an EFIE kernel");
  aifmm_ctx* c = k->ctx;
  AIFMM_CUDA(cudaSetDevice(c->device));
  DevBuf d(c, sizeof(zd) * k->geom.N);
  launch_rhs_reference(k->geom, einc, d.as<zd>(), c->stream);
  AIFMM_CUDA(cudaMemcpyAsync(out, d.p, sizeof(zd) * k->geom.N, cudaMemcpyDeviceToHost, c->stream));
  AIFMM_CUDA(cudaStreamSynchronize(c->stream));
  API_END
}

int aifmm_kernel_rhs_plane(aifmm_kernel* k, const double khat[3], const double e0[6], double* out) {
  API_BEGIN
  AIFMM_REQUIRE(k && khat && e0 && out, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(k->geom.efie, AIFMM_EINVAL, "not an EFIE kernel");
  aifmm_ctx* c = k->ctx;
  AIFMM_CUDA(cudaSetDevice(c->device));
  DevBuf d(c, sizeof(zd) * k->geom.N);
  launch_rhs_plane(k->geom, khat, e0, d.as<zd>(), c->stream);
  AIFMM_CUDA(cudaMemcpyAsync(out, d.p, sizeof(zd) * k->geom.N, cudaMemcpyDeviceToHost, c->stream));
  AIFMM_CUDA(cudaStreamSynchronize(c->stream));
  API_END
}

int aifmm_kernel_rhs_conductor(aifmm_kernel* k, int conductor, double* out) {
  API_BEGIN
  AIFMM_REQUIRE(k && out, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(!k->geom.efie, AIFMM_EINVAL, "not an electrostatics kernel");
  for (int i = 0; i < k->geom.N; ++i) {  // a 0/1 indicator vector: no arithmetic to offload
    out[2 * i] = (k->cond[i] == conductor) ? 1.0 : 0.0;
    out[2 * i + 1] = 0.0;
  }
  API_END
}

}  // extern "C"
