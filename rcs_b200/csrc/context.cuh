// Library context: one device, one stream, a stream-ordered device memory
// pool, and the kernel (mesh) objects.
#pragma once
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "arena.cuh"
#include "assemble.cuh"

namespace aifmm {
struct CaptureHold;
}

// Objects created on a context (kernels, solvers) hold a reference; the
// context's stream and memory pool are released when aifmm_ctx_destroy has
// been called and the last such object is gone, so destruction order does
// not matter to callers.
struct aifmm_ctx {
  int device = 0;
  int numSMs = 0;        // streaming multiprocessors of the device (persistent-kernel grids)
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;
  size_t bytes_live = 0;
  int refs = 1;          // the creator's reference
  int gemmRaster = 0;    // tile order of the persistent tensor-core GEMM (set by the autotuner)
  bool splitK = true;    // FP64 launches with few output tiles and long depths split their depth
  int gemmForm = 1;      // operand form of the persistent tensor-core GEMM: 0 packed real, 1 split planes
                         // (the default: 32 instead of 48 KB per 8-deep step; faster on the solver's products)
  // Autotuner choices of the tensor-core GEMM by launch class (autotune.cu)
  std::mutex tuneMu;
  std::map<long long, int> tuneCache;
  std::vector<std::string> tuneLog;
  int gemmPrecision = 0; // grouped GEMMs: 0 complex128 FMA; split TF32 (FP32 accuracy) on the tensor
                         // cores: 1 mma.sync, 2 tcgen05 with tensor-memory accumulators
  // Pinned staging ring for the small host-to-device uploads (problem lists,
  // index arrays): a copy from pinned memory is asynchronous, one from
  // pageable memory is not.  Each chunk remembers the event of its last copy
  // and the lap of the ring it was written in; a chunk written in an earlier
  // lap is reused only after that copy completed.
  static constexpr size_t kRingBytes = (size_t)32 << 20, kRingChunk = (size_t)512 << 10;
  static constexpr int kRingChunks = (int)(kRingBytes / kRingChunk);
  char* ring = nullptr;
  size_t ringHead = 0;
  long ringLap = 1;
  cudaEvent_t ringEvent[kRingChunks] = {};
  long ringChunkLap[kRingChunks] = {};  // 0: never used
  bool closed = false;
  // Wait test of the tensor-core GEMMs (aifmm_debug_gemm_hold): when set, their
  // issuing thread first waits, bounded by 1 ms, on `holdFlag`, a device int
  // that stays zero, so every tile times out and the call reports
  // AIFMM_ETIMEOUT.
  bool gemmHold = false;
  int* holdFlag = nullptr;
  // Rank model used by solvers built on this context to size each box's ACA
  // workspace (aifmm_ctx_set_rank_model keeps a copy; null: fixed bound).
  std::shared_ptr<struct aifmm_mlp> rankModel;
  double rankMargin = 1.25;
  // Sub-allocator for the blocks of 256 KB and more (arena.cuh); its chunks
  // come from `pool`.  Created with the context.
  std::mutex arenaMu;
  std::unique_ptr<aifmm::Arena> arena;
  // While a CUDA graph is being captured on `stream` (the solver's solve
  // plans), `capture` is set: device allocations and host uploads then go
  // through `sideStream`, outside the capture, and every buffer allocated
  // during the capture stays reserved for the graph until the graph is
  // destroyed (CaptureHold).
  std::shared_ptr<aifmm::CaptureHold> capture;
  cudaStream_t sideStream = nullptr;
};

namespace aifmm {
void ctx_retain(aifmm_ctx* c);
void ctx_release(aifmm_ctx* c);
// Drains the stream and returns unused arena chunks and pooled blocks to the device.
void ctx_trim(aifmm_ctx* c);
}  // namespace aifmm

namespace aifmm {

// Device memory that a captured CUDA graph reads or writes.  A replay of the
// graph touches the addresses it was captured with, so none of them may go
// back to the pool or the arena while the graph exists: a buffer allocated
// during the capture carries the hold, and its release only records it here.
// releaseAll(), called once the graph is destroyed, returns what was recorded;
// buffers released after that go back at once.
struct CaptureHold {
  struct Rec {
    void* p;
    size_t bytes;
    bool fromArena;
  };
  aifmm_ctx* ctx = nullptr;
  std::mutex mu;
  bool alive = true;
  std::vector<Rec> held;
  void releaseAll();
};

// Device buffer allocated from the context's stream-ordered pool.
struct DevBuf {
  aifmm_ctx* ctx = nullptr;
  void* p = nullptr;
  size_t bytes = 0;
  bool fromArena = false;  // p came from the context's arena, not the pool
  std::shared_ptr<CaptureHold> hold;  // allocated while a graph was captured
  DevBuf() {}
  DevBuf(aifmm_ctx* c, size_t n) { alloc(c, n); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : ctx(o.ctx), p(o.p), bytes(o.bytes), fromArena(o.fromArena), hold(std::move(o.hold)) {
    o.p = nullptr;
    o.bytes = 0;
    o.fromArena = false;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      ctx = o.ctx; p = o.p; bytes = o.bytes; fromArena = o.fromArena; hold = std::move(o.hold);
      o.p = nullptr; o.bytes = 0; o.fromArena = false;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(aifmm_ctx* c, size_t n);
  void release();
  template <typename T>
  T* as() const { return static_cast<T*>(p); }
};

// Asynchronous host-to-device copy of n bytes on the context stream, staged
// through the pinned ring when it fits (see aifmm_ctx).
void upload_bytes(aifmm_ctx* c, void* dst, const void* src, size_t n);

template <typename T>
DevBuf upload(aifmm_ctx* c, const std::vector<T>& v) {
  DevBuf b(c, std::max<size_t>(1, v.size() * sizeof(T)));
  if (!v.empty()) upload_bytes(c, b.p, v.data(), v.size() * sizeof(T));
  return b;
}

}  // namespace aifmm

struct aifmm_kernel {
  aifmm_ctx* ctx = nullptr;
  aifmm::KernelGeom geom;
  aifmm::DevBuf d_tri, d_node, d_rwg, d_len, d_side;
  aifmm::DevBuf d_t2e_off, d_t2e_inc;  // EFIE: triangle -> RWG edge incidence, built on first use
  std::vector<double> locations;   // N x 3
  std::vector<int> cond;           // electrostatics: conductor per triangle
  std::vector<int> rwg_host;       // EFIE: N x 4
  std::vector<int> edge_host;      // EFIE: N x 2
};
