// Device matrices with value semantics for the solver's host orchestration:
// every block of the H^2 factorization lives in HBM; the host only keeps
// shapes, ids and pointers.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "dense.cuh"

namespace aifmm {

// Per-operation accounting of the host-driven factorization, for diagnosis:
// off by default.  Mode 1: each instrumented scope synchronises the stream on
// exit, so its time is host enqueue + device execution of that operation.
// Mode 2: scopes record host time only (no synchronisation), and the time the
// host spends blocked on the device ("sync_wait") and in the memory pool
// ("pool_alloc", "pool_free") is recorded too, which splits a host-driven
// run into host work and waiting for the GPU.
namespace opprof {
void enable(int mode);
bool enabled();
int mode();
double now();
void add(const char* name, double seconds);
std::string report();
// cudaStreamSynchronize, accounted as "sync_wait" when profiling is on
cudaError_t sync(cudaStream_t s);
// The names of the instrumented scopes open on this thread, outermost first,
// joined by '/' (for tagging device-time records).
std::string path();
struct Scope {
  const char* name;
  cudaStream_t stream;
  double t0;
  Scope(const char* n, cudaStream_t s);
  ~Scope();
};
}  // namespace opprof

struct DMat {
  std::shared_ptr<DevBuf> buf;
  zd* p = nullptr;
  int r = 0, c = 0;
  long size() const { return (long)r * c; }
  int ld() const { return r > 0 ? r : 1; }
};

struct DLU {
  DMat lu;
  std::shared_ptr<DevBuf> piv, info;
  int n = 0;
};

// Collects GEMMs and launches them as one grouped kernel.
struct GemmBatch {
  std::vector<GemmProblem> probs;
  void add(DMat& C, const DMat& A, int opA, const DMat& B, int opB, zd alpha, zd beta);
  void flush(aifmm_ctx* ctx);
};

struct Ops {
  aifmm_ctx* ctx;
  explicit Ops(aifmm_ctx* c) : ctx(c) {}
  DMat alloc(int r, int c) const;
  // Several matrices carved out of shared device allocations (slabs of up to
  // 16 MB, each matrix 512-byte aligned): one pool allocation per slab
  // instead of one per matrix.  A slab's memory returns to the pool when the
  // last matrix in it is released.
  std::vector<DMat> allocMany(const std::vector<std::pair<int, int>>& shapes) const;
  DMat zeros(int r, int c) const;
  DMat ident(int n, zd d) const;
  DMat copy(const DMat& a) const;
  DMat block(const DMat& a, int i0, int j0, int nr, int nc) const;
  DMat adj(const DMat& a) const;
  DMat neg(const DMat& a) const;
  DMat hcat(const DMat& a, const DMat& b) const;
  DMat vcat(const std::vector<DMat>& parts) const;
  DMat hcatv(const std::vector<DMat>& parts) const;
  DMat mul(const DMat& a, int opA, const DMat& b, int opB, zd alpha = zmk(1, 0)) const;
  void setBlock(DMat& dst, int i0, int j0, const DMat& src) const;
  std::vector<double> norms(const std::vector<const DMat*>& ms) const;  // synchronises
  double norm(const DMat& a) const { return norms({&a})[0]; }
  double maxColNorm(const DMat& a) const;                                // synchronises
  DLU factor(const DMat& a) const;
  DMat solve(const DLU& f, const DMat& b) const;
  void sync() const;
  std::vector<zd> download(const DMat& a) const;                        // synchronises
  DMat fromHost(const std::vector<zd>& v, int r, int c) const;
};

}  // namespace aifmm
