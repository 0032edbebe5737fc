// aifmm_rrqr_noalloc: the partitioned column-pivoted QR for callers that may
// not allocate device memory -- code that runs inside another framework's
// memory manager, on a stream that is being captured into a CUDA graph by a
// host that forbids allocation during capture, or under a strict memory
// budget that pre-reserves everything.  Such callers pass device pointers to
// their own input and outputs; the working storage (the copy of A that the
// factorization overwrites, the Householder vectors, the column norms and the
// permutation) lives in the fixed-size device array below, which every GPU
// that loads this library keeps until the process exits.
//
// Set-up: the first call in a CUDA context (normally a device's primary
// context), with that device current, looks up the array's device address
// with cudaGetSymbolAddress (the name of a __device__ array is only a
// host-side stand-in, not a device address) and caches it for that context.
// Make that first call before any stream capture.  A context created later
// (after cudaDeviceReset, or another context made current) gets its own
// lookup on its first call.
//
// All calls share the one array: calls whose work overlaps on the GPU (two
// streams, or two host threads) race and corrupt each other.  Serialise them,
// e.g. on one stream.
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>

#include "lowrank.cuh"

namespace aifmm {

// Defined in lowrank.cu; launched unchanged with 1024 threads per block.
__global__ void rrqr_kernel(const RRQRProblem* __restrict__ probs);
constexpr int kRRQRThreads = 1024;

// 32 MiB of scratch: enough for an m x n problem with
// 16 (m n + m (min(m, n) + 1)) + 12 n + 1 KiB <= 32 MiB, e.g. 1000 x 1000.
constexpr size_t kNoAllocScratchBytes = (size_t)32 << 20;
static __device__ __align__(256) unsigned char g_rrqr_scratch[kNoAllocScratchBytes];

// The descriptor of the problem sits in the array's first KiB.
static_assert(sizeof(RRQRProblem) <= 1024, "the RRQR descriptor must fit the scratch array's first KiB");

static std::mutex g_scratch_mu;
static std::map<CUcontext, void*> g_scratch_addr;  // per CUDA context

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// The calling thread's current CUDA context, through the driver entry point
// that the runtime hands out (the library does not link the driver library).
static CUcontext current_context() {
  using Fn = CUresult (*)(CUcontext*);
  static Fn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<Fn>(p);
  });
  CUcontext c = nullptr;
  if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
  return c;
}

__global__ void rrqr_noalloc_setup_kernel(RRQRProblem P, RRQRProblem* dst, const zd* A) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *dst = P;
  const size_t n = (size_t)P.m * P.n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    P.R[i] = A[i];
}

}  // namespace aifmm

using namespace aifmm;

extern "C" int aifmm_rrqr_noalloc(const void* A_device, int m, int n, int partition, int tol_pow1, int tol_pow2,
                                  double input_pivot, int fill_rank, int real_mode, void* Q_device,
                                  int* rank_device, double* max_pivot_device, void* stream) {
  try {
    AIFMM_REQUIRE(A_device && Q_device && rank_device && max_pivot_device, AIFMM_EINVAL, "NULL argument");
    AIFMM_REQUIRE(m > 0 && n > 0 && partition >= 0 && partition <= n, AIFMM_EINVAL, "bad sizes");
    AIFMM_REQUIRE(tol_pow1 >= 0 && tol_pow2 >= 0 && fill_rank >= 0, AIFMM_EINVAL,
                  "negative tolerance power or fill-in rank");
    const size_t hs = (size_t)std::min(m, n) + 1;
    const size_t off_R = 1024;
    const size_t off_H = align256(off_R + sizeof(zd) * (size_t)m * n);
    const size_t off_nsq = align256(off_H + sizeof(zd) * (size_t)m * hs);
    const size_t off_perm = align256(off_nsq + sizeof(double) * (size_t)n);
    const size_t need = off_perm + sizeof(int) * (size_t)n;
    AIFMM_REQUIRE(need <= kNoAllocScratchBytes, AIFMM_EOVERFLOW,
                  "problem needs " + std::to_string(need) + " bytes of scratch; the fixed scratch array holds " +
                      std::to_string(kNoAllocScratchBytes));
    CUcontext cu = current_context();
    if (!cu) {
      int dev = 0;  // nothing current yet: cudaSetDevice makes the device's primary context current
      AIFMM_CUDA(cudaGetDevice(&dev));
      AIFMM_CUDA(cudaSetDevice(dev));
      cu = current_context();
      AIFMM_REQUIRE(cu, AIFMM_ECUDA, "no current CUDA context");
    }
    void* base = nullptr;
    {
      std::lock_guard<std::mutex> l(g_scratch_mu);
      auto it = g_scratch_addr.find(cu);
      if (it == g_scratch_addr.end()) {
        void* p = nullptr;
        AIFMM_CUDA(cudaGetSymbolAddress(&p, g_rrqr_scratch));  // in this context, with this device current
        it = g_scratch_addr.emplace(cu, p).first;
      }
      base = it->second;
    }
    unsigned char* b = static_cast<unsigned char*>(base);
    RRQRProblem P;
    P.R = reinterpret_cast<zd*>(b + off_R);
    P.m = m;
    P.n = n;
    P.partition = partition;
    P.tol1 = std::pow(10.0, -tol_pow1);
    P.tol2 = std::pow(10.0, -tol_pow2);
    P.inputPivot = input_pivot;
    P.fillInRank = fill_rank;
    P.realMode = real_mode;
    P.H = reinterpret_cast<zd*>(b + off_H);
    P.nsq = reinterpret_cast<double*>(b + off_nsq);
    P.perm = reinterpret_cast<int*>(b + off_perm);
    P.Q = static_cast<zd*>(Q_device);
    P.rank = rank_device;
    P.maxPivot = max_pivot_device;
    P.istate = nullptr;  // the single-kernel form keeps its state in registers
    P.dstate = nullptr;
    P.p2cap = -1;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    RRQRProblem* desc = reinterpret_cast<RRQRProblem*>(b);
    const int grid = (int)std::min<size_t>(((size_t)m * n + 255) / 256, 148 * 4);
    rrqr_noalloc_setup_kernel<<<std::max(grid, 1), 256, 0, s>>>(P, desc, static_cast<const zd*>(A_device));
    AIFMM_LAUNCHED();
    rrqr_kernel<<<1, kRRQRThreads, 0, s>>>(desc);
    AIFMM_LAUNCHED();
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return AIFMM_EINVAL;
  }
  return AIFMM_OK;
}
