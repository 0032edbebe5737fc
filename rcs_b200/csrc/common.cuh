// Shared helpers of the B200 AIFMM library: status handling, complex
// arithmetic on double2/float2, and small device utilities.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../include/aifmm_b200.h"

namespace aifmm {

// Error carried from deep inside the library to the C ABI boundary.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);
// cudaFuncSetAttribute(kernel, MaxDynamicSharedMemorySize, bytes) once per
// (kernel, device), safe to call from several host threads; the device must
// be current.
void smem_attr_once(const void* kernel, int device, int bytes);
// Number of kernels this library has launched (all contexts, process-wide).
void count_launch(long n = 1);
long launch_count();
// The launches counted on the calling thread only (for a thread's own
// before/after differences while other threads launch too).
long thread_launch_count();

#define AIFMM_CUDA(expr)                                                                                  \
  do {                                                                                                    \
    cudaError_t _e = (expr);                                                                              \
    if (_e != cudaSuccess)                                                                                \
      throw ::aifmm::Error(AIFMM_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(_e) + " at " +     \
                                            __FILE__ + ":" + std::to_string(__LINE__));                   \
  } while (0)

// After every kernel launch: surface launch errors and count the launch.
#define AIFMM_LAUNCHED()                \
  do {                                  \
    AIFMM_CUDA(cudaGetLastError());     \
    ::aifmm::count_launch();            \
  } while (0)

#define AIFMM_REQUIRE(cond, code, msg)                 \
  do {                                                 \
    if (!(cond)) throw ::aifmm::Error((code), (msg)); \
  } while (0)

// ---------------------------------------------------------------- complex
typedef double2 zd;
typedef float2 zf;

__host__ __device__ __forceinline__ zd zmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ zd zadd(zd a, zd b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ zd zsub(zd a, zd b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ zd zmul(zd a, zd b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ zd zscale(zd a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ zd zconj(zd a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ double zabs2(zd a) { return a.x * a.x + a.y * a.y; }
// conj(a) * b
__host__ __device__ __forceinline__ zd zcmul(zd a, zd b) {
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
// a / b by scaling with the larger component (Smith's method).
__host__ __device__ __forceinline__ zd zdiv(zd a, zd b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, d = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  } else {
    double r = b.x / b.y, d = b.y + b.x * r;
    return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
}

__host__ __device__ __forceinline__ zf cmk(float r, float i) { return make_float2(r, i); }

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

}  // namespace aifmm
