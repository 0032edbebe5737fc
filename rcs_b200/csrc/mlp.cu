// Rank model kernels: forward, backward and Adam for the 6 -> 64 -> 64 -> 1
// perceptron of mlp.cuh.  BF16 weights (rounded from the FP32 master copy
// once per step), FP32 activations and FP32 accumulation.
//
// One 64-thread block walks a fixed range of samples in order; thread u owns
// hidden unit u of both layers, so it alone accumulates that unit's weight
// gradients (row u of W1 and of W2, b1[u], b2[u], w3[u]) in shared memory.
// The per-block sums are then added block by block in a fixed order: the
// gradient does not depend on timing, and repeated runs give the same bits.
//
// Training replays one captured CUDA graph of TRAIN_EPOCHS_PER_GRAPH steps
// (gradient, block reduction, Adam), so a few thousand steps cost a few
// hundred graph launches.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "capi_guard.cuh"
#include "mlp.cuh"

namespace aifmm {

namespace {

constexpr int MLP_THREADS = MLP_H;  // one thread per hidden unit
constexpr int TRAIN_EPOCHS_PER_GRAPH = 50;

struct MlpNorm {
  float mean[MLP_IN], scale[MLP_IN];
};

// Loads the BF16 weights into shared memory as FP32 (exact: BF16 -> FP32).
__device__ __forceinline__ void mlp_load_weights(const __nv_bfloat16* __restrict__ w, float* ws) {
  for (int p = threadIdx.x; p < MLP_NP; p += blockDim.x) ws[p] = __bfloat162float(w[p]);
}

// Forward pass of one sample: xs (normalised input) must be in shared memory.
// Returns this thread's pre-activations z1, z2; a1 (shared) gets layer 1's
// activations; the block-wide output y is returned to every thread.
__device__ __forceinline__ float mlp_forward_one(const float* ws, const float* xs, float* a1, float* red, float& z1,
                                                 float& z2, float& a2) {
  const int u = threadIdx.x;
  float acc = ws[MLP_B1 + u];
#pragma unroll
  for (int i = 0; i < MLP_IN; ++i) acc += ws[MLP_W1 + u * MLP_IN + i] * xs[i];
  z1 = acc;
  a1[u] = fmaxf(acc, 0.0f);
  __syncthreads();
  acc = ws[MLP_B2 + u];
  for (int h = 0; h < MLP_H; ++h) acc += ws[MLP_W2 + u * MLP_H + h] * a1[h];
  z2 = acc;
  a2 = fmaxf(acc, 0.0f);
  float p = ws[MLP_W3 + u] * a2;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
  if ((u & 31) == 0) red[u >> 5] = p;
  __syncthreads();
  const float y = ws[MLP_B3] + (red[0] + red[1]);
  return y;
}

__global__ void __launch_bounds__(MLP_THREADS) mlp_forward_kernel(const __nv_bfloat16* __restrict__ w, MlpNorm nrm,
                                                                  const float* __restrict__ X, int n,
                                                                  float* __restrict__ y) {
  __shared__ float ws[MLP_NP];
  __shared__ float xs[MLP_IN], a1[MLP_H], red[2];
  mlp_load_weights(w, ws);
  __syncthreads();
  for (int s = blockIdx.x; s < n; s += gridDim.x) {
    if (threadIdx.x < MLP_IN)
      xs[threadIdx.x] = (X[(size_t)s * MLP_IN + threadIdx.x] - nrm.mean[threadIdx.x]) * nrm.scale[threadIdx.x];
    __syncthreads();
    float z1, z2, a2;
    const float out = mlp_forward_one(ws, xs, a1, red, z1, z2, a2);
    if (threadIdx.x == 0) y[s] = out;
    __syncthreads();
  }
}

// Gradient of L = (1/n) sum_s (y_s - t_s)^2 over the samples of this block
// ([blockIdx.x * per, min(n, (blockIdx.x + 1) * per))); partial[b] gets
// MLP_NP gradient entries followed by this block's sum of squared errors.
__global__ void __launch_bounds__(MLP_THREADS) mlp_grad_kernel(const __nv_bfloat16* __restrict__ w, MlpNorm nrm,
                                                               const float* __restrict__ X,
                                                               const float* __restrict__ T, int n, int per,
                                                               float* __restrict__ partial) {
  __shared__ float ws[MLP_NP];
  __shared__ float g[MLP_NP + 1];
  __shared__ float xs[MLP_IN], a1[MLP_H], d2s[MLP_H], red[2];
  const int u = threadIdx.x;
  mlp_load_weights(w, ws);
  for (int p = u; p < MLP_NP + 1; p += blockDim.x) g[p] = 0.0f;
  __syncthreads();
  const float inv_n = 1.0f / (float)n;
  const int s0 = blockIdx.x * per, s1 = min(n, s0 + per);
  for (int s = s0; s < s1; ++s) {
    if (u < MLP_IN) xs[u] = (X[(size_t)s * MLP_IN + u] - nrm.mean[u]) * nrm.scale[u];
    __syncthreads();
    float z1, z2, a2;
    const float y = mlp_forward_one(ws, xs, a1, red, z1, z2, a2);
    const float r = y - T[s];
    const float dy = 2.0f * r * inv_n;
    if (u == 0) {
      g[MLP_B3] += dy;
      g[MLP_NP] += r * r;
    }
    g[MLP_W3 + u] += dy * a2;
    const float d2 = (z2 > 0.0f) ? dy * ws[MLP_W3 + u] : 0.0f;
    g[MLP_B2 + u] += d2;
    for (int h = 0; h < MLP_H; ++h) g[MLP_W2 + u * MLP_H + h] += d2 * a1[h];
    d2s[u] = d2;
    __syncthreads();
    float acc = 0.0f;
    for (int o = 0; o < MLP_H; ++o) acc += ws[MLP_W2 + o * MLP_H + u] * d2s[o];
    const float d1 = (z1 > 0.0f) ? acc : 0.0f;
    g[MLP_B1 + u] += d1;
#pragma unroll
    for (int i = 0; i < MLP_IN; ++i) g[MLP_W1 + u * MLP_IN + i] += d1 * xs[i];
    __syncthreads();
  }
  for (int p = u; p < MLP_NP + 1; p += blockDim.x) partial[(size_t)blockIdx.x * (MLP_NP + 1) + p] = g[p];
}

// out[p] = sum over blocks b = 0, 1, ... of partial[b][p] (fixed order).
__global__ void mlp_reduce_kernel(const float* __restrict__ partial, int nblk, float* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > MLP_NP) return;
  float s = 0.0f;
  for (int b = 0; b < nblk; ++b) s += partial[(size_t)b * (MLP_NP + 1) + p];
  out[p] = s;
}

// One Adam step on the FP32 master weights (single block; the step counter
// lives on the device so that a captured graph can replay steps), then the
// BF16 copy that the next forward pass reads.
__global__ void mlp_adam_kernel(float* __restrict__ master, const float* __restrict__ grad, float* __restrict__ m1,
                                float* __restrict__ m2, int* __restrict__ step, float lr,
                                __nv_bfloat16* __restrict__ w) {
  const int t = *step + 1;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
  for (int p = threadIdx.x; p < MLP_NP; p += blockDim.x) {
    const float gp = grad[p];
    const float a = b1 * m1[p] + (1.0f - b1) * gp;
    const float b = b2 * m2[p] + (1.0f - b2) * gp * gp;
    m1[p] = a;
    m2[p] = b;
    const float v = master[p] - lr * (a / c1) / (sqrtf(b / c2) + eps);
    master[p] = v;
    w[p] = __float2bfloat16_rn(v);
  }
  __syncthreads();
  if (threadIdx.x == 0) *step = t;
}

__global__ void mlp_round_kernel(const float* __restrict__ master, __nv_bfloat16* __restrict__ w) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < MLP_NP; p += gridDim.x * blockDim.x)
    w[p] = __float2bfloat16_rn(master[p]);
}

MlpNorm norm_of(const aifmm_mlp* m) {
  MlpNorm n;
  for (int i = 0; i < MLP_IN; ++i) {
    n.mean[i] = m->mean[i];
    n.scale[i] = m->scale[i];
  }
  return n;
}

// Device copies of the master weights and their BF16 rounding.
struct MlpDevice {
  DevBuf master, w;
  MlpDevice(aifmm_mlp* m) : master(m->ctx, sizeof(float) * MLP_NP), w(m->ctx, sizeof(__nv_bfloat16) * MLP_NP) {
    upload_bytes(m->ctx, master.p, m->params.data(), sizeof(float) * MLP_NP);
    mlp_round_kernel<<<ceil_div(MLP_NP, 256), 256, 0, m->ctx->stream>>>(master.as<float>(),
                                                                      w.as<__nv_bfloat16>());
    AIFMM_LAUNCHED();
  }
};

int grad_blocks(int n, int& per) {
  const int nblk = std::max(1, std::min(ceil_div(n, 8), 148 * 4));
  per = ceil_div(n, nblk);
  return ceil_div(n, per);
}

// splitmix64 stream -> standard normal (Box-Muller), for the seeded initialisation.
struct SeededNormal {
  unsigned long long s;
  double next_u() {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return ((z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  }
  double next() {
    const double a = next_u(), b = next_u();
    return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b);
  }
};

}  // namespace

void mlp_infer(aifmm_mlp* m, const std::vector<RankFeatures>& x, std::vector<float>& y) {
  const int n = (int)x.size();
  y.assign(n, 0.0f);
  if (n == 0) return;
  aifmm_ctx* c = m->ctx;
  MlpDevice d(m);
  DevBuf dx(c, sizeof(float) * MLP_IN * (size_t)n), dy(c, sizeof(float) * (size_t)n);
  upload_bytes(c, dx.p, x.data(), sizeof(float) * MLP_IN * (size_t)n);
  mlp_forward_kernel<<<std::min(n, 148 * 8), MLP_THREADS, 0, c->stream>>>(d.w.as<__nv_bfloat16>(), norm_of(m),
                                                                          dx.as<float>(), n, dy.as<float>());
  AIFMM_LAUNCHED();
  AIFMM_CUDA(cudaMemcpyAsync(y.data(), dy.p, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
  AIFMM_CUDA(cudaStreamSynchronize(c->stream));
}

}  // namespace aifmm

using namespace aifmm;

extern "C" {

int aifmm_mlp_create(aifmm_ctx* ctx, unsigned long long seed, aifmm_mlp** out) {
  API_BEGIN
  AIFMM_REQUIRE(ctx && out, AIFMM_EINVAL, "NULL argument");
  std::unique_ptr<aifmm_mlp> m(new aifmm_mlp);
  m->ctx = ctx;
  m->params.assign(MLP_NP, 0.0f);
  SeededNormal g{seed};
  // He initialisation of the ReLU layers, small output layer, zero biases
  for (int p = 0; p < MLP_H * MLP_IN; ++p) m->params[MLP_W1 + p] = (float)(g.next() * std::sqrt(2.0 / MLP_IN));
  for (int p = 0; p < MLP_H * MLP_H; ++p) m->params[MLP_W2 + p] = (float)(g.next() * std::sqrt(2.0 / MLP_H));
  for (int p = 0; p < MLP_H; ++p) m->params[MLP_W3 + p] = (float)(g.next() * std::sqrt(1.0 / MLP_H));
  ctx_retain(ctx);
  *out = m.release();
  API_END
}

int aifmm_mlp_destroy(aifmm_mlp* m) {
  API_BEGIN
  if (!m) return AIFMM_OK;
  aifmm_ctx* c = m->ctx;
  delete m;
  ctx_release(c);
  API_END
}

int aifmm_mlp_set_normalization(aifmm_mlp* m, const float* mean, const float* scale) {
  API_BEGIN
  AIFMM_REQUIRE(m && mean && scale, AIFMM_EINVAL, "NULL argument");
  for (int i = 0; i < MLP_IN; ++i) {
    AIFMM_REQUIRE(std::isfinite(mean[i]) && std::isfinite(scale[i]), AIFMM_EINVAL, "normalisation not finite");
    m->mean[i] = mean[i];
    m->scale[i] = scale[i];
  }
  API_END
}

int aifmm_mlp_get_params(aifmm_mlp* m, float* params) {
  API_BEGIN
  AIFMM_REQUIRE(m && params, AIFMM_EINVAL, "NULL argument");
  std::memcpy(params, m->params.data(), sizeof(float) * MLP_NP);
  API_END
}

int aifmm_mlp_set_params(aifmm_mlp* m, const float* params) {
  API_BEGIN
  AIFMM_REQUIRE(m && params, AIFMM_EINVAL, "NULL argument");
  for (int p = 0; p < MLP_NP; ++p) AIFMM_REQUIRE(std::isfinite(params[p]), AIFMM_EINVAL, "parameter not finite");
  std::memcpy(m->params.data(), params, sizeof(float) * MLP_NP);
  m->m1.clear();
  m->m2.clear();
  m->adamStep = 0;
  API_END
}

int aifmm_mlp_num_params(int* n) {
  if (!n) return AIFMM_EINVAL;
  *n = MLP_NP;
  return AIFMM_OK;
}

int aifmm_mlp_infer(aifmm_mlp* m, const float* X, int n, float* y) {
  API_BEGIN
  AIFMM_REQUIRE(m && X && y && n >= 0, AIFMM_EINVAL, "bad argument");
  AIFMM_CUDA(cudaSetDevice(m->ctx->device));
  std::vector<RankFeatures> x((size_t)n);
  std::memcpy(x.data(), X, sizeof(float) * MLP_IN * (size_t)n);
  std::vector<float> out;
  mlp_infer(m, x, out);
  if (n) std::memcpy(y, out.data(), sizeof(float) * (size_t)n);
  API_END
}

int aifmm_mlp_grad(aifmm_mlp* m, const float* X, const float* t, int n, float* grad, float* loss) {
  API_BEGIN
  AIFMM_REQUIRE(m && X && t && grad && loss && n > 0, AIFMM_EINVAL, "bad argument");
  aifmm_ctx* c = m->ctx;
  AIFMM_CUDA(cudaSetDevice(c->device));
  MlpDevice d(m);
  DevBuf dx(c, sizeof(float) * MLP_IN * (size_t)n), dt(c, sizeof(float) * (size_t)n);
  upload_bytes(c, dx.p, X, sizeof(float) * MLP_IN * (size_t)n);
  upload_bytes(c, dt.p, t, sizeof(float) * (size_t)n);
  int per = 0;
  const int nblk = grad_blocks(n, per);
  DevBuf part(c, sizeof(float) * (size_t)nblk * (MLP_NP + 1)), g(c, sizeof(float) * (MLP_NP + 1));
  mlp_grad_kernel<<<nblk, MLP_THREADS, 0, c->stream>>>(d.w.as<__nv_bfloat16>(), norm_of(m), dx.as<float>(),
                                                       dt.as<float>(), n, per, part.as<float>());
  AIFMM_LAUNCHED();
  mlp_reduce_kernel<<<ceil_div(MLP_NP + 1, 256), 256, 0, c->stream>>>(part.as<float>(), nblk, g.as<float>());
  AIFMM_LAUNCHED();
  std::vector<float> h(MLP_NP + 1);
  AIFMM_CUDA(cudaMemcpyAsync(h.data(), g.p, sizeof(float) * (MLP_NP + 1), cudaMemcpyDeviceToHost, c->stream));
  AIFMM_CUDA(cudaStreamSynchronize(c->stream));
  std::memcpy(grad, h.data(), sizeof(float) * MLP_NP);
  *loss = h[MLP_NP] / (float)n;
  API_END
}

int aifmm_mlp_train(aifmm_mlp* m, const float* X, const float* t, int n, int epochs, float lr, float* loss_first,
                    float* loss_last) {
  API_BEGIN
  AIFMM_REQUIRE(m && X && t && n > 0 && epochs > 0 && lr > 0.0f, AIFMM_EINVAL, "bad argument");
  aifmm_ctx* c = m->ctx;
  AIFMM_CUDA(cudaSetDevice(c->device));
  MlpDevice d(m);
  DevBuf dx(c, sizeof(float) * MLP_IN * (size_t)n), dt(c, sizeof(float) * (size_t)n);
  upload_bytes(c, dx.p, X, sizeof(float) * MLP_IN * (size_t)n);
  upload_bytes(c, dt.p, t, sizeof(float) * (size_t)n);
  if ((int)m->m1.size() != MLP_NP) {
    m->m1.assign(MLP_NP, 0.0f);
    m->m2.assign(MLP_NP, 0.0f);
    m->adamStep = 0;
  }
  DevBuf dm1(c, sizeof(float) * MLP_NP), dm2(c, sizeof(float) * MLP_NP), dstep(c, sizeof(int));
  upload_bytes(c, dm1.p, m->m1.data(), sizeof(float) * MLP_NP);
  upload_bytes(c, dm2.p, m->m2.data(), sizeof(float) * MLP_NP);
  const int step0 = (int)m->adamStep;
  upload_bytes(c, dstep.p, &step0, sizeof(int));
  int per = 0;
  const int nblk = grad_blocks(n, per);
  DevBuf part(c, sizeof(float) * (size_t)nblk * (MLP_NP + 1)), g(c, sizeof(float) * (MLP_NP + 1));
  const MlpNorm nrm = norm_of(m);
  auto one_step = [&](cudaStream_t s) {
    mlp_grad_kernel<<<nblk, MLP_THREADS, 0, s>>>(d.w.as<__nv_bfloat16>(), nrm, dx.as<float>(), dt.as<float>(), n,
                                                 per, part.as<float>());
    mlp_reduce_kernel<<<ceil_div(MLP_NP + 1, 256), 256, 0, s>>>(part.as<float>(), nblk, g.as<float>());
    mlp_adam_kernel<<<1, 1024, 0, s>>>(d.master.as<float>(), g.as<float>(), dm1.as<float>(), dm2.as<float>(),
                                       dstep.as<int>(), lr, d.w.as<__nv_bfloat16>());
  };
  // first step eagerly: its loss is the starting loss
  one_step(c->stream);
  AIFMM_CUDA(cudaGetLastError());
  count_launch(3);
  float first = 0.0f;
  AIFMM_CUDA(cudaMemcpyAsync(&first, g.as<float>() + MLP_NP, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  int done = 1;
  if (epochs - done >= TRAIN_EPOCHS_PER_GRAPH) {
    // the remaining steps as replays of one captured graph of TRAIN_EPOCHS_PER_GRAPH steps
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    AIFMM_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    for (int e = 0; e < TRAIN_EPOCHS_PER_GRAPH; ++e) one_step(c->stream);
    cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
    AIFMM_CUDA(ce);
    ce = cudaGraphInstantiate(&exec, graph, 0);
    if (ce != cudaSuccess) {
      cudaGraphDestroy(graph);
      AIFMM_CUDA(ce);
    }
    while (epochs - done >= TRAIN_EPOCHS_PER_GRAPH) {
      ce = cudaGraphLaunch(exec, c->stream);
      if (ce != cudaSuccess) break;
      count_launch(3 * TRAIN_EPOCHS_PER_GRAPH);
      done += TRAIN_EPOCHS_PER_GRAPH;
    }
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    AIFMM_CUDA(ce);
  }
  for (; done < epochs; ++done) {
    one_step(c->stream);
    AIFMM_CUDA(cudaGetLastError());
    count_launch(3);
  }
  float last = 0.0f;
  int stepN = 0;
  AIFMM_CUDA(cudaMemcpyAsync(&last, g.as<float>() + MLP_NP, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  AIFMM_CUDA(cudaMemcpyAsync(m->params.data(), d.master.p, sizeof(float) * MLP_NP, cudaMemcpyDeviceToHost, c->stream));
  AIFMM_CUDA(cudaMemcpyAsync(m->m1.data(), dm1.p, sizeof(float) * MLP_NP, cudaMemcpyDeviceToHost, c->stream));
  AIFMM_CUDA(cudaMemcpyAsync(m->m2.data(), dm2.p, sizeof(float) * MLP_NP, cudaMemcpyDeviceToHost, c->stream));
  AIFMM_CUDA(cudaMemcpyAsync(&stepN, dstep.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  AIFMM_CUDA(cudaStreamSynchronize(c->stream));
  m->adamStep = stepN;
  if (loss_first) *loss_first = first / (float)n;
  if (loss_last) *loss_last = last / (float)n;
  API_END
}

}  // extern "C"
