// Flexible GMRES(m): device kernels for the block inner products and
// updates, host Arnoldi/Givens bookkeeping.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>

#include "krylov.cuh"

namespace aifmm {

static double wall() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

constexpr int DOT_CHUNK = 4096;

// part[(r * nv + i) * nchunk + c] = sum over rows n of chunk c of conj(V_i[n, r]) w[n, r]
// V_i = V + i * vstride, every block N x nr with ld N.
__global__ void __launch_bounds__(256) zdotc_blocks_kernel(const zd* __restrict__ V, size_t vstride, int nv,
                                                           const zd* __restrict__ w, int N, int nchunk, zd* part) {
  const int c = blockIdx.x, r = blockIdx.y;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lo = c * DOT_CHUNK, hi = min(N, lo + DOT_CHUNK);
  const zd* wr = w + (size_t)r * N;
  for (int i = warp; i < nv; i += 8) {
    const zd* v = V + (size_t)i * vstride + (size_t)r * N;
    zd s = zmk(0, 0);
    for (int n = lo + lane; n < hi; n += 32) s = zadd(s, zcmul(v[n], wr[n]));
    for (int o = 16; o > 0; o >>= 1) {
      s.x += __shfl_xor_sync(0xffffffff, s.x, o);
      s.y += __shfl_xor_sync(0xffffffff, s.y, o);
    }
    if (lane == 0) part[((size_t)r * nv + i) * nchunk + c] = s;
  }
}

__global__ void zdotc_finish_kernel(const zd* __restrict__ part, int nchunk, int total, zd* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  zd s = zmk(0, 0);
  for (int c = 0; c < nchunk; ++c) s = zadd(s, part[(size_t)t * nchunk + c]);
  out[t] = s;
}

// out[n, r] = beta * out[n, r] + alpha * sum_{i < nv} V_i[n, r] coef[r * nv + i]
__global__ void zcombine_kernel(const zd* __restrict__ V, size_t vstride, int nv, const zd* __restrict__ coef, int N,
                                int nr, double alpha, double beta, zd* out) {
  const long total = (long)N * nr;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const int r = (int)(t / N);
    zd s = zmk(0, 0);
    for (int i = 0; i < nv; ++i) s = zadd(s, zmul(V[(size_t)i * vstride + t], coef[(size_t)r * nv + i]));
    const zd o = (beta == 0.0) ? zmk(0, 0) : zscale(out[t], beta);
    out[t] = zadd(o, zscale(s, alpha));
  }
}

// dst[n, r] = src[n, r] * s[r]
__global__ void zscale_cols_kernel(const zd* __restrict__ src, const double* __restrict__ s, int N, int nr, zd* dst) {
  const long total = (long)N * nr;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x)
    dst[t] = zscale(src[t], s[t / N]);
}

// d = a - b
__global__ void zsub_kernel(const zd* __restrict__ a, const zd* __restrict__ b, long n, zd* d) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
    d[t] = zsub(a[t], b[t]);
}

static int grid_for(long n) { return (int)std::min<long>((n + 255) / 256, 148L * 16); }

namespace {
struct Krylov {
  aifmm_ctx* ctx;
  int N, nr;
  DevBuf part, out;
  int nchunk;
  std::vector<zd> host;
  Krylov(aifmm_ctx* c, int n, int r, int maxv) : ctx(c), N(n), nr(r) {
    nchunk = (N + DOT_CHUNK - 1) / DOT_CHUNK;
    part = DevBuf(ctx, sizeof(zd) * (size_t)nchunk * nr * maxv + 16);
    out = DevBuf(ctx, sizeof(zd) * (size_t)nr * maxv + 16);
  }
  // host[r * nv + i] = V_i[:, r]^H w[:, r]
  const std::vector<zd>& dots(const zd* V, size_t vstride, int nv, const zd* w) {
    zdotc_blocks_kernel<<<dim3(nchunk, nr), 256, 0, ctx->stream>>>(V, vstride, nv, w, N, nchunk, part.as<zd>());
    AIFMM_LAUNCHED();
    const int total = nr * nv;
    zdotc_finish_kernel<<<(total + 127) / 128, 128, 0, ctx->stream>>>(part.as<zd>(), nchunk, total, out.as<zd>());
    AIFMM_LAUNCHED();
    host.resize(total);
    AIFMM_CUDA(cudaMemcpyAsync(host.data(), out.p, sizeof(zd) * total, cudaMemcpyDeviceToHost, ctx->stream));
    AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
    return host;
  }
  std::vector<double> norms(const zd* w) {
    const std::vector<zd>& d = dots(w, 0, 1, w);
    std::vector<double> n(nr);
    for (int r = 0; r < nr; ++r) n[r] = std::sqrt(std::max(d[r].x, 0.0));
    return n;
  }
  void combine(const zd* V, size_t vstride, int nv, const std::vector<zd>& coef, double alpha, double beta, zd* o) {
    DevBuf dc = upload(ctx, coef);
    zcombine_kernel<<<grid_for((long)N * nr), 256, 0, ctx->stream>>>(V, vstride, nv, dc.as<zd>(), N, nr, alpha, beta, o);
    AIFMM_LAUNCHED();
  }
  void scale(const zd* src, const std::vector<double>& s, zd* dst) {
    DevBuf ds = upload(ctx, s);
    zscale_cols_kernel<<<grid_for((long)N * nr), 256, 0, ctx->stream>>>(src, ds.as<double>(), N, nr, dst);
    AIFMM_LAUNCHED();
  }
};
}  // namespace

GmresResult fgmres(Solver& M, H2Operator& A, const zd* b, zd* x, int nr, double tol, int restart, int maxit) {
  AIFMM_REQUIRE(M.ctx == A.ctx, AIFMM_EINVAL, "preconditioner and operator live on different contexts");
  AIFMM_REQUIRE(M.N == A.N, AIFMM_EINVAL, "preconditioner and operator sizes differ");
  AIFMM_REQUIRE(nr >= 1 && tol > 0 && restart >= 1 && restart <= 200 && maxit >= 1, AIFMM_EINVAL,
                "bad GMRES parameters");
  aifmm_ctx* ctx = A.ctx;
  const int N = A.N;
  const size_t blk = (size_t)N * nr;
  GmresResult res;
  Krylov kr(ctx, N, nr, restart + 1);
  DevBuf Vb(ctx, sizeof(zd) * blk * (restart + 1)), Zb(ctx, sizeof(zd) * blk * restart);
  DevBuf wb(ctx, sizeof(zd) * blk), rb(ctx, sizeof(zd) * blk);
  zd* V = Vb.as<zd>();
  zd* Z = Zb.as<zd>();
  zd* w = wb.as<zd>();
  zd* r = rb.as<zd>();
  const std::vector<double> bn = kr.norms(b);
  zfill(ctx, x, blk, zmk(0, 0));
  AIFMM_CUDA(cudaMemcpyAsync(r, b, sizeof(zd) * blk, cudaMemcpyDeviceToDevice, ctx->stream));
  typedef std::complex<double> C;
  const int m = restart;
  while (true) {
    const std::vector<double> beta = kr.norms(r);
    double rel = 0;
    for (int q = 0; q < nr; ++q) rel = std::max(rel, bn[q] > 0 ? beta[q] / bn[q] : 0.0);
    res.relres = rel;
    if (rel <= tol || res.iterations >= maxit) break;
    res.cycles++;
    std::vector<double> inv(nr);
    for (int q = 0; q < nr; ++q) inv[q] = beta[q] > 0 ? 1.0 / beta[q] : 0.0;
    kr.scale(r, inv, V);
    // per column: Hessenberg (column-major (m+1) x m), rotations, rhs g
    std::vector<std::vector<C>> H(nr, std::vector<C>((size_t)(m + 1) * m, C(0, 0)));
    std::vector<std::vector<C>> cs(nr, std::vector<C>(m)), sn(nr, std::vector<C>(m));
    std::vector<std::vector<C>> g(nr, std::vector<C>(m + 1, C(0, 0)));
    for (int q = 0; q < nr; ++q) g[q][0] = C(beta[q], 0);
    int k = 0;
    for (int j = 0; j < m; ++j) {
      // z_j = M^{-1} v_j ; w = A z_j
      const double t0 = wall();
      {
        DMat vj;
        vj.p = V + blk * j;
        vj.r = N;
        vj.c = nr;
        DMat zj = M.solve(vj);
        AIFMM_CUDA(cudaMemcpyAsync(Z + blk * j, zj.p, sizeof(zd) * blk, cudaMemcpyDeviceToDevice, ctx->stream));
      }
      AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
      const double t1 = wall();
      A.apply(Z + blk * j, N, w, N, nr);
      AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
      res.t_precond += t1 - t0;
      res.t_matvec += wall() - t1;
      // classical Gram-Schmidt, twice
      std::vector<zd> hsum((size_t)nr * (j + 1), zmk(0, 0));
      for (int pass = 0; pass < 2; ++pass) {
        const std::vector<zd> h = kr.dots(V, blk, j + 1, w);
        kr.combine(V, blk, j + 1, h, -1.0, 1.0, w);
        for (size_t t = 0; t < h.size(); ++t) hsum[t] = zadd(hsum[t], h[t]);
      }
      const std::vector<double> hn = kr.norms(w);
      std::vector<double> ihn(nr);
      for (int q = 0; q < nr; ++q) ihn[q] = hn[q] > 0 ? 1.0 / hn[q] : 0.0;
      kr.scale(w, ihn, V + blk * (j + 1));
      double worst = 0;
      for (int q = 0; q < nr; ++q) {
        C* hc = &H[q][(size_t)j * (m + 1)];
        for (int i = 0; i <= j; ++i) hc[i] = C(hsum[(size_t)q * (j + 1) + i].x, hsum[(size_t)q * (j + 1) + i].y);
        hc[j + 1] = C(hn[q], 0);
        for (int i = 0; i < j; ++i) {  // earlier rotations
          const C a = hc[i], bb = hc[i + 1];
          hc[i] = std::conj(cs[q][i]) * a + std::conj(sn[q][i]) * bb;
          hc[i + 1] = -sn[q][i] * a + cs[q][i] * bb;
        }
        const double den = std::sqrt(std::norm(hc[j]) + std::norm(hc[j + 1]));
        if (den > 0) {
          cs[q][j] = hc[j] / den;
          sn[q][j] = hc[j + 1] / den;
        } else {
          cs[q][j] = C(1, 0);
          sn[q][j] = C(0, 0);
        }
        hc[j] = std::conj(cs[q][j]) * hc[j] + std::conj(sn[q][j]) * hc[j + 1];
        hc[j + 1] = C(0, 0);
        const C gj = g[q][j];
        g[q][j] = std::conj(cs[q][j]) * gj;
        g[q][j + 1] = -sn[q][j] * gj;
        if (bn[q] > 0) worst = std::max(worst, std::abs(g[q][j + 1]) / bn[q]);
      }
      k = j + 1;
      res.iterations++;
      if (worst <= tol || res.iterations >= maxit) break;
    }
    // y = R^{-1} g per column, x += Z y
    std::vector<zd> coef((size_t)nr * k);
    for (int q = 0; q < nr; ++q) {
      std::vector<C> y(k);
      for (int i = k - 1; i >= 0; --i) {
        C s = g[q][i];
        for (int l = i + 1; l < k; ++l) s -= H[q][(size_t)l * (m + 1) + i] * y[l];
        const C d = H[q][(size_t)i * (m + 1) + i];
        y[i] = (std::abs(d) > 0) ? s / d : C(0, 0);
      }
      for (int i = 0; i < k; ++i) coef[(size_t)q * k + i] = zmk(y[i].real(), y[i].imag());
    }
    kr.combine(Z, blk, k, coef, 1.0, 1.0, x);
    // explicit residual r = b - A x
    const double t1 = wall();
    A.apply(x, N, w, N, nr);
    zsub_kernel<<<grid_for((long)blk), 256, 0, ctx->stream>>>(b, w, (long)blk, r);
    AIFMM_LAUNCHED();
    AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
    res.t_matvec += wall() - t1;
  }
  return res;
}

}  // namespace aifmm
