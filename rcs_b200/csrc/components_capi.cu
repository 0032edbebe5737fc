// C ABI of the low-rank / dense components and the solver state dump.
#include <array>
#include <cstring>

#include "capi_guard.cuh"
#include "solver.cuh"

using namespace aifmm;


extern "C" {

int aifmm_aca(aifmm_kernel* k, const int* rows, int nr, const int* cols, int nc, double tol, int* row_bases,
              int* col_bases, int* rank, double* Ac, double* Ar) {
  API_BEGIN
  AIFMM_REQUIRE(k && rows && cols && row_bases && col_bases && rank && Ac && Ar, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(nr > 0 && nc > 0, AIFMM_EINVAL, "empty block");
  for (int i = 0; i < nr; ++i) AIFMM_REQUIRE(rows[i] >= 0 && rows[i] < k->geom.N, AIFMM_EINVAL, "row id out of range");
  for (int i = 0; i < nc; ++i) AIFMM_REQUIRE(cols[i] >= 0 && cols[i] < k->geom.N, AIFMM_EINVAL, "col id out of range");
  aifmm_ctx* c = k->ctx;
  AIFMM_CUDA(cudaSetDevice(c->device));
  const int mn = std::min(nr, nc);
  int rmax = std::min(mn, 128);
  for (;;) {
    const int nP = nr < nc ? nr : nc, nS = nr < nc ? nc : nr;
    const size_t zU = (size_t)rmax * nP, zV = (size_t)rmax * nS, zAc = (size_t)nr * rmax, zAr = (size_t)rmax * nc;
    DevBuf ws(c, sizeof(zd) * (zU + zV + zAc + zAr) + (nr + nc) + sizeof(int) * 2 * rmax + 64);
    DevBuf ids(c, sizeof(int) * (nr + nc)), out(c, sizeof(int) * 2);
    AIFMM_CUDA(cudaMemcpyAsync(ids.p, rows, sizeof(int) * nr, cudaMemcpyHostToDevice, c->stream));
    AIFMM_CUDA(cudaMemcpyAsync(ids.as<int>() + nr, cols, sizeof(int) * nc, cudaMemcpyHostToDevice, c->stream));
    ACAProblem P;
    P.rows = ids.as<int>();
    P.cols = ids.as<int>() + nr;
    P.nr = nr;
    P.nc = nc;
    P.rmax = rmax;
    P.U = ws.as<zd>();
    P.V = P.U + zU;
    P.Ac = P.V + zV;
    P.Ar = P.Ac + zAc;
    P.rowBases = (int*)(P.Ar + zAr);
    P.colBases = P.rowBases + rmax;
    P.used = (unsigned char*)(P.colBases + rmax);
    P.rank = out.as<int>();
    P.status = out.as<int>() + 1;
    launch_aca(c, k->geom, {P}, tol);
    int h[2];
    AIFMM_CUDA(cudaMemcpyAsync(h, out.p, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    AIFMM_CUDA(cudaStreamSynchronize(c->stream));
    if (h[1] != 0) {
      AIFMM_REQUIRE(rmax < mn && rmax < 1024, AIFMM_EOVERFLOW, "ACA rank exceeds the workspace bound");
      rmax = std::min(mn, std::min(2 * rmax, 1024));
      continue;
    }
    const int r = h[0];
    *rank = r;
    if (r > 0) {
      AIFMM_CUDA(cudaMemcpyAsync(row_bases, P.rowBases, sizeof(int) * r, cudaMemcpyDeviceToHost, c->stream));
      AIFMM_CUDA(cudaMemcpyAsync(col_bases, P.colBases, sizeof(int) * r, cudaMemcpyDeviceToHost, c->stream));
      AIFMM_CUDA(cudaMemcpyAsync(Ac, P.Ac, sizeof(zd) * (size_t)nr * r, cudaMemcpyDeviceToHost, c->stream));
      // Ar in the workspace has leading dimension rmax; return it with ld = rank
      AIFMM_CUDA(cudaMemcpy2DAsync(Ar, sizeof(zd) * r, P.Ar, sizeof(zd) * rmax, sizeof(zd) * r, nc,
                                   cudaMemcpyDeviceToHost, c->stream));
    }
    AIFMM_CUDA(cudaStreamSynchronize(c->stream));
    break;
  }
  API_END
}

static void zgemm_checked(aifmm_ctx* ctx, int precision, int opA, int opB, int m, int n, int k, const double* alpha,
                          const zd* A, int lda, const zd* B, int ldb, const double* beta, zd* C, int ldc);

// Host-array RRQR shared by aifmm_rrqr and aifmm_rrqr_full; R and perm may be
// NULL.  R_trunc is formed as Q_trunc^H (A P), which equals the reference's
// rows 0..rank-1 of the transformed matrix; the entries below the diagonal of
// its leading rank x rank block are exact zeros there and are set so here.
static void rrqr_host(aifmm_ctx* ctx, const double* A, int m, int n, int partition, int tol_pow1, int tol_pow2,
                      double input_pivot, int fill_rank, int real_mode, double* Q, double* Rt, int* perm_out,
                      int* rank, double* max_pivot) {
  AIFMM_REQUIRE(ctx && A && Q && rank && max_pivot, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(m > 0 && n > 0 && partition >= 0 && partition <= n, AIFMM_EINVAL, "bad sizes");
  AIFMM_REQUIRE(tol_pow1 >= 0 && tol_pow2 >= 0 && fill_rank >= 0, AIFMM_EINVAL, "negative tolerance power or fill-in rank");
  AIFMM_CUDA(cudaSetDevice(ctx->device));
  const int hs = std::min(m, n) + 1;
  DevBuf R(ctx, sizeof(zd) * (size_t)m * n), H(ctx, sizeof(zd) * (size_t)m * hs), Qd(ctx, sizeof(zd) * (size_t)m * hs);
  DevBuf nsq(ctx, sizeof(double) * n), perm(ctx, sizeof(int) * n), out(ctx, 64);
  AIFMM_CUDA(cudaMemcpyAsync(R.p, A, sizeof(zd) * (size_t)m * n, cudaMemcpyHostToDevice, ctx->stream));
  RRQRProblem P;
  P.R = R.as<zd>();
  P.m = m;
  P.n = n;
  P.partition = partition;
  P.tol1 = std::pow(10.0, -tol_pow1);
  P.tol2 = std::pow(10.0, -tol_pow2);
  P.inputPivot = input_pivot;
  P.fillInRank = fill_rank;
  P.realMode = real_mode;
  P.H = H.as<zd>();
  P.nsq = nsq.as<double>();
  P.perm = perm.as<int>();
  P.Q = Qd.as<zd>();
  P.rank = out.as<int>();
  P.maxPivot = (double*)((char*)out.p + 8);
  P.istate = (int*)((char*)out.p + 16);
  P.dstate = (double*)((char*)out.p + 48);  // after the 8 ints of istate
  P.p2cap = -1;
  launch_rrqr_split(ctx, {P});
  struct {
    int r, pad;
    double mp;
  } h;
  AIFMM_CUDA(cudaMemcpyAsync(&h, out.p, 16, cudaMemcpyDeviceToHost, ctx->stream));
  AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
  AIFMM_REQUIRE(h.r != -2, AIFMM_ETIMEOUT, "RRQR: a bounded grid-barrier wait ran out");
  *rank = h.r;
  *max_pivot = h.mp;
  if (h.r > 0)
    AIFMM_CUDA(cudaMemcpyAsync(Q, Qd.p, sizeof(zd) * (size_t)m * h.r, cudaMemcpyDeviceToHost, ctx->stream));
  if (perm_out || Rt) {
    std::vector<int> hp(n);
    AIFMM_CUDA(cudaMemcpyAsync(hp.data(), perm.p, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->stream));
    AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
    if (perm_out) std::memcpy(perm_out, hp.data(), sizeof(int) * n);
    if (Rt && h.r > 0) {
      const zd* Ah = reinterpret_cast<const zd*>(A);
      std::vector<zd> ap((size_t)m * n);
      for (int q = 0; q < n; ++q) std::memcpy(&ap[(size_t)q * m], Ah + (size_t)hp[q] * m, sizeof(zd) * m);
      DevBuf APd = upload(ctx, ap), Rd(ctx, sizeof(zd) * (size_t)h.r * n);
      const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
      zgemm_checked(ctx, 0, 1, 0, h.r, n, m, one, Qd.as<zd>(), m, APd.as<zd>(), m, zero, Rd.as<zd>(), h.r);
      AIFMM_CUDA(cudaMemcpyAsync(Rt, Rd.p, sizeof(zd) * (size_t)h.r * n, cudaMemcpyDeviceToHost, ctx->stream));
      AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
      for (int q = 0; q < std::min(h.r, n); ++q)
        for (int i = q + 1; i < h.r; ++i) Rt[2 * ((size_t)q * h.r + i)] = Rt[2 * ((size_t)q * h.r + i) + 1] = 0.0;
    }
  }
  AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
}

int aifmm_rrqr(aifmm_ctx* ctx, const double* A, int m, int n, int partition, int tol_pow1, int tol_pow2,
               double input_pivot, int fill_rank, int real_mode, double* Q, int* rank, double* max_pivot) {
  API_BEGIN
  rrqr_host(ctx, A, m, n, partition, tol_pow1, tol_pow2, input_pivot, fill_rank, real_mode, Q, nullptr, nullptr,
            rank, max_pivot);
  API_END
}

int aifmm_rrqr_full(aifmm_ctx* ctx, const double* A, int m, int n, int partition, int tol_pow1, int tol_pow2,
                    double input_pivot, int fill_rank, int real_mode, double* Q, double* R, int* perm, int* rank,
                    double* max_pivot) {
  API_BEGIN
  AIFMM_REQUIRE(R && perm, AIFMM_EINVAL, "NULL argument");
  rrqr_host(ctx, A, m, n, partition, tol_pow1, tol_pow2, input_pivot, fill_rank, real_mode, Q, R, perm, rank,
            max_pivot);
  API_END
}

static void zgemm_checked(aifmm_ctx* ctx, int precision, int opA, int opB, int m, int n, int k, const double* alpha,
                          const zd* A, int lda, const zd* B, int ldb, const double* beta, zd* C, int ldc) {
  GemmProblem g{A, B, C, m, n, k, lda, ldb, ldc, opA, opB, zmk(alpha[0], alpha[1]), zmk(beta[0], beta[1])};
  const int saved = ctx->gemmPrecision;
  ctx->gemmPrecision = precision;
  const long t0 = precision >= 2 ? tc_timeouts() : 0;
  try {
    zgemm_grouped(ctx, {g});
  } catch (...) {
    ctx->gemmPrecision = saved;
    throw;
  }
  ctx->gemmPrecision = saved;
  if (precision >= 2) {  // a tile that gave up on a bounded wait left C unwritten
    AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
    tc_check(t0, "zgemm");
  }
}

static void zgemm_args(aifmm_ctx* ctx, int precision, int opA, int opB, int m, int n, int k, const double* alpha,
                       const void* A, int lda, const void* B, int ldb, const double* beta, const void* C, int ldc) {
  AIFMM_REQUIRE(ctx && alpha && beta && C && m >= 0 && n >= 0 && k >= 0, AIFMM_EINVAL, "bad argument");
  AIFMM_REQUIRE(precision >= 0 && precision <= 5, AIFMM_EINVAL, "precision must be 0 to 5");
  AIFMM_REQUIRE((opA == 0 || opA == 1) && (opB == 0 || opB == 1), AIFMM_EINVAL, "op must be 0 or 1");
  const int ar = opA ? k : m, br = opB ? n : k;
  AIFMM_REQUIRE(lda >= std::max(ar, 1) && ldb >= std::max(br, 1) && ldc >= std::max(m, 1), AIFMM_EINVAL,
                "leading dimension too small");
  AIFMM_REQUIRE(k == 0 || (A && B), AIFMM_EINVAL, "NULL operand");
}

int aifmm_zgemm(aifmm_ctx* ctx, int precision, int opA, int opB, int m, int n, int k, const double alpha[2],
                const double* A, int lda, const double* B, int ldb, const double beta[2], double* C, int ldc) {
  API_BEGIN
  zgemm_args(ctx, precision, opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  AIFMM_CUDA(cudaSetDevice(ctx->device));
  const int ac = opA ? m : k, bc = opB ? k : n;
  const size_t za = (size_t)lda * ac, zb = (size_t)ldb * bc, zc = (size_t)ldc * n;
  DevBuf dA(ctx, sizeof(zd) * za + 16), dB(ctx, sizeof(zd) * zb + 16), dC(ctx, sizeof(zd) * zc + 16);
  if (za) AIFMM_CUDA(cudaMemcpyAsync(dA.p, A, sizeof(zd) * za, cudaMemcpyHostToDevice, ctx->stream));
  if (zb) AIFMM_CUDA(cudaMemcpyAsync(dB.p, B, sizeof(zd) * zb, cudaMemcpyHostToDevice, ctx->stream));
  if (zc) AIFMM_CUDA(cudaMemcpyAsync(dC.p, C, sizeof(zd) * zc, cudaMemcpyHostToDevice, ctx->stream));
  zgemm_checked(ctx, precision, opA, opB, m, n, k, alpha, dA.as<zd>(), lda, dB.as<zd>(), ldb, beta, dC.as<zd>(), ldc);
  if (zc) AIFMM_CUDA(cudaMemcpyAsync(C, dC.p, sizeof(zd) * zc, cudaMemcpyDeviceToHost, ctx->stream));
  AIFMM_CUDA(cudaStreamSynchronize(ctx->stream));
  API_END
}

int aifmm_zgemm_device(aifmm_ctx* ctx, int precision, int opA, int opB, int m, int n, int k, const double alpha[2],
                       const void* A_device, int lda, const void* B_device, int ldb, const double beta[2],
                       void* C_device, int ldc) {
  API_BEGIN
  zgemm_args(ctx, precision, opA, opB, m, n, k, alpha, A_device, lda, B_device, ldb, beta, C_device, ldc);
  AIFMM_CUDA(cudaSetDevice(ctx->device));
  zgemm_checked(ctx, precision, opA, opB, m, n, k, alpha, static_cast<const zd*>(A_device), lda,
                static_cast<const zd*>(B_device), ldb, beta, static_cast<zd*>(C_device), ldc);
  API_END
}

int aifmm_lu_solve(aifmm_ctx* ctx, const double* A, int n, const double* B, int nrhs, double* X) {
  API_BEGIN
  AIFMM_REQUIRE(ctx && A && B && X && n > 0 && nrhs > 0, AIFMM_EINVAL, "bad argument");
  AIFMM_CUDA(cudaSetDevice(ctx->device));
  Ops ops(ctx);
  std::vector<zd> ha((size_t)n * n), hb((size_t)n * nrhs);
  std::memcpy(ha.data(), A, sizeof(zd) * ha.size());
  std::memcpy(hb.data(), B, sizeof(zd) * hb.size());
  DLU f = ops.factor(ops.fromHost(ha, n, n));
  DMat x = ops.solve(f, ops.fromHost(hb, n, nrhs));
  std::vector<zd> hx = ops.download(x);
  std::memcpy(X, hx.data(), sizeof(zd) * hx.size());
  API_END
}

int aifmm_solver_dump(aifmm_solver* s, double* out, long cap, long* count) {
  API_BEGIN
  AIFMM_REQUIRE(s && count, AIFMM_EINVAL, "NULL argument");
  Solver& S = *s->s;
  std::vector<std::array<double, 6>> meta;
  std::vector<const DMat*> mats;
  for (int j = 0; j <= S.nLevels; ++j)
    for (int k = 0; k < (int)S.tree[j].size(); ++k) {
      DBox& B = S.tree[j][k];
      auto add = [&](int kind, int key, const DMat& m) {
        meta.push_back({(double)j, (double)k, (double)kind, (double)key, (double)m.r, (double)m.c});
        mats.push_back(&m);
      };
      add(0, -1, B.L2P);
      add(1, -1, B.P2M);
      int kind = 2;
      for (auto* mp : {&B.M2L, &B.P2P, &B.M2P, &B.P2L, &B.L2P_f, &B.P2M_f, &B.M2M_f}) {
        for (auto& kv : *mp) add(kind, kv.first, kv.second);
        kind++;
      }
      add(9, -1, B.L2M_f);
    }
  Ops ops(S.ctx);
  std::vector<double> nv = ops.norms(mats);
  *count = (long)meta.size();
  if (out)
    for (long i = 0; i < std::min(cap, (long)meta.size()); ++i) {
      for (int q = 0; q < 6; ++q) out[7 * i + q] = meta[i][q];
      out[7 * i + 6] = nv[i];
    }
  API_END
}

}  // extern "C"
