// C ABI of the H^2 forward operator and the preconditioned GMRES solve.
#include <memory>

#include "capi_guard.cuh"
#include "krylov.cuh"

using namespace aifmm;

extern "C" {

int aifmm_operator_create(aifmm_kernel* k, const aifmm_solver_params* p, aifmm_operator** out) {
  API_BEGIN
  AIFMM_REQUIRE(k && p && out, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(p->precision == 0, AIFMM_ENOTIMPL, "the forward operator is complex128");
  AIFMM_REQUIRE(p->leaf_size > 0 && p->tol_pow >= 0 && p->fillin_tol >= 0 && p->n_levels >= 0, AIFMM_EINVAL,
                "bad operator parameters");
  AIFMM_CUDA(cudaSetDevice(k->ctx->device));
  SolverParams sp;
  sp.leafSize = p->leaf_size;
  sp.tol_pow = p->tol_pow;
  sp.fillin_tol = p->fillin_tol;
  sp.fillin_rank = p->fillin_rank;
  sp.nLevelsInput = p->n_levels;
  sp.realMode = k->geom.efie ? 0 : 1;
  std::unique_ptr<Solver> s(new Solver(k, sp));
  s->build();
  std::unique_ptr<aifmm_operator> o(new aifmm_operator);
  o->op.reset(new H2Operator(std::move(s)));
  ctx_retain(k->ctx);
  *out = o.release();
  API_END
}

int aifmm_operator_apply_device(aifmm_operator* op, const void* x_device, int nrhs, void* y_device) {
  API_BEGIN
  AIFMM_REQUIRE(op && x_device && y_device && nrhs > 0, AIFMM_EINVAL, "bad argument");
  H2Operator& A = *op->op;
  A.apply(static_cast<const zd*>(x_device), A.N, static_cast<zd*>(y_device), A.N, nrhs);
  AIFMM_CUDA(cudaStreamSynchronize(A.ctx->stream));
  API_END
}

int aifmm_operator_apply(aifmm_operator* op, const double* x, int nrhs, double* y) {
  API_BEGIN
  AIFMM_REQUIRE(op && x && y && nrhs > 0, AIFMM_EINVAL, "bad argument");
  H2Operator& A = *op->op;
  AIFMM_CUDA(cudaSetDevice(A.ctx->device));
  const size_t bytes = sizeof(zd) * (size_t)A.N * nrhs;
  DevBuf xd(A.ctx, bytes), yd(A.ctx, bytes);
  AIFMM_CUDA(cudaMemcpyAsync(xd.p, x, bytes, cudaMemcpyHostToDevice, A.ctx->stream));
  A.apply(xd.as<zd>(), A.N, yd.as<zd>(), A.N, nrhs);
  AIFMM_CUDA(cudaMemcpyAsync(y, yd.p, bytes, cudaMemcpyDeviceToHost, A.ctx->stream));
  AIFMM_CUDA(cudaStreamSynchronize(A.ctx->stream));
  API_END
}

int aifmm_operator_info(aifmm_operator* op, double* bytes, double* flops_per_column) {
  API_BEGIN
  AIFMM_REQUIRE(op && bytes && flops_per_column, AIFMM_EINVAL, "NULL argument");
  *bytes = op->op->bytes;
  *flops_per_column = op->op->flopsPerColumn;
  API_END
}

int aifmm_operator_destroy(aifmm_operator* op) {
  API_BEGIN
  if (!op) return AIFMM_OK;
  aifmm_ctx* c = op->op ? op->op->ctx : nullptr;
  if (c) AIFMM_CUDA(cudaSetDevice(c->device));
  delete op;
  if (c) ctx_release(c);
  API_END
}

void fill_gmres_info(const GmresResult& r, aifmm_gmres_info* info) {
  if (!info) return;
  info->iterations = r.iterations;
  info->cycles = r.cycles;
  info->relres = r.relres;
  info->t_precond = r.t_precond;
  info->t_matvec = r.t_matvec;
}

int aifmm_solver_solve_gmres_device(aifmm_solver* s, aifmm_operator* A, const void* rhs_device, int nrhs,
                                    void* x_device, double tol, int restart, int maxit, aifmm_gmres_info* info) {
  API_BEGIN
  AIFMM_REQUIRE(s && A && rhs_device && x_device && nrhs > 0, AIFMM_EINVAL, "bad argument");
  Solver& S = *s->s;
  AIFMM_REQUIRE(S.factored, AIFMM_ESTATE, "solve before factorize");
  AIFMM_CUDA(cudaSetDevice(S.ctx->device));
  const GmresResult r = fgmres(S, *A->op, static_cast<const zd*>(rhs_device), static_cast<zd*>(x_device), nrhs, tol,
                               restart, maxit);
  AIFMM_CUDA(cudaStreamSynchronize(S.ctx->stream));
  fill_gmres_info(r, info);
  API_END
}

int aifmm_solver_solve_gmres(aifmm_solver* s, aifmm_operator* A, const double* rhs, int nrhs, double* x, double tol,
                             int restart, int maxit, aifmm_gmres_info* info) {
  API_BEGIN
  AIFMM_REQUIRE(s && A && rhs && x && nrhs > 0, AIFMM_EINVAL, "bad argument");
  Solver& S = *s->s;
  AIFMM_REQUIRE(S.factored, AIFMM_ESTATE, "solve before factorize");
  AIFMM_CUDA(cudaSetDevice(S.ctx->device));
  const size_t bytes = sizeof(zd) * (size_t)S.N * nrhs;
  DevBuf bd(S.ctx, bytes), xd(S.ctx, bytes);
  AIFMM_CUDA(cudaMemcpyAsync(bd.p, rhs, bytes, cudaMemcpyHostToDevice, S.ctx->stream));
  const GmresResult r = fgmres(S, *A->op, bd.as<zd>(), xd.as<zd>(), nrhs, tol, restart, maxit);
  AIFMM_CUDA(cudaMemcpyAsync(x, xd.p, bytes, cudaMemcpyDeviceToHost, S.ctx->stream));
  AIFMM_CUDA(cudaStreamSynchronize(S.ctx->stream));
  fill_gmres_info(r, info);
  API_END
}

}  // extern "C"
