// C ABI of the AIFMM solver (see include/aifmm_b200.h).
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>

#include "capi_guard.cuh"
#include "solver.cuh"

using namespace aifmm;


extern "C" {

static void solver_create(aifmm_kernel* k, const aifmm_solver_params* p, const double* xyz, const double* dom,
                          aifmm_solver** out) {
  AIFMM_REQUIRE(k && p && out, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(p->precision >= 0 && p->precision <= 5, AIFMM_EINVAL,
                "precision must be 0 (plain) or 1 to 5 (mixed)");
  AIFMM_REQUIRE(p->leaf_size > 0 && p->tol_pow >= 0 && p->fillin_tol >= 0 && p->n_levels >= 0, AIFMM_EINVAL,
                "bad solver parameters");
  SolverParams sp;
  sp.leafSize = p->leaf_size;
  sp.tol_pow = p->tol_pow;
  sp.fillin_tol = p->fillin_tol;
  sp.fillin_rank = p->fillin_rank;
  sp.nLevelsInput = p->n_levels;
  sp.orthoShortcut = p->exact_rrqr == 0;
  sp.precision = p->precision;
  sp.drop_pow = p->drop_pow;
  sp.realMode = k->geom.efie ? 0 : 1;
  const char* pt = std::getenv("AIFMM_PHASE_TIMES");
  sp.phaseTiming = pt && pt[0] == '1';
  std::unique_ptr<aifmm_solver> s(new aifmm_solver);
  s->s.reset(new Solver(k, sp, xyz, dom));
  s->s->build();
  ctx_retain(k->ctx);
  *out = s.release();
}

int aifmm_solver_create(aifmm_kernel* k, const aifmm_solver_params* p, aifmm_solver** out) {
  API_BEGIN
  solver_create(k, p, nullptr, nullptr, out);
  API_END
}

int aifmm_solver_create_at(aifmm_kernel* k, const aifmm_solver_params* p, const double* xyz, int n,
                           const double domain[6], aifmm_solver** out) {
  API_BEGIN
  AIFMM_REQUIRE(k && xyz, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(n == k->geom.N, AIFMM_EINVAL, "one location per unknown is required");
  for (long i = 0; i < 3L * n; ++i) AIFMM_REQUIRE(std::isfinite(xyz[i]), AIFMM_EINVAL, "non-finite location");
  if (domain)
    for (int q = 0; q < 3; ++q)
      AIFMM_REQUIRE(std::isfinite(domain[2 * q]) && std::isfinite(domain[2 * q + 1]) &&
                        domain[2 * q] <= domain[2 * q + 1],
                    AIFMM_EINVAL, "bad domain box");
  solver_create(k, p, xyz, domain, out);
  API_END
}

int aifmm_solver_tree_order(aifmm_solver* s, int* order) {
  API_BEGIN
  AIFMM_REQUIRE(s && order, AIFMM_EINVAL, "NULL argument");
  Solver& S = *s->s;
  int pos = 0;
  for (const DBox& B : S.tree[S.nLevels])
    for (int id : B.chargeLocations) {
      AIFMM_REQUIRE(pos < S.N, AIFMM_EINVAL, "leaves hold more unknowns than the kernel");
      order[pos++] = id;
    }
  AIFMM_REQUIRE(pos == S.N, AIFMM_EINVAL, "leaves do not cover every unknown");
  API_END
}

int aifmm_solver_factorize(aifmm_solver* s) {
  API_BEGIN
  AIFMM_REQUIRE(s, AIFMM_EINVAL, "NULL argument");
  AIFMM_REQUIRE(!s->s->factored, AIFMM_ESTATE, "already factorized");
  s->s->factorize();
  API_END
}

int aifmm_solver_solve_device(aifmm_solver* s, const void* rhs_device, int nrhs, void* x_device) {
  API_BEGIN
  AIFMM_REQUIRE(s && rhs_device && x_device && nrhs > 0, AIFMM_EINVAL, "bad argument");
  Solver& S = *s->s;
  AIFMM_CUDA(cudaSetDevice(S.ctx->device));
  DMat b;
  b.p = (zd*)rhs_device;  // non-owning view
  b.r = S.N;
  b.c = nrhs;
  DMat x = S.solve(b);
  AIFMM_CUDA(cudaMemcpyAsync(x_device, x.p, sizeof(zd) * (size_t)S.N * nrhs, cudaMemcpyDeviceToDevice, S.ctx->stream));
  AIFMM_CUDA(cudaStreamSynchronize(S.ctx->stream));
  API_END
}

int aifmm_solver_solve(aifmm_solver* s, const double* rhs, int nrhs, double* x) {
  API_BEGIN
  AIFMM_REQUIRE(s && rhs && x && nrhs > 0, AIFMM_EINVAL, "bad argument");
  Solver& S = *s->s;
  AIFMM_CUDA(cudaSetDevice(S.ctx->device));
  const size_t bytes = sizeof(zd) * (size_t)S.N * nrhs;
  DMat b = S.ops.alloc(S.N, nrhs);
  AIFMM_CUDA(cudaMemcpyAsync(b.p, rhs, bytes, cudaMemcpyHostToDevice, S.ctx->stream));
  DMat xd = S.solve(b);
  AIFMM_CUDA(cudaMemcpyAsync(x, xd.p, bytes, cudaMemcpyDeviceToHost, S.ctx->stream));
  AIFMM_CUDA(cudaStreamSynchronize(S.ctx->stream));
  API_END
}

int aifmm_solver_set_graph_solve(aifmm_solver* s, int on) {
  API_BEGIN
  AIFMM_REQUIRE(s && (on == 0 || on == 1), AIFMM_EINVAL, "bad argument");
  s->s->graphSolve = on == 1;
  if (!on) s->s->dropPlan();
  API_END
}

int aifmm_solver_get_info(aifmm_solver* s, aifmm_solver_info* info) {
  API_BEGIN
  AIFMM_REQUIRE(s && info, AIFMM_EINVAL, "NULL argument");
  Solver& S = *s->s;
  info->n = S.N;
  info->n_levels = S.nLevels;
  info->start_level = S.startLevel;
  info->avg_leaf_size = S.avgLeafSize();
  info->avg_multipoles = S.avgMultipoles();
  info->max_rank = S.maxRank();
  info->n_rrqr = S.stats.nRRQR;
  info->n_compress_p2p = S.stats.nCompressP2P;
  info->n_compress_p2l = S.stats.nCompressP2L;
  info->n_aca = S.stats.nACA;
  info->n_aca_retry = S.stats.nACARetry;
  info->kernels = S.stats.kernels;
  info->n_solve_graph = S.stats.nSolveGraph;
  info->n_solve_capture = S.stats.nSolveCapture;
  info->t_assemble = S.stats.t_assemble;
  info->t_factor = S.stats.t_factor;
  info->t_solve = S.stats.t_solve;
  info->flops_factor = S.stats.flops_factor;
  info->mem_gb = S.memoryGB(false);
  info->mem_after_gb = S.memoryGB(true);
  info->t_rrqr = S.stats.t_rrqr;
  info->t_compress = S.stats.t_compress;
  info->t_elim_x = S.stats.t_elim_x;
  info->t_elim_z = S.stats.t_elim_z;
  info->t_nonleaf = S.stats.t_nonleaf;
  info->t_lu = S.stats.t_lu;
  info->t_msolve = S.stats.t_msolve;
  info->t_schur = S.stats.t_schur;
  info->t_aca = S.stats.t_aca;
  info->aca_ws_bytes = S.stats.aca_ws_bytes;
  info->n_aca_launches = S.stats.nACALaunches;
  API_END
}

int aifmm_solver_checkpoint(aifmm_solver* s) {
  API_BEGIN
  AIFMM_REQUIRE(s, AIFMM_EINVAL, "NULL argument");
  AIFMM_CUDA(cudaSetDevice(s->s->ctx->device));
  s->s->checkpoint();
  API_END
}

int aifmm_solver_rewind(aifmm_solver* s) {
  API_BEGIN
  AIFMM_REQUIRE(s, AIFMM_EINVAL, "NULL argument");
  AIFMM_CUDA(cudaSetDevice(s->s->ctx->device));
  s->s->rewind();
  API_END
}

int aifmm_profile_gemm(int on) {
  API_BEGIN
  gemm_profile_enable(on != 0);
  API_END
}

int aifmm_profile_gemm_read(double* ms, double* flops, long* launches) {
  API_BEGIN
  AIFMM_REQUIRE(ms && flops && launches, AIFMM_EINVAL, "NULL argument");
  gemm_profile_read(ms, flops, launches);
  API_END
}

int aifmm_profile_gemm_table(char* buf, int cap) {
  API_BEGIN
  AIFMM_REQUIRE(buf && cap > 0, AIFMM_EINVAL, "bad buffer");
  const std::string r = gemm_profile_table();
  const size_t n = std::min(r.size(), (size_t)cap - 1);
  std::memcpy(buf, r.data(), n);
  buf[n] = 0;
  API_END
}

int aifmm_solver_destroy(aifmm_solver* s) {
  API_BEGIN
  if (!s) return AIFMM_OK;
  aifmm_ctx* c = s->s->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  delete s;  // frees every block on the context stream
  ctx_release(c);
  API_END
}

}  // extern "C"

int aifmm_solver_aca_log(aifmm_solver* s, float* features, int* rmax0, int* ranks, int cap, int* n) {
  API_BEGIN
  AIFMM_REQUIRE(s && n && cap >= 0, AIFMM_EINVAL, "bad argument");
  const auto& L = s->s->acaLog;
  *n = (int)L.size();
  const int w = std::min(cap, (int)L.size());
  for (int i = 0; i < w; ++i) {
    if (features) std::memcpy(features + (size_t)MLP_IN * i, L[i].x.f, sizeof(float) * MLP_IN);
    if (rmax0) rmax0[i] = L[i].rmax0;
    if (ranks) ranks[i] = L[i].rank;
  }
  API_END
}

int aifmm_ctx_set_rank_model(aifmm_ctx* ctx, const aifmm_mlp* m, double margin) {
  API_BEGIN
  AIFMM_REQUIRE(ctx, AIFMM_EINVAL, "ctx is NULL");
  if (!m) {
    ctx->rankModel.reset();
    return AIFMM_OK;
  }
  AIFMM_REQUIRE(margin >= 1.0 && margin <= 16.0, AIFMM_EINVAL, "margin must lie in [1, 16]");
  // a value copy bound to this context (not reference-counted: the context owns it)
  auto c = std::make_shared<aifmm_mlp>();
  c->ctx = ctx;
  c->params = m->params;
  std::memcpy(c->mean, m->mean, sizeof(c->mean));
  std::memcpy(c->scale, m->scale, sizeof(c->scale));
  ctx->rankModel = c;
  ctx->rankMargin = margin;
  API_END
}
