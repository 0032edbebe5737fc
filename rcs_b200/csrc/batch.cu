// Many independent bodies factorized and solved at once.
//
// The reference solves one geometry per process (test/sphere.cpp); a batch
// of bodies -- the uneven ellipsoids of a parameter sweep, each a few thousand
// unknowns -- leaves one GPU mostly idle when they run one after another,
// because each body's elimination is a chain of small launches and host
// decisions.  Here every body has its own context (its own stream, memory
// pool and arena) and a pool of host threads drives the bodies' factorizations
// (and then their FGMRES solves) concurrently, so the small kernels of many
// bodies share the GPU.  Results are those of the one-body calls, bit for bit:
// a body's arithmetic does not depend on what runs beside it.
#include <atomic>
#include <chrono>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "capi_guard.cuh"
#include "krylov.cuh"
#include "solver.cuh"

using namespace aifmm;

namespace {

// Runs job(i) for i < n on up to `threads` host threads; the first failure's
// status and message are returned (the other bodies still finish).
template <typename F>
int run_pool(int n, int threads, F job, std::string& msg) {
  std::atomic<int> next{0};
  std::mutex mu;
  int status = AIFMM_OK;
  auto worker = [&]() {
    for (int i = next++; i < n; i = next++) {
      int rc = AIFMM_OK;
      std::string m;
      try {
        job(i);
      } catch (const Error& e) {
        rc = e.code;
        m = e.what();
      } catch (const std::bad_alloc&) {
        rc = AIFMM_ENOMEM;
        m = "host allocation failed";
      } catch (const std::exception& e) {
        rc = AIFMM_EINVAL;
        m = e.what();
      }
      if (rc != AIFMM_OK) {
        std::lock_guard<std::mutex> l(mu);
        if (status == AIFMM_OK) {
          status = rc;
          msg = "body " + std::to_string(i) + ": " + m;
        }
      }
    }
  };
  const int nt = std::max(1, std::min(threads > 0 ? threads : 16, n));
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
  return status;
}

void check_distinct_contexts(aifmm_solver* const* s, int n) {
  for (int i = 0; i < n; ++i) {
    AIFMM_REQUIRE(s[i] != nullptr, AIFMM_EINVAL, "NULL solver in the batch");
    for (int q = 0; q < i; ++q)
      AIFMM_REQUIRE(s[q]->s->ctx != s[i]->s->ctx, AIFMM_EINVAL,
                    "the bodies of a batch need one context each (their streams run concurrently)");
  }
}

}  // namespace

extern "C" {

int aifmm_batch_factorize(aifmm_solver* const* solvers, int n, int threads, double* seconds) {
  API_BEGIN
  AIFMM_REQUIRE(solvers && n > 0, AIFMM_EINVAL, "bad argument");
  check_distinct_contexts(solvers, n);
  const auto t0 = std::chrono::steady_clock::now();
  std::string msg;
  const int rc = run_pool(n, threads, [&](int i) {
    Solver& S = *solvers[i]->s;
    AIFMM_CUDA(cudaSetDevice(S.ctx->device));
    S.factorize();
    ctx_trim(S.ctx);  // the elimination's temporaries go back to the device for the other bodies
  }, msg);
  if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (rc != AIFMM_OK) throw Error(rc, msg);
  API_END
}

int aifmm_batch_solve_gmres(aifmm_solver* const* solvers, aifmm_operator* const* ops, const double* const* rhs,
                            const int* nrhs, double* const* x, int n, double tol, int restart, int maxit, int threads,
                            aifmm_gmres_info* info, double* seconds) {
  API_BEGIN
  AIFMM_REQUIRE(solvers && ops && rhs && nrhs && x && n > 0, AIFMM_EINVAL, "bad argument");
  check_distinct_contexts(solvers, n);
  for (int i = 0; i < n; ++i) {
    AIFMM_REQUIRE(ops[i] && rhs[i] && x[i] && nrhs[i] > 0, AIFMM_EINVAL, "bad body arguments");
    AIFMM_REQUIRE(solvers[i]->s->factored, AIFMM_ESTATE, "solve before factorize");
  }
  const auto t0 = std::chrono::steady_clock::now();
  std::string msg;
  const int rc = run_pool(n, threads, [&](int i) {
    Solver& S = *solvers[i]->s;
    AIFMM_CUDA(cudaSetDevice(S.ctx->device));
    const size_t bytes = sizeof(zd) * (size_t)S.N * nrhs[i];
    DevBuf bd(S.ctx, bytes), xd(S.ctx, bytes);
    AIFMM_CUDA(cudaMemcpyAsync(bd.p, rhs[i], bytes, cudaMemcpyHostToDevice, S.ctx->stream));
    const GmresResult r = fgmres(S, *ops[i]->op, bd.as<zd>(), xd.as<zd>(), nrhs[i], tol, restart, maxit);
    AIFMM_CUDA(cudaMemcpyAsync(x[i], xd.p, bytes, cudaMemcpyDeviceToHost, S.ctx->stream));
    AIFMM_CUDA(cudaStreamSynchronize(S.ctx->stream));
    if (info) fill_gmres_info(r, &info[i]);
    S.dropPlan();  // the captured sweep's intermediates
    ctx_trim(S.ctx);
  }, msg);
  if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (rc != AIFMM_OK) throw Error(rc, msg);
  API_END
}

}  // extern "C"
