// Flexible GMRES(m) in FP64 around an approximate factorization: right
// preconditioning by the H^2 elimination (Solver::solve), residuals by the
// H^2 forward operator.  Every right-hand side runs its own Arnoldi process;
// all of them advance together so that each iteration is one multi-column
// preconditioner solve and one multi-column matvec.  Orthogonalisation is
// classical Gram-Schmidt applied twice; the small Hessenberg least-squares
// problems (Givens rotations) are solved on the host.
#pragma once
#include "h2op.cuh"

namespace aifmm {

struct GmresResult {
  int iterations = 0;  // Arnoldi steps (each: one preconditioner solve + one matvec)
  int cycles = 0;
  double relres = 0;   // max over columns of ||b - A x|| / ||b|| with the forward operator, after the last cycle
  double t_precond = 0, t_matvec = 0;  // seconds (host wall time, synchronised)
};

// x (N x nr, ld N, device) <- solution of A x = b.  tol: target relative
// residual; restart: Krylov dimension per cycle; maxit: cap on iterations.
GmresResult fgmres(Solver& M, H2Operator& A, const zd* b, zd* x, int nr, double tol, int restart, int maxit);

}  // namespace aifmm

// the C ABI's record of a solve (include/aifmm_b200.h)
extern "C" void fill_gmres_info(const aifmm::GmresResult& r, aifmm_gmres_info* info);
