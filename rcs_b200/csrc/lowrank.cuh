// Low-rank kernels of the GPU solver: partially pivoted ACA (one CTA per
// box, all boxes of a level in one launch) and the partitioned
// column-pivoted Householder QR used for fill-in recompression.
#pragma once
#include <vector>

#include "assemble.cuh"
#include "dense.cuh"

namespace aifmm {

// One ACA problem: K(rows[0..nr), cols[0..nc)), rank-revealing pivots.
struct ACAProblem {
  const int* rows;   // global unknown ids
  const int* cols;
  int nr, nc;
  int rmax;          // workspace rank bound
  zd* U;             // rmax x nP residual vectors of the "primary" side
  zd* V;             // rmax x nS normalised vectors of the "secondary" side
  zd* Ac;            // nr x rmax original columns (column-major, ld = nr)
  zd* Ar;            // rmax x nc original rows (ld = rmax)
  unsigned char* used;  // nr + nc flags
  int* rowBases;     // rmax
  int* colBases;     // rmax
  int* rank;         // out
  int* status;       // out: 0 ok, 1 = rmax reached before convergence
};

void launch_aca(aifmm_ctx* ctx, const KernelGeom& k, const std::vector<ACAProblem>& probs, double tol);

struct RRQRProblem {
  zd* R;             // m x n working copy (destroyed), ld = m
  int m, n;
  int partition;
  double tol1, tol2, inputPivot;
  int fillInRank;
  int realMode;
  zd* H;             // m x (min(m,n)+1) reflector storage
  double* nsq;       // n
  int* perm;         // n
  zd* Q;             // out: m x rank (ld = m); at most min(m,n) columns are written
  int* rank;         // out
  double* maxPivot;  // out
  int* istate;       // split pipeline only: 8 ints of scratch
  double* dstate;    // split pipeline only: 2 doubles of scratch
  int p2cap;         // split pipeline only: at most this many partition-2 steps (-1: no cap)
};

// Single-kernel RRQR (one CTA per problem).
void launch_rrqr(aifmm_ctx* ctx, const std::vector<RRQRProblem>& probs);
// Same factorization split into phases: the partition-1 panel in one CTA,
// the committed reflectors applied to the fill-in columns one warp per
// column, the partition-2 steps (pivot in one CTA, the reflector applied one
// warp per column), and Q_trunc one warp per column.  One problem runs as a
// single cooperative launch with grid-wide barriers between the phases;
// several as one launch per phase.  Needs istate/dstate; the result equals
// launch_rrqr's bit for bit.
void launch_rrqr_split(aifmm_ctx* ctx, const std::vector<RRQRProblem>& probs);

}  // namespace aifmm
