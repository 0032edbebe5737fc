// ACA and partitioned RRQR kernels.
//
// ACA follows LowRank<K>::ACA_only_nodes2 (src/ACA.cpp:639-859): the first
// pivot is the first primary index whose largest remaining entry exceeds
// 1e-16; each step evaluates the secondary vector at the primary pivot, takes
// its largest remaining entry (lowest index on ties, maxAbsVector :25-38),
// normalises by it, evaluates the primary vector at that pivot, subtracts the
// previous rank-one terms in order, and updates the reference's normS
// recurrence (:750-754) -- including the term of the new vector with itself.
// "Primary" = rows when nr < nc (the reference's first branch), else columns.
//
// RRQR follows RRQR::colPivHouseholderQRWithPartition (src/rrqr.cpp:98-182):
// partition 1 pivots among the old-basis columns with tolerance tol1
// relative to its first pivot (early exit sets rank_partition1 = j-1, as the
// reference does), partition 2 pivots among all remaining columns with
// tolerance tol2 relative to max(inputPivot, its first pivot) and stops after
// fillInRank columns.  Columns are selected by the largest downdated norm;
// the reference re-sorts all remaining columns each step, which selects the
// same column except for exact ties.  Q_trunc is formed by applying the
// committed reflectors to the first rank columns of the identity, which
// equals the reference's explicit accumulation of the full Q.
#include "lowrank.cuh"

namespace aifmm {

// ------------------------------------------------------------------ reductions
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffff, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = (threadIdx.x < NT / 32) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffff, t, o);
    if (threadIdx.x == 0) sh[32] = t;
  }
  __syncthreads();
  return sh[32];
}

// Largest value, lowest index on ties; idx = -1 when nothing qualifies.
template <int NT>
__device__ __forceinline__ void block_argmax(double v, int idx, double* shv, int* shi, double& ov, int& oi) {
  for (int o = 16; o > 0; o >>= 1) {
    const double pv = __shfl_xor_sync(0xffffffff, v, o);
    const int pi = __shfl_xor_sync(0xffffffff, idx, o);
    if (pi >= 0 && (idx < 0 || pv > v || (pv == v && pi < idx))) { v = pv; idx = pi; }
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) { shv[threadIdx.x >> 5] = v; shi[threadIdx.x >> 5] = idx; }
  __syncthreads();
  if (threadIdx.x < 32) {
    v = (threadIdx.x < NT / 32) ? shv[threadIdx.x] : -1.0;
    idx = (threadIdx.x < NT / 32) ? shi[threadIdx.x] : -1;
    for (int o = 16; o > 0; o >>= 1) {
      const double pv = __shfl_xor_sync(0xffffffff, v, o);
      const int pi = __shfl_xor_sync(0xffffffff, idx, o);
      if (pi >= 0 && (idx < 0 || pv > v || (pv == v && pi < idx))) { v = pv; idx = pi; }
    }
    if (threadIdx.x == 0) { shv[32] = v; shi[32] = idx; }
  }
  __syncthreads();
  ov = shv[32];
  oi = shi[32];
}

__device__ __forceinline__ double zabs(zd z) { return hypot(z.x, z.y); }

// ------------------------------------------------------------------ ACA
constexpr int ACA_NT = 512;
constexpr int ACA_MAXR = 1024;  // shared dot buffers

template <bool EFIE>
__device__ __forceinline__ zd kentry(const KernelGeom& kg, int r, int c) {
  if (EFIE) return efie_entry(kg.ge, r, c);
  return zmk(es_entry(kg.gs, r, c), 0.0);
}

template <bool EFIE>
__global__ void __launch_bounds__(ACA_NT) aca_kernel(KernelGeom kg, const ACAProblem* __restrict__ probs, double tol) {
  __shared__ double shv[33];
  __shared__ int shi[33];
  __shared__ zd d1[ACA_MAXR], d2[ACA_MAXR];
  __shared__ zd s_piv;
  const ACAProblem P = probs[blockIdx.x];
  const int tid = threadIdx.x;
  const bool br1 = P.nr < P.nc;  // primary = rows
  const int nP = br1 ? P.nr : P.nc, nS = br1 ? P.nc : P.nr;
  const int* idP = br1 ? P.rows : P.cols;
  const int* idS = br1 ? P.cols : P.rows;
  unsigned char* usedP = br1 ? P.used : P.used + P.nr;
  unsigned char* usedS = br1 ? P.used + P.nr : P.used;
  const int mn = min(P.nr, P.nc);
  const int rmax = min(P.rmax, ACA_MAXR);
  // entry(p, s) in reference orientation
  auto ent = [&](int p, int s) -> zd { return br1 ? kentry<EFIE>(kg, idP[p], idS[s]) : kentry<EFIE>(kg, idS[s], idP[p]); };
  // original vectors: the secondary vector is a row of K when br1 (stored in Ar), a column otherwise (Ac)
  auto origS = [&](int r, int s) -> zd& { return br1 ? P.Ar[(size_t)s * P.rmax + r] : P.Ac[(size_t)r * P.nr + s]; };
  auto origP = [&](int r, int p) -> zd& { return br1 ? P.Ac[(size_t)r * P.nr + p] : P.Ar[(size_t)p * P.rmax + r]; };
  zd* U = P.U;  // U[r * nP + p]
  zd* V = P.V;  // V[r * nS + s]
  for (int i = tid; i < P.nr + P.nc; i += ACA_NT) P.used[i] = 0;
  __syncthreads();

  // ---- first pivot (ACA.cpp:670-677 / :761-768)
  int l, sidx = -1;
  double mval;
  for (l = 0; l < nP; ++l) {
    double bv = -1.0;
    int bi = -1;
    for (int s = tid; s < nS; s += ACA_NT) {
      const zd z = ent(l, s);
      V[s] = z;
      origS(0, s) = z;
      const double a = zabs(z);
      if (bi < 0 || a > bv) { bv = a; bi = s; }
    }
    block_argmax<ACA_NT>(bv, bi, shv, shi, mval, sidx);
    if (mval > 1e-16) break;
  }
  if (l == nP || sidx < 0) {
    if (tid == 0) { *P.rank = 0; *P.status = 0; }
    return;
  }
  int pidx = l;
  if (tid == 0) s_piv = V[sidx];
  __syncthreads();
  const zd piv0 = s_piv;
  for (int s = tid; s < nS; s += ACA_NT) V[s] = zdiv(V[s], piv0);
  for (int p = tid; p < nP; p += ACA_NT) {
    const zd z = ent(p, sidx);
    U[p] = z;
    origP(0, p) = z;
  }
  if (tid == 0) {
    (br1 ? P.rowBases : P.colBases)[0] = pidx;
    (br1 ? P.colBases : P.rowBases)[0] = sidx;
    usedP[pidx] = 1;
    usedS[sidx] = 1;
  }
  __syncthreads();
  int rank = 1;
  double normS = 0.0;
  // next primary pivot from u (= the first primary vector)
  {
    double bv = -1.0;
    int bi = -1;
    for (int p = tid; p < nP; p += ACA_NT)
      if (!usedP[p]) {
        const double a = zabs(U[p]);
        if (bi < 0 || a > bv) { bv = a; bi = p; }
      }
    double dummy;
    block_argmax<ACA_NT>(bv, bi, shv, shi, dummy, pidx);
  }
  double un, vn;
  {
    double s1 = 0.0, s2 = 0.0;
    for (int p = tid; p < nP; p += ACA_NT) s1 += zabs2(U[p]);
    un = sqrt(block_sum<ACA_NT>(s1, shv));
    for (int s = tid; s < nS; s += ACA_NT) s2 += zabs2(V[s]);
    vn = sqrt(block_sum<ACA_NT>(s2, shv));
  }
  int status = 0;
  while (un * vn > tol * normS && rank < mn) {
    if (rank >= rmax || pidx < 0) {
      status = 1;
      break;
    }
    const int r = rank;
    zd* Vr = V + (size_t)r * nS;
    zd* Ur = U + (size_t)r * nP;
    // secondary residual at the primary pivot
    double bv = -1.0;
    int bi = -1;
    for (int s = tid; s < nS; s += ACA_NT) {
      zd z = ent(pidx, s);
      origS(r, s) = z;
      for (int q = 0; q < r; ++q) z = zsub(z, zmul(U[(size_t)q * nP + pidx], V[(size_t)q * nS + s]));
      Vr[s] = z;
      if (!usedS[s]) {
        const double a = zabs(z);
        if (bi < 0 || a > bv) { bv = a; bi = s; }
      }
    }
    block_argmax<ACA_NT>(bv, bi, shv, shi, mval, sidx);
    if (tid == 0) s_piv = Vr[sidx];
    __syncthreads();
    const zd piv = s_piv;
    for (int s = tid; s < nS; s += ACA_NT) Vr[s] = zdiv(Vr[s], piv);
    // primary residual at the secondary pivot
    for (int p = tid; p < nP; p += ACA_NT) {
      zd z = ent(p, sidx);
      origP(r, p) = z;
      for (int q = 0; q < r; ++q) z = zsub(z, zmul(V[(size_t)q * nS + sidx], U[(size_t)q * nP + p]));
      Ur[p] = z;
    }
    __syncthreads();
    if (tid == 0) {
      (br1 ? P.rowBases : P.colBases)[r] = pidx;
      (br1 ? P.colBases : P.rowBases)[r] = sidx;
      usedP[pidx] = 1;
      usedS[sidx] = 1;
    }
    rank = r + 1;
    // norms and the normS recurrence (ACA.cpp:748-754)
    {
      double s1 = 0.0, s2 = 0.0;
      for (int p = tid; p < nP; p += ACA_NT) s1 += zabs2(Ur[p]);
      un = sqrt(block_sum<ACA_NT>(s1, shv));
      for (int s = tid; s < nS; s += ACA_NT) s2 += zabs2(Vr[s]);
      vn = sqrt(block_sum<ACA_NT>(s2, shv));
    }
    const int warp = tid >> 5, lane = tid & 31;
    for (int q = warp; q < rank; q += ACA_NT / 32) {
      zd a = zmk(0, 0), b = zmk(0, 0);
      for (int p = lane; p < nP; p += 32) a = zadd(a, zcmul(U[(size_t)q * nP + p], Ur[p]));
      for (int s = lane; s < nS; s += 32) b = zadd(b, zcmul(V[(size_t)q * nS + s], Vr[s]));
      for (int o = 16; o > 0; o >>= 1) {
        a.x += __shfl_xor_sync(0xffffffff, a.x, o);
        a.y += __shfl_xor_sync(0xffffffff, a.y, o);
        b.x += __shfl_xor_sync(0xffffffff, b.x, o);
        b.y += __shfl_xor_sync(0xffffffff, b.y, o);
      }
      if (lane == 0) { d1[q] = a; d2[q] = b; }
    }
    __syncthreads();
    if (tid == 0) {
      double ns = normS * normS + (un * vn) * (un * vn);
      for (int q = 0; q < rank; ++q) ns += 2 * zabs(zmul(d1[q], d2[q]));
      shv[32] = sqrt(ns);
    }
    __syncthreads();
    normS = shv[32];
    __syncthreads();
    // next primary pivot from the new primary residual
    {
      double pv = -1.0;
      int pi = -1;
      for (int p = tid; p < nP; p += ACA_NT)
        if (!usedP[p]) {
          const double a = zabs(Ur[p]);
          if (pi < 0 || a > pv) { pv = a; pi = p; }
        }
      double dummy;
      block_argmax<ACA_NT>(pv, pi, shv, shi, dummy, pidx);
    }
  }
  if (tid == 0) {
    *P.rank = rank;
    *P.status = status;
  }
}

void launch_aca(aifmm_ctx* ctx, const KernelGeom& k, const std::vector<ACAProblem>& probs, double tol) {
  if (probs.empty()) return;
  DevBuf dp = upload(ctx, probs);
  if (k.efie) aca_kernel<true><<<(unsigned)probs.size(), ACA_NT, 0, ctx->stream>>>(k, dp.as<ACAProblem>(), tol);
  else aca_kernel<false><<<(unsigned)probs.size(), ACA_NT, 0, ctx->stream>>>(k, dp.as<ACAProblem>(), tol);
  AIFMM_LAUNCHED();
}

// ------------------------------------------------------------------ RRQR
constexpr int QR_NT = 1024;

__global__ void __launch_bounds__(QR_NT) rrqr_kernel(const RRQRProblem* __restrict__ probs) {
  __shared__ double shv[33];
  __shared__ int shi[33];
  __shared__ zd s_alpha;
  const RRQRProblem P = probs[blockIdx.x];
  const int tid = threadIdx.x, m = P.m, n = P.n;
  const int warp = tid >> 5, lane = tid & 31, nwarp = QR_NT / 32;
  zd* R = P.R;
  // column norms (rrqr.cpp:111) and identity permutation
  for (int c = warp; c < n; c += nwarp) {
    double s = 0.0;
    for (int i = lane; i < m; i += 32) s += zabs2(R[(size_t)c * m + i]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffff, s, o);
    if (lane == 0) { P.nsq[c] = s; P.perm[c] = c; }
  }
  __syncthreads();
  int nref = 0;  // committed reflectors
  double maxPivot = 0.0, mp1 = 0.0;
  const int partition = P.partition;
  int rank_p1 = min(partition, m);
  int steps = min(m, n);
  // One pivoting step at position j over positions [j, end).  Returns false
  // when the pivot test says stop; the reflector is then not committed.
  auto step = [&](int j, int end, bool part1, int first) -> bool {
    // pivot: largest downdated norm among positions [j, end)
    double bv = -1.0;
    int bi = -1;
    for (int q = j + tid; q < end; q += QR_NT) {
      const double v = P.nsq[q];
      if (bi < 0 || v > bv) { bv = v; bi = q; }
    }
    double mv;
    int pos;
    block_argmax<QR_NT>(bv, bi, shv, shi, mv, pos);
    if (tid == 0 && pos != j) {
      double t = P.nsq[j]; P.nsq[j] = P.nsq[pos]; P.nsq[pos] = t;
      int u = P.perm[j]; P.perm[j] = P.perm[pos]; P.perm[pos] = u;
    }
    __syncthreads();
    const int c = P.perm[j];
    zd* x = R + (size_t)c * m;
    // Householder vector (gethouselholderVec, rrqr.cpp:75-96)
    double s = 0.0;
    for (int i = j + tid; i < m; i += QR_NT) s += zabs2(x[i]);
    const double xn = sqrt(block_sum<QR_NT>(s, shv));
    zd* h = P.H + (size_t)nref * m;
    if (tid == 0) {
      const zd xj = x[j];
      zd add;
      if (P.realMode) add = zmk((xj.x >= 0 ? 1.0 : -1.0) * xn, 0.0);
      else {
        double sn, cs;
        sincos(atan2(xj.y, xj.x), &sn, &cs);
        add = zmk(cs * xn, sn * xn);
      }
      s_alpha = zadd(xj, add);
    }
    __syncthreads();
    double s2 = 0.0;
    for (int i = tid; i < m; i += QR_NT) {
      zd v = (i < j) ? zmk(0, 0) : ((i == j) ? s_alpha : x[i]);
      h[i] = v;
      s2 += zabs2(v);
    }
    const double hn = sqrt(block_sum<QR_NT>(s2, shv));
    __syncthreads();
    if (hn > 0) {  // v = v * sqrt(2) / |v|
      const double r2 = sqrt(2.0);
      for (int i = j + tid; i < m; i += QR_NT) h[i] = zmk((h[i].x * r2) / hn, (h[i].y * r2) / hn);
    }
    __syncthreads();
    // pivot value after the reflection: R(j,c) - h_j (h^H x)
    zd w = zmk(0, 0);
    for (int i = j + tid; i < m; i += QR_NT) w = zadd(w, zcmul(h[i], x[i]));
    double wr = block_sum<QR_NT>(w.x, shv);
    double wi = block_sum<QR_NT>(w.y, shv);
    const zd rjj = zsub(x[j], zmul(h[j], zmk(wr, wi)));
    const double pivot = zabs(rjj);
    bool stop;
    if (part1) {
      if (j == 0) mp1 = pivot;
      maxPivot = mp1;
      stop = (pivot / mp1 < P.tol1);
    } else {
      if (j == first) maxPivot = fmax(P.inputPivot, pivot);
      stop = (pivot / maxPivot < P.tol2 || j - first >= P.fillInRank);
    }
    if (stop) return false;
    // apply the reflector to the columns at positions >= j
    for (int q = j + warp; q < n; q += nwarp) {
      zd* y = R + (size_t)P.perm[q] * m;
      zd a = zmk(0, 0);
      for (int i = j + lane; i < m; i += 32) a = zadd(a, zcmul(h[i], y[i]));
      for (int o = 16; o > 0; o >>= 1) {
        a.x += __shfl_xor_sync(0xffffffff, a.x, o);
        a.y += __shfl_xor_sync(0xffffffff, a.y, o);
      }
      for (int i = j + lane; i < m; i += 32) y[i] = zsub(y[i], zmul(h[i], a));
    }
    __syncthreads();
    for (int i = j + 1 + tid; i < m; i += QR_NT) x[i] = zmk(0, 0);
    for (int q = j + 1 + tid; q < n; q += QR_NT) {
      const zd rjq = R[(size_t)P.perm[q] * m + j];
      const double a = zabs(rjq);
      P.nsq[q] = P.nsq[q] - a * a;
    }
    nref++;
    __syncthreads();
    return true;
  };
  for (int j = 0; j < rank_p1; ++j)
    if (!step(j, partition, true, 0)) {
      rank_p1 = j - 1;  // rrqr.cpp:116
      break;
    }
  for (int q = rank_p1 + tid; q < partition; q += QR_NT) P.nsq[q] = 0.0;
  __syncthreads();
  steps = steps - (partition - rank_p1);
  const int first = rank_p1;
  int rank_p2 = min(steps - first, m);
  for (int j = first; j < steps; ++j)
    if (!step(j, n, false, first)) {
      rank_p2 = j - first;
      break;
    }
  const int rank = rank_p1 + rank_p2;
  // Q_trunc = H_0 H_1 ... H_{nref-1} [I_rank; 0]
  for (int t = tid; t < m * rank; t += QR_NT) {
    const int i = t % m, c = t / m;
    P.Q[(size_t)c * m + i] = (i == c) ? zmk(1, 0) : zmk(0, 0);
  }
  __syncthreads();
  for (int r = nref - 1; r >= 0; --r) {
    const zd* h = P.H + (size_t)r * m;
    for (int c = warp; c < rank; c += nwarp) {
      zd* y = P.Q + (size_t)c * m;
      zd a = zmk(0, 0);
      for (int i = lane; i < m; i += 32) a = zadd(a, zcmul(h[i], y[i]));
      for (int o = 16; o > 0; o >>= 1) {
        a.x += __shfl_xor_sync(0xffffffff, a.x, o);
        a.y += __shfl_xor_sync(0xffffffff, a.y, o);
      }
      for (int i = lane; i < m; i += 32) y[i] = zsub(y[i], zmul(h[i], a));
    }
    __syncthreads();
  }
  if (tid == 0) {
    *P.rank = rank;
    *P.maxPivot = maxPivot;
  }
}

void launch_rrqr(aifmm_ctx* ctx, const std::vector<RRQRProblem>& probs) {
  if (probs.empty()) return;
  DevBuf dp = upload(ctx, probs);
  rrqr_kernel<<<(unsigned)probs.size(), QR_NT, 0, ctx->stream>>>(dp.as<RRQRProblem>());
  AIFMM_LAUNCHED();
}

}  // namespace aifmm

// ------------------------------------------------------------------ RRQR, split
namespace aifmm {

// Partition 2 runs as per-step launches when it has at most this many steps
// (the solver's fill-in recompressions have 5 to 11); longer runs keep the
// single-CTA panel kernel.
constexpr int kRRQRStepLaunchMax = 32;

// One pivoting step at position j: pivot among positions [j, end), reflector
// applied to (and norms downdated for) positions [j, applyEnd).  Same
// arithmetic as the step of rrqr_kernel.  Returns false on the stop test.
__device__ bool rrqr_step_dev(const RRQRProblem& P, int j, int end, int applyEnd, bool part1, int first, int& nref,
                              double& mp1, double& maxPivot, double* shv, int* shi, zd& s_alpha) {
  const int tid = threadIdx.x, m = P.m;
  const int warp = tid >> 5, lane = tid & 31, nwarp = QR_NT / 32;
  zd* R = P.R;
  double bv = -1.0;
  int bi = -1;
  for (int q = j + tid; q < end; q += QR_NT) {
    const double v = P.nsq[q];
    if (bi < 0 || v > bv) { bv = v; bi = q; }
  }
  double mv;
  int pos;
  block_argmax<QR_NT>(bv, bi, shv, shi, mv, pos);
  if (tid == 0 && pos != j) {
    double t = P.nsq[j]; P.nsq[j] = P.nsq[pos]; P.nsq[pos] = t;
    int u = P.perm[j]; P.perm[j] = P.perm[pos]; P.perm[pos] = u;
  }
  __syncthreads();
  const int c = P.perm[j];
  zd* x = R + (size_t)c * m;
  double s = 0.0;
  for (int i = j + tid; i < m; i += QR_NT) s += zabs2(x[i]);
  const double xn = sqrt(block_sum<QR_NT>(s, shv));
  zd* h = P.H + (size_t)nref * m;
  if (tid == 0) {
    const zd xj = x[j];
    zd add;
    if (P.realMode) add = zmk((xj.x >= 0 ? 1.0 : -1.0) * xn, 0.0);
    else {
      double sn, cs;
      sincos(atan2(xj.y, xj.x), &sn, &cs);
      add = zmk(cs * xn, sn * xn);
    }
    s_alpha = zadd(xj, add);
  }
  __syncthreads();
  double s2 = 0.0;
  for (int i = tid; i < m; i += QR_NT) {
    zd v = (i < j) ? zmk(0, 0) : ((i == j) ? s_alpha : x[i]);
    h[i] = v;
    s2 += zabs2(v);
  }
  const double hn = sqrt(block_sum<QR_NT>(s2, shv));
  __syncthreads();
  if (hn > 0) {
    const double r2 = sqrt(2.0);
    for (int i = j + tid; i < m; i += QR_NT) h[i] = zmk((h[i].x * r2) / hn, (h[i].y * r2) / hn);
  }
  __syncthreads();
  zd w = zmk(0, 0);
  for (int i = j + tid; i < m; i += QR_NT) w = zadd(w, zcmul(h[i], x[i]));
  double wr = block_sum<QR_NT>(w.x, shv);
  double wi = block_sum<QR_NT>(w.y, shv);
  const zd rjj = zsub(x[j], zmul(h[j], zmk(wr, wi)));
  const double pivot = zabs(rjj);
  bool stop;
  if (part1) {
    if (j == 0) mp1 = pivot;
    maxPivot = mp1;
    stop = (pivot / mp1 < P.tol1);
  } else {
    if (j == first) maxPivot = fmax(P.inputPivot, pivot);
    stop = (pivot / maxPivot < P.tol2 || j - first >= P.fillInRank);
  }
  if (stop) return false;
  for (int q = j + warp; q < applyEnd; q += nwarp) {
    zd* y = R + (size_t)P.perm[q] * m;
    zd a = zmk(0, 0);
    for (int i = j + lane; i < m; i += 32) a = zadd(a, zcmul(h[i], y[i]));
    for (int o = 16; o > 0; o >>= 1) {
      a.x += __shfl_xor_sync(0xffffffff, a.x, o);
      a.y += __shfl_xor_sync(0xffffffff, a.y, o);
    }
    for (int i = j + lane; i < m; i += 32) y[i] = zsub(y[i], zmul(h[i], a));
  }
  __syncthreads();
  for (int i = j + 1 + tid; i < m; i += QR_NT) x[i] = zmk(0, 0);
  for (int q = j + 1 + tid; q < applyEnd; q += QR_NT) {
    const zd rjq = R[(size_t)P.perm[q] * m + j];
    const double a = zabs(rjq);
    P.nsq[q] = P.nsq[q] - a * a;
  }
  nref++;
  __syncthreads();
  return true;
}

// ---- partition 2 as one launch pair per step (pivot/reflector on one CTA,
// reflector application one warp per column across the GPU).  The arithmetic
// of each column is the same as in rrqr_step_dev, so the result equals the
// single-CTA panel bit for bit.  State between launches lives in istate
// ([0] committed reflectors, [1] rank of partition 1, [4] done, [5] partition-2
// commits, [6] position of the step to apply or -1, [7] its reflector) and
// dstate ([0] first pivot of partition 1, [1] maxPivot).  A step after the stop
// (or past the step bound) returns at once.

__device__ inline void rrqr_p2_bounds(const RRQRProblem& P, int& first, int& steps) {
  const int rank_p1 = P.istate[1];
  first = rank_p1;
  steps = min(P.m, P.n) - (P.partition - rank_p1);
  if (P.p2cap >= 0) steps = min(steps, first + P.p2cap);
}

__device__ void rrqr_p2_init_body(const RRQRProblem& P) {
  for (int q = P.istate[1] + threadIdx.x; q < P.partition; q += blockDim.x) P.nsq[q] = 0.0;
  if (threadIdx.x == 0) {
    P.istate[4] = 0;
    P.istate[5] = 0;
    P.istate[6] = -1;
    P.istate[7] = 0;
  }
}
__global__ void rrqr_p2_init_kernel(const RRQRProblem* __restrict__ probs) { rrqr_p2_init_body(probs[blockIdx.x]); }

// one CTA of QR_NT threads
__device__ void rrqr_p2_pivot_body(const RRQRProblem& P, int t, double* shv, int* shi, zd& s_alpha) {
  const int tid = threadIdx.x, m = P.m, n = P.n;
  if (P.istate[4]) {  // stopped earlier: nothing to apply
    if (tid == 0) P.istate[6] = -1;
    return;
  }
  int first, steps;
  rrqr_p2_bounds(P, first, steps);
  const int j = first + t;
  if (j >= steps) {
    if (tid == 0) {
      P.istate[4] = 1;
      P.istate[6] = -1;
    }
    return;
  }
  const int nref = P.istate[0];
  double maxPivot = P.dstate[1];
  zd* R = P.R;
  // pivot, Householder vector and stop test: the first half of rrqr_step_dev
  double bv = -1.0;
  int bi = -1;
  for (int q = j + tid; q < n; q += QR_NT) {
    const double v = P.nsq[q];
    if (bi < 0 || v > bv) { bv = v; bi = q; }
  }
  double mv;
  int pos;
  block_argmax<QR_NT>(bv, bi, shv, shi, mv, pos);
  if (tid == 0 && pos != j) {
    double tt = P.nsq[j]; P.nsq[j] = P.nsq[pos]; P.nsq[pos] = tt;
    int u = P.perm[j]; P.perm[j] = P.perm[pos]; P.perm[pos] = u;
  }
  __syncthreads();
  const int c = P.perm[j];
  zd* x = R + (size_t)c * m;
  double s = 0.0;
  for (int i = j + tid; i < m; i += QR_NT) s += zabs2(x[i]);
  const double xn = sqrt(block_sum<QR_NT>(s, shv));
  zd* h = P.H + (size_t)nref * m;
  if (tid == 0) {
    const zd xj = x[j];
    zd add;
    if (P.realMode) add = zmk((xj.x >= 0 ? 1.0 : -1.0) * xn, 0.0);
    else {
      double sn, cs;
      sincos(atan2(xj.y, xj.x), &sn, &cs);
      add = zmk(cs * xn, sn * xn);
    }
    s_alpha = zadd(xj, add);
  }
  __syncthreads();
  double s2 = 0.0;
  for (int i = tid; i < m; i += QR_NT) {
    zd v = (i < j) ? zmk(0, 0) : ((i == j) ? s_alpha : x[i]);
    h[i] = v;
    s2 += zabs2(v);
  }
  const double hn = sqrt(block_sum<QR_NT>(s2, shv));
  __syncthreads();
  if (hn > 0) {
    const double r2 = sqrt(2.0);
    for (int i = j + tid; i < m; i += QR_NT) h[i] = zmk((h[i].x * r2) / hn, (h[i].y * r2) / hn);
  }
  __syncthreads();
  zd w = zmk(0, 0);
  for (int i = j + tid; i < m; i += QR_NT) w = zadd(w, zcmul(h[i], x[i]));
  double wr = block_sum<QR_NT>(w.x, shv);
  double wi = block_sum<QR_NT>(w.y, shv);
  const zd rjj = zsub(x[j], zmul(h[j], zmk(wr, wi)));
  const double pivot = zabs(rjj);
  if (j == first) maxPivot = fmax(P.inputPivot, pivot);
  const bool stop = (pivot / maxPivot < P.tol2 || j - first >= P.fillInRank);
  if (tid == 0) {
    P.dstate[1] = maxPivot;
    if (stop) {
      P.istate[4] = 1;
      P.istate[6] = -1;
    } else {
      P.istate[6] = j;
      P.istate[7] = nref;
      P.istate[0] = nref + 1;
      P.istate[5] += 1;
    }
  }
}
__global__ void __launch_bounds__(QR_NT) rrqr_p2_pivot_kernel(const RRQRProblem* __restrict__ probs, int t) {
  __shared__ double shv[33];
  __shared__ int shi[33];
  __shared__ zd s_alpha;
  rrqr_p2_pivot_body(probs[blockIdx.x], t, shv, shi, s_alpha);
}

// The committed reflector of the step applied to the columns at positions
// >= j, one warp per column, with the pivot column's sub-diagonal zeroed and
// the downdates of the norms at positions > j.
// column at position q (>= j) by one warp
__device__ void rrqr_p2_apply_col(const RRQRProblem& P, int j, int q, int lane) {
  const int m = P.m;
  const zd* h = P.H + (size_t)P.istate[7] * m;
  zd* y = P.R + (size_t)P.perm[q] * m;
  zd a = zmk(0, 0);
  // unrolled so that several loads of h and y are in flight per lane (the
  // accumulation order of each lane is unchanged)
#pragma unroll 4
  for (int i = j + lane; i < m; i += 32) a = zadd(a, zcmul(h[i], y[i]));
  for (int o = 16; o > 0; o >>= 1) {
    a.x += __shfl_xor_sync(0xffffffff, a.x, o);
    a.y += __shfl_xor_sync(0xffffffff, a.y, o);
  }
#pragma unroll 4
  for (int i = j + lane; i < m; i += 32) y[i] = zsub(y[i], zmul(h[i], a));
  __syncwarp();
  if (q == j) {
    for (int i = j + 1 + lane; i < m; i += 32) y[i] = zmk(0, 0);
  } else if (lane == 0) {
    const double ab = zabs(y[j]);
    P.nsq[q] = P.nsq[q] - ab * ab;
  }
}
__global__ void rrqr_p2_apply_kernel(const RRQRProblem* __restrict__ probs) {
  const RRQRProblem P = probs[blockIdx.y];
  const int j = P.istate[6];
  if (j < 0) return;
  const int q = j + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (q >= P.n) return;
  rrqr_p2_apply_col(P, j, q, threadIdx.x & 31);
}

__device__ void rrqr_p2_finish_body(const RRQRProblem& P) {
  if (threadIdx.x != 0) return;
  int first, steps;
  rrqr_p2_bounds(P, first, steps);
  const int rank_p2 = (steps - first <= 0) ? min(steps - first, P.m) : P.istate[5];
  const int rank = P.istate[1] + rank_p2;
  P.istate[2] = P.istate[0];
  P.istate[3] = rank;
  *P.rank = rank;
  *P.maxPivot = P.dstate[1];
}
__global__ void rrqr_p2_finish_kernel(const RRQRProblem* __restrict__ probs) { rrqr_p2_finish_body(probs[blockIdx.x]); }

// Partition 1 on the old-basis panel (positions [0, partition)).
// one CTA of QR_NT threads
__device__ void rrqr_p1_body(const RRQRProblem& P, double* shv, int* shi, zd& s_alpha) {
  const int tid = threadIdx.x, m = P.m, n = P.n;
  const int warp = tid >> 5, lane = tid & 31, nwarp = QR_NT / 32;
  for (int q = tid; q < n; q += QR_NT) P.perm[q] = q;
  for (int c = warp; c < P.partition; c += nwarp) {
    double s = 0.0;
    for (int i = lane; i < m; i += 32) s += zabs2(P.R[(size_t)c * m + i]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffff, s, o);
    if (lane == 0) P.nsq[c] = s;
  }
  __syncthreads();
  int nref = 0;
  double mp1 = 0.0, maxPivot = 0.0;
  int rank_p1 = min(P.partition, m);
  for (int j = 0; j < rank_p1; ++j)
    if (!rrqr_step_dev(P, j, P.partition, P.partition, true, 0, nref, mp1, maxPivot, shv, shi, s_alpha)) {
      rank_p1 = j - 1;
      break;
    }
  if (tid == 0) {
    P.istate[0] = nref;
    P.istate[1] = rank_p1;
    P.dstate[0] = mp1;
    P.dstate[1] = maxPivot;
  }
}
__global__ void __launch_bounds__(QR_NT) rrqr_p1_kernel(const RRQRProblem* __restrict__ probs) {
  __shared__ double shv[33];
  __shared__ int shi[33];
  __shared__ zd s_alpha;
  rrqr_p1_body(probs[blockIdx.x], shv, shi, s_alpha);
}

// The committed partition-1 reflectors applied to every fill-in column (one
// warp per column), with the reference's norm downdates in step order.
// fill-in column q by one warp
__device__ void rrqr_fill_col(const RRQRProblem& P, int q, int lane) {
  const int m = P.m;
  const int nref = P.istate[0];
  zd* y = P.R + (size_t)q * m;
  double s = 0.0;
  for (int i = lane; i < m; i += 32) s += zabs2(y[i]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffff, s, o);
  double nsq = s;
  for (int r = 0; r < nref; ++r) {
    const zd* h = P.H + (size_t)r * m;
    zd a = zmk(0, 0);
    for (int i = r + lane; i < m; i += 32) a = zadd(a, zcmul(h[i], y[i]));
    for (int o = 16; o > 0; o >>= 1) {
      a.x += __shfl_xor_sync(0xffffffff, a.x, o);
      a.y += __shfl_xor_sync(0xffffffff, a.y, o);
    }
    for (int i = r + lane; i < m; i += 32) y[i] = zsub(y[i], zmul(h[i], a));
    __syncwarp();
    const double ab = zabs(y[r]);
    nsq = nsq - ab * ab;
  }
  if (lane == 0) P.nsq[q] = nsq;
}
__global__ void rrqr_fill_kernel(const RRQRProblem* __restrict__ probs) {
  const RRQRProblem P = probs[blockIdx.y];
  const int q = P.partition + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (q >= P.n) return;
  rrqr_fill_col(P, q, threadIdx.x & 31);
}

// Partition 2 over positions [first, n), then the rank and outputs.
__global__ void __launch_bounds__(QR_NT) rrqr_p2_kernel(const RRQRProblem* __restrict__ probs) {
  __shared__ double shv[33];
  __shared__ int shi[33];
  __shared__ zd s_alpha;
  const RRQRProblem P = probs[blockIdx.x];
  const int tid = threadIdx.x, m = P.m, n = P.n;
  int nref = P.istate[0];
  int rank_p1 = P.istate[1];
  double mp1 = P.dstate[0], maxPivot = P.dstate[1];
  const int partition = P.partition;
  for (int q = rank_p1 + tid; q < partition; q += QR_NT) P.nsq[q] = 0.0;
  __syncthreads();
  int steps = min(m, n) - (partition - rank_p1);
  const int first = rank_p1;
  if (P.p2cap >= 0) steps = min(steps, first + P.p2cap);
  int rank_p2 = min(steps - first, m);
  for (int j = first; j < steps; ++j)
    if (!rrqr_step_dev(P, j, n, n, false, first, nref, mp1, maxPivot, shv, shi, s_alpha)) {
      rank_p2 = j - first;
      break;
    }
  if (tid == 0) {
    P.istate[2] = nref;
    P.istate[3] = rank_p1 + rank_p2;
    *P.rank = rank_p1 + rank_p2;
    *P.maxPivot = maxPivot;
  }
}

// Q_trunc column c = H_0 ... H_{nref-1} e_c, one warp per column.
// Q_trunc column c (< rank) by one warp
__device__ void rrqr_q_col(const RRQRProblem& P, int c, int lane) {
  const int m = P.m;
  const int nref = P.istate[2];
  zd* y = P.Q + (size_t)c * m;
  for (int i = lane; i < m; i += 32) y[i] = (i == c) ? zmk(1, 0) : zmk(0, 0);
  __syncwarp();
  for (int r = nref - 1; r >= 0; --r) {
    const zd* h = P.H + (size_t)r * m;
    zd a = zmk(0, 0);
    for (int i = lane; i < m; i += 32) a = zadd(a, zcmul(h[i], y[i]));
    for (int o = 16; o > 0; o >>= 1) {
      a.x += __shfl_xor_sync(0xffffffff, a.x, o);
      a.y += __shfl_xor_sync(0xffffffff, a.y, o);
    }
    for (int i = lane; i < m; i += 32) y[i] = zsub(y[i], zmul(h[i], a));
    __syncwarp();
  }
}
__global__ void rrqr_q_kernel(const RRQRProblem* __restrict__ probs) {
  const RRQRProblem P = probs[blockIdx.y];
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (c >= P.istate[3]) return;
  rrqr_q_col(P, c, threadIdx.x & 31);
}

// ---- the split pipeline of one problem as one cooperative launch
// The same device bodies as the per-step launches (so the same arithmetic,
// bit for bit), separated by grid-wide barriers instead of kernel
// boundaries: CTA 0 runs the single-CTA phases (partition 1, each step's
// pivot and reflector, the outputs), every warp of the grid the per-column
// phases.  A cooperative launch makes every CTA resident at once, so the
// barriers complete; each wait is still bounded (one second) and a barrier
// that runs out marks the problem's rank -2 (the host reports a timeout).
__device__ __forceinline__ unsigned long long rrqr_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ bool rrqr_grid_sync(unsigned* bar, unsigned target, int* err) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(bar, 1u);
    const unsigned long long t0 = rrqr_now();
    while (*(volatile unsigned*)bar < target) {
      if (*(volatile int*)err || rrqr_now() - t0 > 1000000000ull) {
        atomicExch(err, 1);
        break;
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile int*)err == 0;
}

// Several independent problems share one cooperative launch: problem p owns
// the CTAs [start[p], start[p+1]) and runs its phases on them alone; the
// barriers span the whole grid, so a problem whose partition 2 stops early
// only waits for the others.
constexpr int kRRQRFusedMax = 8;
struct RRQRFusedLayout {
  int np;
  int start[kRRQRFusedMax + 1];
};

__global__ void __launch_bounds__(QR_NT) rrqr_fused_kernel(const RRQRProblem* __restrict__ probs,
                                                           RRQRFusedLayout lay, int p2steps, unsigned* bar,
                                                           int* err) {
  __shared__ double shv[33];
  __shared__ int shi[33];
  __shared__ zd s_alpha;
  int pi = 0;
  while (pi + 1 < lay.np && (int)blockIdx.x >= lay.start[pi + 1]) ++pi;
  const RRQRProblem P = probs[pi];
  const int cta = (int)blockIdx.x - lay.start[pi], nctas = lay.start[pi + 1] - lay.start[pi];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = QR_NT / 32;
  const int stride = nctas * nw;
  unsigned target = 0;
  auto sync = [&]() {
    target += gridDim.x;
    if (rrqr_grid_sync(bar, target, err)) return true;
    if (cta == 0 && threadIdx.x == 0) *P.rank = -2;
    return false;
  };
  if (cta == 0) rrqr_p1_body(P, shv, shi, s_alpha);
  if (!sync()) return;
  for (int q = P.partition + cta * nw + warp; q < P.n; q += stride) rrqr_fill_col(P, q, lane);
  if (!sync()) return;
  if (cta == 0) rrqr_p2_init_body(P);
  if (!sync()) return;
  for (int t = 0; t < p2steps; ++t) {
    if (cta == 0) rrqr_p2_pivot_body(P, t, shv, shi, s_alpha);
    if (!sync()) return;
    const int j = *(volatile int*)&P.istate[6];
    if (j >= 0)
      for (int q = j + cta * nw + warp; q < P.n; q += stride) rrqr_p2_apply_col(P, j, q, lane);
    if (!sync()) return;
  }
  if (cta == 0) rrqr_p2_finish_body(P);
  if (!sync()) return;
  const int rank = *(volatile int*)&P.istate[3];
  for (int c = cta * nw + warp; c < rank; c += stride) rrqr_q_col(P, c, lane);
}

void launch_rrqr_split(aifmm_ctx* ctx, const std::vector<RRQRProblem>& probs) {
  if (probs.empty()) return;
  int maxFill = 1, maxCols = 1;
  for (const RRQRProblem& p : probs) {
    AIFMM_REQUIRE(p.istate && p.dstate, AIFMM_EINVAL, "split RRQR needs istate/dstate");
    maxFill = std::max(maxFill, p.n - p.partition);
    maxCols = std::max(maxCols, std::min(p.m, p.n));
  }
  AIFMM_REQUIRE(probs.size() <= 65535, AIFMM_EINVAL, "too many RRQR problems in one launch");
  // partition-2 steps to launch: at most fillInRank commits plus the step that
  // stops, at most p2cap steps, at most min(m, n) positions
  int p2steps = 0;
  for (const RRQRProblem& p : probs) {
    long t = (long)p.fillInRank + 1;
    if (p.p2cap >= 0) t = std::min<long>(t, p.p2cap);
    t = std::min<long>(t, std::min(p.m, p.n));
    p2steps = std::max(p2steps, (int)std::max<long>(t, 0));
  }
  DevBuf dp = upload(ctx, probs);
  const unsigned np = (unsigned)probs.size();
  if (np <= (unsigned)kRRQRFusedMax && p2steps <= kRRQRStepLaunchMax) {  // one cooperative launch
    // resident CTAs of the fused kernel per SM (a property of the kernel and the architecture)
    static const int maxPerSM = [] {
      int v = 0;
      AIFMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, rrqr_fused_kernel, QR_NT, 0));
      return v;
    }();
    const int sms = ctx->numSMs > 0 ? ctx->numSMs : 148;
    const int resident = sms * maxPerSM;
    if (maxPerSM > 0 && (int)np <= resident) {
      // one warp per column: CTAs by column count, scaled down together to what is resident at once
      std::vector<int> want(np);
      long total = 0;
      for (unsigned p = 0; p < np; ++p) {
        want[p] = std::max((probs[p].n + QR_NT / 32 - 1) / (QR_NT / 32), 1);
        total += want[p];
      }
      RRQRFusedLayout lay{};
      lay.np = (int)np;
      int grid = 0;
      for (unsigned p = 0; p < np; ++p) {
        int g = want[p];
        if (total > resident) g = std::max(1, (int)((long)want[p] * (resident - (long)np) / total));
        lay.start[p] = grid;
        grid += g;
      }
      lay.start[np] = grid;
      AIFMM_REQUIRE(grid <= resident, AIFMM_EINVAL, "fused RRQR grid exceeds the resident CTAs");
      DevBuf sync(ctx, 16);
      AIFMM_CUDA(cudaMemsetAsync(sync.p, 0, 16, ctx->stream));
      const RRQRProblem* pp = dp.as<RRQRProblem>();
      unsigned* bar = sync.as<unsigned>();
      int* err = reinterpret_cast<int*>(sync.as<unsigned>() + 1);
      int steps = p2steps;
      void* args[] = {(void*)&pp, (void*)&lay, (void*)&steps, (void*)&bar, (void*)&err};
      AIFMM_CUDA(cudaLaunchCooperativeKernel((const void*)rrqr_fused_kernel, dim3(grid), dim3(QR_NT), args, 0,
                                             ctx->stream));
      AIFMM_LAUNCHED();
      return;
    }
  }
  rrqr_p1_kernel<<<np, QR_NT, 0, ctx->stream>>>(dp.as<RRQRProblem>());
  AIFMM_LAUNCHED();
  rrqr_fill_kernel<<<dim3((maxFill + 7) / 8, np), 256, 0, ctx->stream>>>(dp.as<RRQRProblem>());
  AIFMM_LAUNCHED();
  if (p2steps <= kRRQRStepLaunchMax) {
    // one launch pair per step: the column updates spread over the GPU
    int maxApply = 1;
    for (const RRQRProblem& p : probs) maxApply = std::max(maxApply, p.n);
    rrqr_p2_init_kernel<<<np, 256, 0, ctx->stream>>>(dp.as<RRQRProblem>());
    AIFMM_LAUNCHED();
    for (int t = 0; t < p2steps; ++t) {
      rrqr_p2_pivot_kernel<<<np, QR_NT, 0, ctx->stream>>>(dp.as<RRQRProblem>(), t);
      AIFMM_LAUNCHED();
      rrqr_p2_apply_kernel<<<dim3((maxApply + 7) / 8, np), 256, 0, ctx->stream>>>(dp.as<RRQRProblem>());
      AIFMM_LAUNCHED();
    }
    rrqr_p2_finish_kernel<<<np, 32, 0, ctx->stream>>>(dp.as<RRQRProblem>());
    AIFMM_LAUNCHED();
  } else {
    rrqr_p2_kernel<<<np, QR_NT, 0, ctx->stream>>>(dp.as<RRQRProblem>());
    AIFMM_LAUNCHED();
  }
  rrqr_q_kernel<<<dim3((maxCols + 7) / 8, np), 256, 0, ctx->stream>>>(dp.as<RRQRProblem>());
  AIFMM_LAUNCHED();
}

}  // namespace aifmm
