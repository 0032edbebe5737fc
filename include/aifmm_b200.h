/*
 * aifmm_b200.h -- C ABI of the B200 AIFMM library (libaifmm_b200.so).
 *
 * The library implements the hot path of the vaishna77/RCS AIFMM direct
 * solver on one NVIDIA B200: Green's-function matrix-entry assembly (EFIE
 * with RWG basis functions, and piecewise-constant electrostatics), ACA
 * skeletonisation with RRQR recompression, the level-by-level hierarchical
 * elimination and the forward/backward solve sweeps.  The C++ drop-in
 * classes (AIFMM<K>, FMM2DTree<K>, EFIEMatrix, ...) and the Python package
 * are thin callers of these entry points.
 *
 * Conventions
 *   - Every function returns an int status: AIFMM_OK (0) or a negative
 *     AIFMM_E* code; aifmm_last_error() describes the last failure of the
 *     calling thread.
 *   - Complex numbers are interleaved (re, im) doubles; matrices are
 *     column-major with a leading dimension ld >= rows.
 *   - Unknown ids are zero-based; triangle vertex ids are ONE-based, as in the
 *     reference's patchList files (src/EFIEMatrix.cpp:72-95).
 *   - Host pointers unless the name ends in _device.  A context owns all
 *     device memory and one CUDA stream; calls on one context must not
 *     overlap (they are not re-entrant).
 */
#ifndef AIFMM_B200_H
#define AIFMM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define AIFMM_OK 0
#define AIFMM_EINVAL (-1)    /* bad argument */
#define AIFMM_ECUDA (-2)     /* CUDA runtime error */
#define AIFMM_ENOMEM (-3)    /* device or host allocation failed */
#define AIFMM_ETIMEOUT (-4)  /* a bounded device wait gave up */
#define AIFMM_ESTATE (-5)    /* call out of order (e.g. solve before factorize) */
#define AIFMM_ESINGULAR (-6) /* exactly singular pivot met */
#define AIFMM_ENOTIMPL (-7)  /* feature not available in this library */
#define AIFMM_EOVERFLOW (-8) /* a workspace bound was exceeded */

typedef struct aifmm_ctx aifmm_ctx;
typedef struct aifmm_kernel aifmm_kernel;
typedef struct aifmm_solver aifmm_solver;

/* ---- context ------------------------------------------------------------ */
/* Message of the last failed call on the calling thread. */
const char* aifmm_last_error(void);
int aifmm_ctx_create(int device, aifmm_ctx** out);
int aifmm_ctx_destroy(aifmm_ctx* ctx);
int aifmm_ctx_synchronize(aifmm_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time or
 * overlap work on it. */
int aifmm_ctx_stream(aifmm_ctx* ctx, void** stream);
/* The GEMM autotuner's trials on this context (GEMM precision 5; no
 * counterpart in the reference): one line per launch class with each
 * candidate kernel's time and the choice, NUL-terminated into buf (cap
 * bytes); *len = the report's full length.  The environment variable
 * AIFMM_TUNE_FILE names a file that stores the choices across runs. */
int aifmm_ctx_tune_report(aifmm_ctx* ctx, char* buf, int cap, int* len);
/* Fixes the operand form (0 packed real, 1 split planes: the default) and
 * tile order (0 row-major: the default, 1 column-major) of GEMM precision 4
 * on this context, the autotuner's knobs (no counterpart in the reference). */
int aifmm_ctx_set_gemm_tiling(aifmm_ctx* ctx, int form, int raster);
/* Device memory of the context: *live = bytes of the buffers its objects
 * hold, *reserved = bytes its memory pool holds from the device (live
 * buffers, the arena's chunks and freed blocks kept for reuse).  Either
 * pointer may be NULL. */
int aifmm_ctx_memory(aifmm_ctx* ctx, size_t* live, size_t* reserved);
/* Waits for the context's stream, then returns to the device the arena
 * chunks that hold no buffer and the blocks its pool keeps for reuse, so
 * that other contexts on the device can use them (a batch of bodies trims
 * each body's context after its factorization and after its solve). */
int aifmm_ctx_trim(aifmm_ctx* ctx);

/* ---- matrix-entry kernels ------------------------------------------------ */
/* EFIE kernel over a flat-triangle mesh: replaces
 * EFIEMatrix::EFIEMatrix(inputsToKernelClass) (src/EFIEMatrix.cpp:5-20) --
 * the RWG unknowns are numbered in the reference's std::map order of
 * (min node, max node) edge keys; "+" triangle = first patch in file order.
 * nodes: n_nodes x 3; tris: n_tris x 3 one-based ids; freq in Hz (the
 * reference hard-codes 1e7, include/includes.hpp:58). */
int aifmm_kernel_create_efie(aifmm_ctx* ctx, const double* nodes, int n_nodes, const int* tris, int n_tris,
                             double freq, aifmm_kernel** out);
/* Electrostatics kernel (collocation at centroids, piecewise-constant
 * charge): replaces ElectrostaticsMatrix::ElectrostaticsMatrix
 * (src/ElectrostaticsMatrix.cpp:48-52).  cond may be NULL (all 1). */
int aifmm_kernel_create_es(aifmm_ctx* ctx, const double* nodes, int n_nodes, const int* tris, const int* cond,
                           int n_tris, aifmm_kernel** out);
int aifmm_kernel_destroy(aifmm_kernel* k);
/* EFIE only: 0 (default) keeps the reference's projection of the test point
 * onto the source triangle's normal plane through the ORIGIN
 * (findProjectionOnTriangle, src/EFIEMatrix.cpp:457-476); 1 projects onto the
 * triangle's own plane, which makes the RCS of a sphere match the Mie series.
 * No counterpart in the reference beyond that one function. */
int aifmm_kernel_set_plane_projection(aifmm_kernel* k, int on);
/* kernel::N -- number of unknowns (EFIEMatrix::getSizeOfMatrix, :97-99). */
int aifmm_kernel_size(const aifmm_kernel* k, int* n);
/* Unknown locations, n x 3: RWG-edge midpoints (EFIE; as the driver builds
 * them, test/sphere.cpp:143-152) or triangle centroids (electrostatics,
 * ElectrostaticsMatrix::getCentroids, :82-88). */
int aifmm_kernel_locations(const aifmm_kernel* k, double* xyz);
/* Dense block of entries K(rows[a], cols[b]) into out (nr x nc, leading
 * dimension ld): replaces kernel::getMatrix(row_indices, col_indices)
 * (src/kernel.cpp:49-61), and with nr==1 / nc==1 kernel::getRow / getCol
 * (:11-29).  precision 0 = complex128 output, 1 = complex64 output (out is
 * then interleaved floats). */
int aifmm_kernel_matrix(aifmm_kernel* k, const int* rows, int nr, const int* cols, int nc, int precision,
                        void* out, int ld);
/* Same with device pointers, asynchronous on the context stream. */
int aifmm_kernel_matrix_device(aifmm_kernel* k, const int* rows_device, int nr, const int* cols_device, int nc,
                               int precision, void* out_device, int ld);
/* EFIE right-hand side exactly as EFIEMatrix::getRhs (src/EFIEMatrix.cpp:785-829),
 * including its phase quirk (exp(i z) for the default incidence). */
int aifmm_kernel_rhs_reference(aifmm_kernel* k, const double einc[3], double* out);
/* Physical plane wave E0 exp(-i kappa khat.r), khat = propagation direction,
 * e0 = complex polarisation (6 doubles), sampled at the triangle centroids. */
int aifmm_kernel_rhs_plane(aifmm_kernel* k, const double khat[3], const double e0[6], double* out);
/* Electrostatics right-hand side: 1 V on the triangles of one conductor
 * (ElectrostaticsMatrix::getRhs, :374-381). */
int aifmm_kernel_rhs_conductor(aifmm_kernel* k, int conductor, double* out);

/* Surface current at the triangle centroids of an EFIE solution, as
 * EFIEMatrix::getJAtCentroids (src/EFIEMatrix.cpp:1100-1130): coeff holds the
 * n RWG coefficients (complex), J receives n_tris x 3 complex values,
 * column-major (the reference's MatrixXcd JAtCentroids). */
int aifmm_kernel_currents(aifmm_kernel* k, const double* coeff, double* J);
/* Bistatic radar cross-section of centroid currents J (n_tris x 3 complex,
 * column-major) at n_angles observation directions (theta[a], phi[a]) by the
 * one-point rule of EFIEMatrix::getRCS_OnePointQuadrature (:916-930), with the
 * kernel's wavenumber; rcs receives n_angles values. */
int aifmm_kernel_rcs(aifmm_kernel* k, const double* J, int n_angles, const double* theta, const double* phi,
                     double* rcs);

/* ---- low-rank and dense components ----------------------------------------- */
/* Partially pivoted ACA of K(rows, cols): replaces
 * LowRank<K>::ACA_only_nodes2(row_bases, col_bases, rank, Ac, Ar)
 * (src/ACA.cpp:639-859).  row_bases/col_bases receive up to min(nr, nc)
 * indices into rows/cols; Ac (nr x rank) holds the original columns and Ar
 * (rank x nc, leading dimension rank) the original rows; both buffers must
 * hold min(nr, nc) columns/rows. */
int aifmm_aca(aifmm_kernel* k, const int* rows, int nr, const int* cols, int nc, double tol, int* row_bases,
              int* col_bases, int* rank, double* Ac, double* Ar);
/* RRQR(A, TOL_POW1, TOL_POW2, partition, inputPivot, flag, fillInRank)
 * .colPivHouseholderQRWithPartition() (src/rrqr.cpp:3-182): Q_trunc
 * (m x rank, buffer of m x min(m, n) complex) and maxPivot.  real_mode 1
 * selects the real Householder sign of a USE_DOUBLE build. */
int aifmm_rrqr(aifmm_ctx* ctx, const double* A, int m, int n, int partition, int tol_pow1, int tol_pow2,
               double input_pivot, int fill_rank, int real_mode, double* Q, int* rank, double* max_pivot);
/* The same RRQR with its other outputs, for RRQR::R_trunc and RRQR::P
 * (include/rrqr.hpp:5-27): R (rank x n complex, leading dimension rank; a
 * buffer of min(m, n) x n) receives R_trunc = Q_trunc^H A P, upper trapezoidal,
 * and perm (n ints) the column order of A P: column q of A P is column perm[q]
 * of A.  The first rank entries of perm are the reference's pivots; the order
 * of the remaining columns differs, because the reference re-sorts them at
 * every step while this kernel swaps the pivot into place. */
int aifmm_rrqr_full(aifmm_ctx* ctx, const double* A, int m, int n, int partition, int tol_pow1, int tol_pow2,
                    double input_pivot, int fill_rank, int real_mode, double* Q, double* R, int* perm, int* rank,
                    double* max_pivot);
/* The same RRQR for callers that cannot allocate device memory (code running
 * inside another framework's allocator, during stream capture, or under a
 * pre-reserved memory budget).  No counterpart in the reference.  Every
 * argument is a device pointer: A (m x n complex128, column-major, not
 * modified), Q (m x min(m, n) complex128; its first *rank columns receive
 * Q_trunc), rank (one int) and max_pivot (one double).  Work is enqueued on
 * `stream` (a cudaStream_t; NULL = legacy default stream) and is complete when
 * the stream is.  The call allocates nothing: its working storage is a fixed
 * 32 MiB device array of the library (held by every GPU that loads it), so
 * problems with 16 (m n + m (min(m, n) + 1)) + 12 n + 1024 bytes above 32 MiB
 * are rejected with AIFMM_EOVERFLOW.  The first call on a device looks up that
 * array's address and must come before any stream capture.  All calls share
 * the array: calls that overlap on the GPU race. */
int aifmm_rrqr_noalloc(const void* A_device, int m, int n, int partition, int tol_pow1, int tol_pow2,
                       double input_pivot, int fill_rank, int real_mode, void* Q_device, int* rank_device,
                       double* max_pivot_device, void* stream);
/* C = alpha op(A) op(B) + beta C (complex128 host arrays, column-major;
 * op: 0 none, 1 conjugate transpose) through the solver's grouped GEMM:
 * precision 0 = FP64 FMA; 1 and 2 = split-TF32 tensor cores with FP32
 * accumulation (FP32 accuracy): 1 by warp-level mma.sync, 2 by tcgen05 with
 * tensor-memory accumulators, 3 by tcgen05 over operands split once into
 * pre-tiled planes streamed with bulk copies, 4 by the persistent,
 * warp-specialised tcgen05 kernel over the real form of the complex product
 * (128 x 128 complex tiles), 5 by the autotuner's choice among 3 and 4.  The dense products of the reference go through Eigen;
 * this is the kernel that replaces them on the GPU. */
int aifmm_zgemm(aifmm_ctx* ctx, int precision, int opA, int opB, int m, int n, int k, const double alpha[2],
                const double* A, int lda, const double* B, int ldb, const double beta[2], double* C, int ldc);
/* Same with device pointers, asynchronous on the context stream. */
int aifmm_zgemm_device(aifmm_ctx* ctx, int precision, int opA, int opB, int m, int n, int k, const double alpha[2],
                       const void* A_device, int lda, const void* B_device, int ldb, const double beta[2],
                       void* C_device, int ldc);
/* X = A^{-1} B by partial-pivot LU (Eigen PartialPivLU semantics, as in
 * EFIEMatrix::getCoefficients, src/EFIEMatrix.cpp:831-837). */
int aifmm_lu_solve(aifmm_ctx* ctx, const double* A, int n, const double* B, int nrhs, double* X);

/* ---- AIFMM solver ----------------------------------------------------------- */
typedef struct {
  int leaf_size;   /* inputsToSolverClass::leafSize (include/includes.hpp:73-77) */
  int tol_pow;     /* TOL_POW: ACA tolerance 10^-tol_pow, RRQR partition-1 tolerance */
  int fillin_tol;  /* RRQR partition-2 tolerance 10^-fillin_tol */
  int fillin_rank; /* accepted for compatibility; the reference's active path ignores it */
  int n_levels;    /* 0 = the reference's rule max(2, floor(log8(N / leaf))) */
  int precision;   /* 0 = plain complex128 (the reference's arithmetic); 1 = mixed:
                    * the elimination's Schur-complement products run on the
                    * tensor cores in split TF32 with FP32 accumulation (about
                    * 1e-5 relative at K = 2048) while the box LU factors, RRQR,
                    * pivots, norms and solves stay FP64 -- a preconditioner for
                    * aifmm_solver_solve_gmres; 2 = the same with the tcgen05
                    * kernel (tensor-memory accumulators) instead of mma.sync;
                    * 3 = tcgen05 over operands split once into pre-tiled planes;
                    * 4 = the persistent, warp-specialised tcgen05 GEMM over
                    * pre-tiled planes of the real form [Ar Ai][[Br Bi][-Bi Br]]
                    * (128 x 128 complex tiles, double-buffered accumulators);
                    * 5 = the tensor-core kernel and tile order chosen per
                    * launch class by the library's autotuner (3 or 4; see
                    * aifmm_ctx_tune_report) */
  int exact_rrqr;  /* 1 = run every recompression RRQR through the full partition-1
                    * Householder pass, as the reference does; 0 (default) skips
                    * that pass when the old basis is one this solver produced with
                    * orthonormal columns: its partition 1 then keeps every column,
                    * so only the fill-in's component outside the old span is
                    * factorized (same ranks and spans, different rounding) */
  int drop_pow;    /* fill-in queue threshold of the factorization used as a
                    * preconditioner: a well-separated fill-in whose norm relative
                    * to its M2L block is at most 10^-drop_pow is dropped instead
                    * of recompressed into the bases.  0 (default) = the
                    * reference's threshold 10^-tol_pow (T:4413, T:4450); a
                    * negative value drops every such fill-in. */
} aifmm_solver_params;

typedef struct {
  int n, n_levels, start_level, avg_leaf_size, avg_multipoles, max_rank;
  long n_rrqr, n_compress_p2p, n_compress_p2l, n_aca, n_aca_retry, kernels;
  double t_assemble, t_factor, t_solve; /* seconds, wall clock on the host thread */
  double flops_factor;                  /* algorithmic flops of the factorization (complex counted) */
  double mem_gb, mem_after_gb;          /* findMemory / findMemoryAfterFactorize */
  /* Factorization phase seconds: RRQR calls, fill-in recompressions (RRQR
   * included), eliminate_x, eliminate_z, non-leaf P2P assembly.  Exact when the
   * environment variable AIFMM_PHASE_TIMES=1 was set at solver creation (the
   * solver then synchronises at every phase boundary), else host-side
   * approximations. */
  double t_rrqr, t_compress, t_elim_x, t_elim_z, t_nonleaf;
  /* inside eliminate_x/z: box LU factorizations, their multi-column solves,
   * the Schur-complement GEMM launches */
  double t_lu, t_msolve, t_schur;
  /* ACA phase of the build: host seconds, workspace bytes allocated over all
   * launches (reruns included), number of launches */
  double t_aca, aca_ws_bytes;
  long n_aca_launches;
  /* solves replayed from a captured CUDA graph of the solve sweep, and
   * graphs captured (one per factorization and right-hand-side count) */
  long n_solve_graph, n_solve_capture;
} aifmm_solver_info;

/* AIFMM<K>::AIFMM(inputsToSolverClass, K*) (src/AIFMM.cpp:7-93): builds the
 * octree over the kernel's unknown locations, the ACA skeletons of every box
 * (getNodes), the L2P/P2M operators, the M2L blocks and the leaf P2P blocks,
 * all resident in device memory. */
int aifmm_solver_create(aifmm_kernel* k, const aifmm_solver_params* p, aifmm_solver** out);
/* The same with the tree built over caller-given unknown locations (xyz,
 * n x 3 row-major, n = the kernel's size) inside the box domain = {xmin, xmax,
 * ymin, ymax, zmin, zmax} (NULL: the locations' bounding box), as
 * inputsToSolverClass::locations and xmin..zmax (include/includes.hpp:73-77)
 * feed FMM2DTree's constructor.  The box must contain every location. */
int aifmm_solver_create_at(aifmm_kernel* k, const aifmm_solver_params* p, const double* xyz, int n,
                           const double domain[6], aifmm_solver** out);
/* The tree order of the unknowns: order[p] = the unknown at position p of the
 * leaf-by-leaf vector that FMM2DTree::getx assembles before reorder
 * (T:4874-4907, T:466-476 of the tree header). */
int aifmm_solver_tree_order(aifmm_solver* s, int* order);
/* AIFMM<K>::factorize() -> eliminate_phase_efficient (src/AIFMM.cpp:96-100). */
int aifmm_solver_factorize(aifmm_solver* s);
/* backSubstitute1/2/3 + getPhi (src/AIFMM.cpp:120-147) for nrhs right-hand
 * sides at once: rhs and x are n x nrhs column-major complex host arrays. */
int aifmm_solver_solve(aifmm_solver* s, const double* rhs, int nrhs, double* x);
/* Same with device pointers (complex128, n x nrhs, ld = n). */
int aifmm_solver_solve_device(aifmm_solver* s, const void* rhs_device, int nrhs, void* x_device);
/* on = 1 (the default): the first solve for a right-hand-side count after a
 * factorization captures the whole solve sweep as a CUDA graph, and solves
 * replay it (same kernels, same results, one launch from the host); on = 0:
 * every solve issues its kernels one by one.  The per-launch profilers of
 * this library turn replays off while they run. */
int aifmm_solver_set_graph_solve(aifmm_solver* s, int on);
/* Tree statistics and phase timings (getAvgLeafSize, getAvgMultipoles,
 * findMemory*, T:490-552 and T:4511-4571 of the tree header). */
int aifmm_solver_get_info(aifmm_solver* s, aifmm_solver_info* info);
int aifmm_solver_destroy(aifmm_solver* s);
/* Keep a device copy of the assembled, not yet factorized operator
 * (checkpoint) and restore it (rewind) so that factorize() can run again on
 * the same blocks, e.g. to time repeated factorizations.  No counterpart in
 * the reference, whose tree can be factorized only once. */
int aifmm_solver_checkpoint(aifmm_solver* s);
int aifmm_solver_rewind(aifmm_solver* s);
/* One record of 7 doubles per block of the tree -- level, box, kind, key,
 * rows, cols, Frobenius norm -- for comparing two solvers' states; kinds:
 * 0 L2P, 1 P2M, 2 M2L, 3 P2P, 4 M2P, 5 P2L, 6 L2P_f, 7 P2M_f, 8 M2M_f, 9 L2M_f.
 * Writes at most cap records; *count receives the total. */
int aifmm_solver_dump(aifmm_solver* s, double* out, long cap, long* count);
/* Factorization checkpoint file (no counterpart call in the reference, whose
 * factors live only in memory: FMM2DTree's per-box blocks,
 * include/AIFMMBox.hpp:13-71).  save writes a factorized solver -- tree,
 * index lists, every block and the base-level LU -- to path; load reads one
 * into a new solver on kernel k (same unknown count), ready for
 * aifmm_solver_solve* without assembly or factorization.  A loaded solver
 * cannot refactorize (the assembled operator is not in the file). */
int aifmm_solver_save(aifmm_solver* s, const char* path);
int aifmm_solver_load(aifmm_kernel* k, const char* path, aifmm_solver** out);

/* ---- forward operator and FP64 refinement ----------------------------------- */
/* No counterpart in the reference, which factorizes its tree directly and
 * measures the backward error with a dense product (test/sphere.cpp:331-338).
 * The H^2 forward operator y = A x of the kernel: the assembly of
 * aifmm_solver_create (octree, ACA skeletons, L2P/P2M, M2L, leaf P2P) run with
 * p->tol_pow as the operator's ACA tolerance and kept unfactorized; applied
 * upward (P2M), across (M2L) and downward (L2P) plus the leaf near field.  Used
 * as the residual operator of aifmm_solver_solve_gmres, so its tolerance should
 * be tighter than the factorization's. */
typedef struct aifmm_operator aifmm_operator;
int aifmm_operator_create(aifmm_kernel* k, const aifmm_solver_params* p, aifmm_operator** out);
/* y = A x, n x nrhs column-major complex host arrays. */
int aifmm_operator_apply(aifmm_operator* op, const double* x, int nrhs, double* y);
/* Same with device pointers (complex128, n x nrhs, ld = n). */
int aifmm_operator_apply_device(aifmm_operator* op, const void* x_device, int nrhs, void* y_device);
/* Device bytes of the operator's blocks and complex-counted flops of one column. */
int aifmm_operator_info(aifmm_operator* op, double* bytes, double* flops_per_column);
int aifmm_operator_destroy(aifmm_operator* op);

typedef struct {
  int iterations;    /* Arnoldi steps: one preconditioner solve and one product each */
  int cycles;        /* restarts + 1 */
  double relres;     /* max over columns of ||b - A x|| / ||b||, A = the operator */
  double t_precond;  /* seconds in preconditioner solves */
  double t_matvec;   /* seconds in operator products */
} aifmm_gmres_info;
/* Flexible GMRES(restart) for A x = b, right-preconditioned by the factorized
 * solver s (its solve sweeps), until relres <= tol or maxit Arnoldi steps.
 * s and A must come from the same context and kernel. */
int aifmm_solver_solve_gmres(aifmm_solver* s, aifmm_operator* A, const double* rhs, int nrhs, double* x, double tol,
                             int restart, int maxit, aifmm_gmres_info* info);
/* Same with device pointers (complex128, n x nrhs, ld = n). */
int aifmm_solver_solve_gmres_device(aifmm_solver* s, aifmm_operator* A, const void* rhs_device, int nrhs,
                                    void* x_device, double tol, int restart, int maxit, aifmm_gmres_info* info);

/* ---- batches of independent bodies (no counterpart call in the reference,
 * whose driver solves one geometry per process, test/sphere.cpp) ---------- */
/* Factorizes n solvers concurrently: up to `threads` host threads (<= 0: 16)
 * each drive one body's AIFMM::factorize() at a time.  Every solver must be
 * on its own context, so that the bodies' streams overlap on the GPU.  Each
 * body's result is bit-identical to aifmm_solver_factorize on it alone.
 * seconds (may be NULL): wall time of the whole batch.  The first failing
 * body's status is returned; the others still complete. */
int aifmm_batch_factorize(aifmm_solver* const* solvers, int n, int threads, double* seconds);
/* FGMRES of every body as aifmm_solver_solve_gmres (host arrays rhs[i], x[i]
 * of N_i x nrhs[i]), concurrently on the bodies' streams; info: n records
 * (may be NULL). */
int aifmm_batch_solve_gmres(aifmm_solver* const* solvers, aifmm_operator* const* ops, const double* const* rhs,
                            const int* nrhs, double* const* x, int n, double tol, int restart, int maxit, int threads,
                            aifmm_gmres_info* info, double* seconds);

/* ---- Learned rank prediction (no counterpart in the reference) ----
 * A 6 -> 64 -> 64 -> 1 perceptron (ReLU) with BF16 weights, FP32 activations
 * and FP32 accumulation that predicts log2(1 + rank) of a box's ACA skeleton
 * (LowRank::ACA_only_nodes2, src/ACA.cpp:639-859) from six features: mean
 * centre distance to the interaction-list boxes over the box side,
 * wavenumber times the box side, log2(1 + rows), log2(1 + columns), tree
 * level, leaf flag.  Training and inference run as this library's own CUDA
 * kernels.  Parameter layout (aifmm_mlp_num_params floats): W1 [64 x 6]
 * row-major, b1 [64], W2 [64 x 64] row-major (output, input), b2 [64],
 * w3 [64], b3. */
typedef struct aifmm_mlp aifmm_mlp;
int aifmm_mlp_num_params(int* n);
/* Seeded He initialisation, zero biases, identity normalisation. */
int aifmm_mlp_create(aifmm_ctx* ctx, unsigned long long seed, aifmm_mlp** out);
int aifmm_mlp_destroy(aifmm_mlp* m);
/* Inputs are normalised on the device as (x - mean) * scale (6 floats each). */
int aifmm_mlp_set_normalization(aifmm_mlp* m, const float* mean, const float* scale);
int aifmm_mlp_get_params(aifmm_mlp* m, float* params);
int aifmm_mlp_set_params(aifmm_mlp* m, const float* params);
/* y[i] = prediction for the raw features X[6 i .. 6 i + 5]. */
int aifmm_mlp_infer(aifmm_mlp* m, const float* X, int n, float* y);
/* Gradient of the mean squared error (1/n) sum (y_i - t_i)^2 at the current
 * parameters (the BF16 rounding of the FP32 master weights), and the loss. */
int aifmm_mlp_grad(aifmm_mlp* m, const float* X, const float* t, int n, float* grad, float* loss);
/* Full-batch Adam (lr, beta 0.9 / 0.999) on the mean squared error for
 * `epochs` steps; loss_first / loss_last: the loss before the first and the
 * last step (either may be NULL). */
int aifmm_mlp_train(aifmm_mlp* m, const float* X, const float* t, int n, int epochs, float lr, float* loss_first,
                    float* loss_last);
/* Solvers created on ctx afterwards size each box's ACA workspace from the
 * model's prediction times `margin` (plus 8 terms) instead of the fixed
 * bound of 128; a box whose ACA needs more terms is rerun with twice the
 * bound, so the ranks are the plain ACA's either way.  The context keeps a
 * copy of the model; m = NULL restores the fixed bound. */
int aifmm_ctx_set_rank_model(aifmm_ctx* ctx, const aifmm_mlp* m, double margin);
/* The ACA problems of the solver's build, in launch order: raw features
 * (n x 6 floats), the rank bound each was first launched with, and the
 * rank the ACA found.  *n receives the count; at most cap records are
 * written. */
int aifmm_solver_aca_log(aifmm_solver* s, float* features, int* rmax0, int* ranks, int cap, int* n);

/* Per-operation accounting of the solver's host-driven factorization and
 * solve (diagnosis only): on = 1 clears and starts it -- every accounted
 * operation then synchronises the stream when it ends -- and on = 0 stops it.
 * The report is text, one line per operation: name, calls, seconds; it is
 * truncated to cap bytes. */
int aifmm_profile_ops(int on);
int aifmm_profile_ops_read(char* buf, int cap);
/* Number of tcgen05 GEMM tiles whose bounded pipeline wait ran out (their
 * output was left unwritten); 0 in a healthy run.  The factorization and the
 * GEMM entry points compare this count before and after their work and
 * return AIFMM_ETIMEOUT when it grew. */
int aifmm_tc5_timeouts(long* n);
/* Test of the bounded waits (no counterpart in the reference): with on = 1,
 * the tensor-core GEMMs of this context first wait, for at most 1 ms, on a
 * device flag that nothing sets, so every tile gives up, writes nothing and
 * the call returns AIFMM_ETIMEOUT with the context still usable; on = 0
 * restores normal operation. */
int aifmm_debug_gemm_hold(aifmm_ctx* ctx, int on);
/* Number of CUDA kernels this library has launched in the process. */
int aifmm_launch_count(long* n);
/* Switch per-launch CUDA-event timing of the grouped complex GEMM on (1) or
 * off (0; also clears the record), and read the accumulated device time (ms),
 * algorithmic flops (8 m n k per complex product) and launch count. */
int aifmm_profile_gemm(int on);
int aifmm_profile_gemm_read(double* ms, double* flops, long* launches);
/* The device-time records of the GEMM profiler (grouped GEMM launches tagged
 * "gemm:<precision>:<scope path>", RRQR launch chains "rrqr:<scope path>") as
 * text lines "tag launches seconds flops", truncated to cap bytes. */
int aifmm_profile_gemm_table(char* buf, int cap);

#ifdef __cplusplus
}
#endif
#endif /* AIFMM_B200_H */
