/*
 * grimgpu.h -- C ABI of the B200 method-of-moments RCS solve path (libgrimgpu.so).
 *
 * Plain C: opaque handles, plain pointers and sizes, integer status codes.  No
 * PyTorch or C++ types cross this boundary.  Matrices are column-major (LAPACK
 * order) with an explicit leading dimension; complex numbers are interleaved
 * (re, im) pairs of double (complex128) or float (complex64).
 *
 * Pointer kinds: functions whose name ends in _host take host memory; every
 * other function takes DEVICE memory of the handle's device and runs on the
 * handle's stream (asynchronously unless stated).
 *
 * Reference interfaces replaced (paths inside tools/GHOST/ghost_backend/):
 *   grim_zgesv_batched   twod/solver.py:355-392  _solve_dense_gpu(a_eval, rhs_eval)
 *                        (the GHOST_DENSE_BACKEND=gpu hook; CuPy cp.linalg.solve there)
 *   grim_zgetrf/zgetrs   linalg/dense.py:114-155,241  DenseFactor (scipy lu_factor / lu_solve)
 *   grim_cgetrf/cgetrs   linalg/refined_lu.py:25-61   RefinedLU complex64 factor
 *   grim_zgesv_mixed     linalg/refined_lu.py:25-61   RefinedLU (complex64 LU + FP64 refinement)
 *   grim_fill2d          twod/operators.py:2087-2607  _assemble_multi (system-matrix fill)
 *   grim_rhs2d           twod/assembly/kernels.py:223-294  incident_loads
 *   grim_farfield2d      twod/assembly/kernels.py:163-219  farfield (matched monostatic)
 *   grim_gal_*           twod/operators.py:2087-2607 _assemble_multi, combined_regions.py:149-204,
 *                        scatter.py:282-368 (linear-Galerkin S + gamma(D + M/2) / K' - M/2 - gamma W fill),
 *                        twod/assembly/kernels.py:223-294 loads, twod/operators.py:2925-3030 far field
 *   grim_backward_error  twod/solver.py:695-720  backward_metrics (normwise backward error)
 *   grim_solution_errors bor/factor.py:289-300  ModalFactor.errors (BoR release measures)
 *   grim_zcond1_factored bor/factor.py:205-229  ModalFactor._condition (zgecon per BoR mode)
 *   grim_bor_*           bor/solver.py:1769-1962,2558-2608  per-mode assembly, excitation, far field
 *   ghost_far_block      twod/assembly/native/far.c:193-207  ghost_far_block (same signature, GPU)
 *   grim_far_block       the same on device pointers
 *
 * Status codes: 0 = success; any other value is an error and grim_last_error()
 * returns a message for the calling thread.
 */
#ifndef GRIMGPU_H
#define GRIMGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GRIM_OK 0
#define GRIM_ERR_ARGUMENT 3      /* same meaning as far.c:193-207's "bad arguments" */
#define GRIM_ERR_CUDA 4
#define GRIM_ERR_NOMEM 5
#define GRIM_ERR_SINGULAR 6
#define GRIM_ERR_NOT_CONVERGED 7
#define GRIM_ERR_NONFINITE 8

#define GRIM_POL_TM 0            /* HH, Dirichlet, EFIE */
#define GRIM_POL_TE 1            /* VV, Neumann, MFIE   */

#define GRIM_PREC_FP64 0         /* plain FP64 drop-in                               */
#define GRIM_PREC_MIXED 1        /* FP32 factor, FP64 residual / update refinement   */
#define GRIM_PREC_MIXED_BERR 2   /* as MIXED, stopping on the normwise backward error */
#define GRIM_PREC_STATIC_PIVOT 8   /* or-ed into a mode: this factorization keeps the
                                      diagonal pivots (no partial-pivoting fallback)  */
#define GRIM_PREC_PARTIAL_PIVOT 16 /* or-ed into a mode: partial pivoting throughout    */
#define GRIM_PREC_TOURNAMENT_PIVOT 32 /* or-ed into a mode: tournament pivoting throughout */
/* Pivot modes of a factorization (grim_set_tuning GRIM_TUNE_PIVOT, grim_zgesv_guarded):
 * CERTIFIED  diagonal pivots, each 64-column panel certified to be what partial pivoting
 *            picks and refactored with partial pivoting when it is not (fast for
 *            diagonally dominant systems: the pulse-basis matrices, the BoR modes);
 * STATIC     diagonal pivots, no fallback (callers guard the solution);
 * PARTIAL    partial pivoting of every panel on a thread-block cluster (the
 *            linear-Galerkin combined-field systems, whose pivots leave the diagonal);
 * TOURNAMENT tournament pivoting of every panel (communication-avoiding LU: each panel's
 *            64 pivot rows chosen by a reduction tree of partial-pivoting selections on
 *            128-row blocks; stable like partial pivoting in practice, other pivots).
 * CERTIFIED and PARTIAL give LAPACK getrf's pivots (|re| + |im|, first row on ties). */
#define GRIM_PIVOT_CERTIFIED 0
#define GRIM_PIVOT_STATIC 1
#define GRIM_PIVOT_PARTIAL 2
#define GRIM_PIVOT_TOURNAMENT 3

typedef struct grim_context *grim_handle_t;

/* Per-solve telemetry (reference: twod/solver.py:226-288 dense-backend events). */
typedef struct grim_solve_info {
    double backward_error;       /* max normwise backward error over columns        */
    double initial_backward_error;
    int refinement_steps;
    int pivoted_panels;          /* panels that needed row interchanges (0 = diagonal pivots certified) */
    int precision_mode;
    int info;                    /* LAPACK-style: >0 = U(info,info) exactly zero      */
    double ms_factor;            /* device time of the factorization                 */
    double ms_solve;             /* device time of the triangular solves + refinement */
} grim_solve_info;

/* ---- context ------------------------------------------------------------------ */
int grim_create(int device, grim_handle_t *out);
int grim_destroy(grim_handle_t h);
/* Run on a caller stream (cudaStream_t passed as void*; NULL = the CUDA default stream).
 * A new handle runs on its own non-blocking stream until this is called. */
int grim_set_stream(grim_handle_t h, void *stream);
void *grim_get_stream(grim_handle_t h);
/* Waits for the handle's stream; also reports (GRIM_ERR_CUDA, then cleared) a bounded wait
 * that ran out in a tensor-core kernel queued without a host check (grim_solution_errors). */
int grim_synchronize(grim_handle_t h);
const char *grim_last_error(void);
int grim_device_name(grim_handle_t h, char *buf, int len);
int grim_version(void);
/* Number of kernel launches this handle has issued (for launch accounting). */
int64_t grim_launch_count(grim_handle_t h);
/* Release the handle's cached device workspace. */
int grim_release_workspace(grim_handle_t h);

/* ---- 2-D pulse-basis fill, excitation, far field --------------------------------
 * geom: 7*n doubles, panel-major: (cx, cy, tx, ty, h, nx, ny) per panel -- midpoint,
 *       unit tangent, half-length, outward unit normal.
 * diag_extra: NULL or n doubles added to the TE diagonal 1/2 (curvature correction).
 * Z is written in full (n x n, leading dimension ldz); out_complex64 selects the
 * complex64 fill (FP32 arithmetic for kR >= 12, FP64 for small kR, self terms and
 * phases) instead of complex128.
 */
int grim_fill2d(grim_handle_t h, int pol, int n, const double *geom, const double *diag_extra,
                double k, void *Z, int64_t ldz, int out_complex64);
/* B[:, a] = TM: -exp(jk d_a.c), TE: -jk (d_a.n) exp(jk d_a.c); d_a = (cos, sin)(angle_deg[a]). */
int grim_rhs2d(grim_handle_t h, int pol, int n, const double *geom, int nang, const double *angles_deg,
               double k, void *B, int64_t ldb, int out_complex64);
/* amp[a] = sum_n X[n, a] * 2h_n exp(jk d_a.c_n) sinc(k (d_a.t_n) h_n)  (complex128 out). */
int grim_farfield2d(grim_handle_t h, int n, const double *geom, int nang, const double *angles_deg,
                    double k, const void *X, int64_t ldx, int x_complex64, void *amp);

/* ---- 2-D linear-Galerkin combined-field fill (the reference's own formulation) ----
 * Replaces twod/operators.py:2087-2607 _assemble_multi with the combined routing of
 * twod/formulations/combined_regions.py:21-62,149-204 and the scatter of
 * twod/assembly/scatter.py:282-368 (closed PEC contours in air, real k).
 * elem: 8*ne doubles per element (ax, ay, bx, by, nx, ny, L, 0): start and end point, unit
 *       normal (-t_y, t_x) of the tangent t = (b - a)/L, length.
 * nodes: 2*ne ints, the element's start and end node.  start_of / end_of: n ints, the
 *       element that starts / ends at each node (-1 for none).
 * Near-pair structure (geometry only, reusable for every k and polarisation):
 *   grim_gal_near_count  row_off (ne + 1 ints, device) = CSR offsets of the pairs that are
 *                        not far (centre distance < 3 max(L), a shared node, or self);
 *                        *nnz_host = row_off[ne] (synchronises the stream);
 *   grim_gal_near_list   col (nnz ints, ascending per row) and route (nnz ints: 0 self,
 *                        1 touching, 2 16-point tensor rule, 3 adaptive bisection).
 * adapt_idx: the nadapt indices (into col / route) of the route-3 pairs, each integrated
 *   by its own CTA.
 * grim_gal_fill writes the n x n node matrix: TM (pol 0) S + gamma (D + M/2), TE (pol 1)
 * K' - M/2 - gamma W, gamma = 1/(j k).  far_min_order: floor on the far Gauss order (the
 * TE rows' W rule: 8, or 16 outside its calibration; 0 for TM).  Near pairs in FP64;
 * out_complex64 stores Z as complex64.  An adaptive pair that did not converge or a
 * failed self series sets a flag that grim_gal_status returns (and clears; synchronises).
 * grim_gal_rhs: B[:, a] = TM -load, TE -(normal-derivative load) of the plane wave
 *   exp(jk d_a.x), d_a = (cos, sin)(angle_deg[a]) (twod/assembly/kernels.py:223-294).
 * grim_gal_farfield: amp[a] = sum_e L_e int (phi_0 x_n0 + phi_1 x_n1) exp(jk d_a.x)
 *   (1 + d_a.n_e) (twod/operators.py:2925-3030 single + gamma double layer). */
int grim_gal_near_count(grim_handle_t h, int ne, const double *elem, const int *nodes, int *row_off,
                        int *nnz_host);
int grim_gal_near_list(grim_handle_t h, int ne, const double *elem, const int *nodes, const int *row_off,
                       int *col, int *route);
int grim_gal_fill(grim_handle_t h, int pol, int ne, int n, const double *elem, const int *nodes,
                  const int *start_of, const int *end_of, const int *row_off, const int *col,
                  const int *route, int nnz, const int *adapt_idx, int nadapt, double k, int far_min_order,
                  void *Z, int64_t ldz, int out_complex64);
int grim_gal_status(grim_handle_t h, int *flag_host);
int grim_gal_rhs(grim_handle_t h, int pol, int n, const double *elem, const int *start_of,
                 const int *end_of, int nang, const double *angles_deg, double k, void *B, int64_t ldb,
                 int out_complex64);
int grim_gal_farfield(grim_handle_t h, int ne, const double *elem, const int *nodes, int nang,
                      const double *angles_deg, double k, const void *X, int64_t ldx, int x_complex64,
                      void *amp);

/* ---- dense LU / solve ------------------------------------------------------------
 * grim_zgetrf / grim_cgetrf: LAPACK getrf semantics (partial pivoting by |re|+|im|,
 * 1-based ipiv, info > 0 for an exactly singular U).  The factorization first
 * eliminates without interchanges and certifies, panel by panel, that partial
 * pivoting would have chosen every diagonal pivot; a panel that fails the
 * certificate is refactored with row interchanges.
 */
int grim_zgetrf(grim_handle_t h, int n, void *A, int64_t lda, int *ipiv, int *info);
int grim_zgetrs(grim_handle_t h, int n, int nrhs, const void *LU, int64_t lda, const int *ipiv,
                void *B, int64_t ldb);
int grim_cgetrf(grim_handle_t h, int n, void *A, int64_t lda, int *ipiv, int *info);
int grim_cgetrs(grim_handle_t h, int n, int nrhs, const void *LU, int64_t lda, const int *ipiv,
                void *B, int64_t ldb);

/* C[MxN] -= A[MxK] B[KxN], complex64 column-major: use_tensor_cores = 1 runs the tcgen05
 * split-TF32 kernel used by grim_cgetrf / grim_cgetrs for their updates, 0 the SIMT kernel
 * (reference: the BLAS zgemm calls inside LAPACK getrf/getrs, linalg/dense.py:139-155). */
int grim_cgemm_sub(grim_handle_t h, int M, int N, int K, const void *A, int64_t lda, const void *B, int64_t ldb,
                   void *C, int64_t ldc, int use_tensor_cores);

/* R = B - A X (complex128 X, B, R; A complex64 if a_complex64 else complex128), the
 * residual of the FP64 refinement (reference linalg/refined_lu.py:50-53, the numpy
 * residual of RefinedLU).  slices = 0: FP64 SIMT GEMM; 6, 7 or 8: int8 slicing of both
 * operands on the tcgen05 integer tensor cores (error per product term below
 * 2^-7s of max|A row| max|X column|; 8 slices match an FP64 GEMM), as used inside
 * grim_zgesv_mixed (backward-error targets: 6 slices for 1e-11 and looser, 7 for 1e-13
 * and looser; relative-residual targets: 8).  R must not
 * overlap B.  Needs n < 2^31 / (2 slices 64^2). */
int grim_residual(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda, int a_complex64, const void *X,
                  int64_t ldx, const void *B, int64_t ldb, void *R, int64_t ldr, int slices);

/* Normwise backward error per column (reference twod/solver.py:695-720):
 * berr[j] = max_i |A x_j - b_j|_i / (||A||_inf max|x_j| + max|b_j|), A complex128 or complex64. */
int grim_backward_error(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda, int a_complex64,
                        const void *X, int64_t ldx, const void *B, int64_t ldb, double *berr_dev);

/* Residual and release measures of a computed solution X of A X = B (reference
 * bor/factor.py:289-300, ModalFactor.errors, used by the BoR per-mode gate of
 * bor/factor.py:302-355): R = B - A X; per column berr[j] = max_i |R_ij| / (||A||_inf
 * max_i |X_ij| + max_i |B_ij|) (inf for a zero denominator under a non-zero residual, or
 * any NaN) and relres[j] = ||R_j||_2 / ||B_j||_2 (||R_j||_2 for a zero column); maxes[0]
 * and maxes[1] = their maxima.  A, X, B, R complex128; berr_dev / relres_dev may be NULL.
 * slices = 0 computes R with the FP64 GEMM, 8 on the integer tensor cores (8 int8 slices:
 * FP64 GEMM accuracy).  No host synchronisation: the tensor-core kernels' error flag is
 * reported by the next grim_synchronize.  R must not overlap B. */
int grim_solution_errors(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda, const void *X, int64_t ldx,
                         const void *B, int64_t ldb, void *R, int64_t ldr, int slices, double *berr_dev,
                         double *relres_dev, double *maxes_dev);

/* Allocation-free grim_backward_error (no counterpart in the reference).  For callers
 * that cannot allocate device memory when they call it (memory owned by another
 * framework's allocator, allocation-free serving loops, FFI callers without a device
 * allocator): same arguments and result as grim_backward_error, but its scratch is one
 * fixed array compiled into the library (about 2.6 MB on every device that loads it,
 * kept until the process exits) instead of handle workspace.  Limits: n <= 1024,
 * nrhs <= 128; larger sizes return GRIM_ERR_ARGUMENT.  Every call looks up the array's
 * device address on the handle's device (so a recreated device context is picked up);
 * the first lookup on a device may load the library's module there, so make the first
 * call on each device before any stream capture on it.  All calls on a device share the
 * array: calls whose GPU work overlaps race and must be serialized by the caller. */
int grim_backward_error_noalloc(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda, int a_complex64,
                                const void *X, int64_t ldx, const void *B, int64_t ldb, double *berr_dev);

/* Device-resident solve of A X = B, X overwrites B (complex128).
 * precision_mode GRIM_PREC_FP64: zgetrf + zgetrs.  GRIM_PREC_MIXED: complex64 LU of A
 * (or of A32 when given), FP64 residual against A (complex128, or the exact promotion
 * of A32 when A is NULL) and FP64 update, at most max_iter steps until the relative
 * residual max|r| / max|b| of every column is <= tol or stalls (ratio > 0.98);
 * reference linalg/refined_lu.py:25-61.  GRIM_PREC_MIXED_BERR: the same refinement
 * stopping when the normwise backward error |r| / (|A| |x| + |b|) of every column is
 * <= tol (the form of test LAPACK's zcgesv uses), for callers whose accuracy target
 * is a backward error (the RCS solves).  A is preserved.  info: LAPACK-style.  stats
 * may be NULL.  GRIM_PREC_STATIC_PIVOT or GRIM_PREC_PARTIAL_PIVOT or-ed into the mode
 * picks the factorization's pivot mode (GRIM_PIVOT_STATIC / GRIM_PIVOT_PARTIAL; the
 * default is CERTIFIED); with static pivots the refinement guards the solution (a stall
 * returns GRIM_ERR_NOT_CONVERGED). */
int grim_zgesv_mixed(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda, const void *A32,
                     int64_t lda32, void *B, int64_t ldb, int precision_mode, double tol, int max_iter,
                     int *info, grim_solve_info *stats);

/* FP64 solve with the reference's backward-error gate (twod/solver.py:694-760): LU in the
 * given pivot mode (GRIM_PIVOT_*), getrs, the per-column normwise backward error
 * |r| / (|A|_inf |x| + |b|) into berr_dev (nrhs doubles, may be NULL), at most max_refine
 * FP64 refinement steps with the same factors while the largest exceeds tol (each kept
 * only if it lowers it), and, when the gate still fails, a CERTIFIED factorization and
 * solve (stats->pivoted_panels = -1 - its pivoted panel count then records the
 * fallback).  X overwrites B; A is preserved; synchronises the stream. */
int grim_zgesv_guarded(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda, void *B, int64_t ldb,
                       int pivot, double tol, int max_refine, double *berr_dev, int *info, grim_solve_info *stats);

/* Condition estimate of A (complex128, preserved): cond_1 of the row/column-equilibrated
 * matrix B = R^-1 A C^-1 (r_i = max_j |a_ij|, c_j = max_i |a_ij| / r_i), ||B||_1 times a
 * Hager-Higham estimate of ||B^-1||_1 (LAPACK zlacn2's iteration on partial-pivoting LUs of
 * A and A^H, at most 11 single-vector solves); *cond on the host, INFINITY for an exactly
 * singular or non-finite A.  Replaces the reference's _equilibrated_condition_from_lu
 * (twod/solver.py:472-577, linalg/dense.py:157-198: the same matrix B, SciPy's block
 * estimator).  Synchronises the stream. */
int grim_zcond1_equilibrated(grim_handle_t h, int n, const void *A, int64_t lda, double *cond);

/* One factored system for grim_zcond1_factored: the full matrix A (complex128, column-major,
 * for ||A||_1) and either its LU (halves = 0: LAPACK layout, lu[0] / ldlu[0]; the row
 * interchanges are not needed) or the LUs of its mirror halves (halves = 1: lu[0] / ipiv[0]
 * of the even half of order k + nfe, lu[1] / ipiv[1] of the odd half of order k + nfo, with
 * 2k + nfe + nfo = n, and the split of grim_bor_mirror_split: pairs p1[k], p2[k] with
 * signs s[k] = +-1, fixed unknowns fe[nfe] / fo[nfo]; every pointer on the device). */
typedef struct grim_cond_system {
    int n;
    const void *A;
    int64_t lda;
    int halves;
    int lu_complex64;  /* bit h set: lu[h] stored in complex64 (else complex128) */
    const void *lu[2];
    int64_t ldlu[2];
    const int *ipiv[2];
    int k, nfe, nfo;
    const int *p1, *p2, *fe, *fo;
    const double *s;
} grim_cond_system;

/* 1-norm condition estimates of already factored systems (reference bor/factor.py:205-229,
 * ModalFactor._condition: LAPACK zgecon on each BoR mode's LU with ||A||_1 of the mode
 * matrix, rcond^-1 = ||A||_1 est(||A^-1||_1)).  The estimate is zgecon's: the zlacn2
 * iteration on inv(U) inv(L) (adjoint inv(L^H) inv(U^H)); a mirror-split system uses the
 * true inverse through its halves.  One CTA per system, all systems in one launch:
 * cond_dev[count] on the device, NaN for a system holding a NaN, INFINITY where zgecon
 * returns rcond = 0 (zero norm or estimate, or overflow).  No host synchronisation. */
int grim_zcond1_factored(grim_handle_t h, int count, const grim_cond_system *systems, double *cond_dev);

/* Mixed solve reusing a complex64 factorization (LU32 and ipiv from grim_cgetrf, leading
 * dimension n) with FP64 refinement against A or the promotion of A32; for resident
 * factor caches (reference linalg/refined_lu.py:41-61 RefinedLU.solve on a kept factor). */
int grim_zgesv_mixed_factored(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda, const void *A32,
                              int64_t lda32, void *LU32, const int *ipiv, void *B, int64_t ldb, double tol,
                              int max_iter, grim_solve_info *stats);

/* grim_zgesv_mixed_factored with the stopping test of grim_zgesv_mixed: precision_mode
 * GRIM_PREC_MIXED (relative residual) or GRIM_PREC_MIXED_BERR (backward error).  Used
 * after grim_getrf_grouped for the systems of a sweep. */
int grim_zgesv_refine_factored(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda, const void *A32,
                               int64_t lda32, void *LU32, const int *ipiv, void *B, int64_t ldb, int precision_mode,
                               double tol, int max_iter, grim_solve_info *stats);

/* Grouped LU of `count` (<= 65535) independent systems of different orders in one
 * sequence of launches: the systems of a frequency sweep or the Fourier modes of a body
 * of revolution, which the reference factors one per worker process
 * (execution/frequency_sweep.py:140-188 _plan / _compute; bor/solver.py:2827-3250
 * _mode_sweep_impl with bor/factor.py:120 ModalFactor per mode).  Each step of 64
 * columns is one launch per stage over all systems (diagonal blocks, panel solves,
 * trailing updates: split-TF32 tcgen05 for complex64, FP64 tensor cores for
 * complex128).  Per system: n[i], device matrix A[i] (lda[i] >= n[i], complex64 if
 * complex64 else complex128, overwritten by L\U with the same certified diagonal-pivot
 * / partial-pivot fallback as grim_cgetrf / grim_zgetrf, identical factors), device
 * pivots ipiv[i] (n[i] ints, 1-based).  use_graph: capture the launch sequence in a
 * CUDA graph, kept on the handle and replayed while the orders (and the handle's
 * buffers) stay the same.  info[i] (host): 0, or k+1 when U(k,k) is exactly zero;
 * pivoted[i] (host, may be NULL): panels that fell back to partial pivoting.  Blocks
 * until done. */
int grim_getrf_grouped(grim_handle_t h, int count, const int *n, void *const *A, const int64_t *lda,
                       int *const *ipiv, int complex64, int use_graph, int *info, int *pivoted);

/* ---- linear-Galerkin far-field element-pair blocks (boundary B2) -------------------
 * Replaces twod/assembly/native/far.c:100-207 ghost_far_block, the native far pass of
 * the reference's Galerkin fill (twod/operators.py:2447-2458 _far_tile calls it through
 * twod/assembly/native/far.py:184-249 far_block).  For every pair (i, j) with far[i*nb+j]
 * != 0: acc[(width*a + b), i, j] += sum_qi qw[qi] phi[qi,a] sum_qj qw[qj] phi[qj,b] K(r),
 * K = G (acc_s), the normal derivative (acc_k) and, if mirrored, the transposed-normal
 * kernel (acc_kt), all interleaved complex128 of shape (width^2, mb, nb); G and dG from
 * the caller's kernel table (bounds[intervals+1], coeff[intervals][degree+1][2] complex
 * normalized power coefficients) or, beyond it, the large-argument Hankel expansion.
 * Same arithmetic and order as the reference (no fused multiply-add): pairs inside the
 * table get bitwise the reference's sums.  Status: 0; 2 when a distance falls below the
 * table (the caller's fallback case; accumulators then undefined); 3 on bad arguments
 * (far.c:114-117); other codes: GRIM_ERR_*.
 *
 * ghost_far_block: HOST buffers and the exact signature of the reference's export, so
 * the reference's far.py can load this library in place of libghost_far.so; each calling
 * thread gets its own device handle on the current device (kept until process exit). */
int ghost_far_block(int64_t mb, int64_t nb, int q, int width, const double *obs_pts, const double *src_pts,
                    const double *qw, const double *phi, const double *obs_norm, const double *src_norm,
                    const uint8_t *far, int obs_normal_deriv, int want_s, int want_k, int mirrored, double k_re,
                    double k_im, int intervals, const double *bounds, int degree, const double *coeff, double *acc_s,
                    double *acc_k, double *acc_kt);
/* grim_far_block: the same on DEVICE pointers, on the handle's stream (blocks until done). */
int grim_far_block(grim_handle_t h, int64_t mb, int64_t nb, int q, int width, const double *obs_pts,
                   const double *src_pts, const double *qw, const double *phi, const double *obs_norm,
                   const double *src_norm, const uint8_t *far, int obs_normal_deriv, int want_s, int want_k,
                   int mirrored, double k_re, double k_im, int intervals, const double *bounds, int degree,
                   const double *coeff, double *acc_s, double *acc_k, double *acc_kt);

/* B1 drop-in (host buffers): solve A X = B for all nrhs columns, X overwrites B.
 * A: n x n complex128 column-major (lda >= n), B: n x nrhs complex128 (ldb >= n).
 * Copies host -> device, solves, copies device -> host; synchronous. */
int grim_zgesv_batched(grim_handle_t h, int n, int nrhs, const double *A, int lda, double *B, int ldb,
                       int precision_mode, int *info);
int grim_last_solve_info(grim_handle_t h, grim_solve_info *out);

/* ---- body of revolution (PEC EFIE / MFIE / CFIE per azimuthal mode) ----------------
 * nodes: 2*(ne+1) doubles (rho, z) of the generatrix, +z pole to -z pole (device).
 * grim_bor_moments: mode-independent element-pair moments for n = 0..mmax+1 of the modal
 *   Green's function (mom, grim_bor_moments_size bytes) and, when mom_k is not NULL, of
 *   the four modal MFIE brackets (mom_k, grim_bor_mfie_moments_size bytes)
 *   (reference bor/kernels.py:632 banded_modal_kernels, :896,996 the MFIE brackets,
 *   bor/bor_stream_kernel.c:332-418,915-1045 samplers and near rules).
 *   pair_class (host, ne*ne bytes): 0 far (3 x 3 Gauss points, trapezoid in xi), 1 self or
 *   adjacent, 2 other near pairs (reference bor/solver.py:1520-1580 near-pair routing);
 *   near pairs take their point pairs from rule (host, n_rule x (s, s', w)) in the ranges
 *   rule_start[0..4]: self, adjacent f = e + 1, adjacent f = e - 1, other near
 *   (reference bor/solver.py:718-806 graded cells, :843 regular cells).
 *   nxi_max bounds the far pairs' azimuthal sample count (<= 8192).
 * grim_bor_assemble: reduced mode-m matrix alpha C EFIE + (1 - alpha) eta0 MFIE
 *   (reference bor/solver.py:1769 assemble_mode, :1962 assemble_mfie_mode, CFIE
 *   :4285-4301, pole reduction :2428 reduce_pole_operator); 0 <= alpha <= 1 (0: the MFIE
 *   alone); mom_k = NULL for the EFIE alone, with alpha = 1; red_full[2*nred] lists the full components (t: node, phi:
 *   (ne+1)+node; -1 unused) of each reduced function and red_w[2*nred] (complex128) their
 *   weights.
 * grim_bor_excitation: reduced right-hand sides alpha <W, E_inc> + (1 - alpha) eta0
 *   <W, n x H_inc> (far = 0) or far-field weights (far = 1), columns [VV theta...,
 *   HH theta...] (reference bor/solver.py:2558 rhs_vv_hh_batch, :2048 rhs_mfie_mode,
 *   :2608 farfield_vv_hh_batch).
 * grim_bor_farfield_accumulate: amp[c] += sum_r W[r, c] X[r, c]. */
int64_t grim_bor_moments_size(int ne, int mmax);
int64_t grim_bor_mfie_moments_size(int ne, int mmax);
int grim_bor_moments(grim_handle_t h, int ne, const double *nodes, double k, int mmax, int nxi_max,
                     const unsigned char *pair_class, int n_rule, const double *rule, const int *rule_start,
                     void *mom, void *mom_k);
int grim_bor_assemble(grim_handle_t h, int ne, const double *nodes, double k, int mmax, int m, const void *mom,
                      const void *mom_k, double alpha, int nred, const int *red_full, const void *red_w, void *Z,
                      int64_t ldz);
int grim_bor_excitation(grim_handle_t h, int ne, const double *nodes, double k, int m, int nth,
                        const double *thetas_deg, int far, double alpha, int nred, const int *red_full,
                        const void *red_w, void *V, int64_t ldv);
/* Mirror-symmetric bodies (reference bor/factor.py:37 MirrorSplit): with the mirror map of
 * the reduced unknowns as k pairs (p1[i] < p2[i], s[i] = +-1 the sign of p2[i]) and fixed
 * unknowns fe (sign +1), fo (sign -1), n = 2k + nfe + nfo (device int / double arrays):
 * grim_bor_mirror_halves: the even (k + nfe) and odd (k + nfo) halves He, Ho (column-major,
 *   leading dimension = order) of the n x n mode matrix Z, exact when Z = R Z R;
 * grim_bor_mirror_asymmetry: out (device, 2 doubles) = (max |Z - R Z R|, max |Z|) for the
 *   full map target[n], sign[n];
 * grim_bor_mirror_split / grim_bor_mirror_join: right-hand sides into the halves' parts, and
 *   the halves' solutions back to the n unknowns. */
int grim_bor_mirror_halves(grim_handle_t h, int n, const void *Z, int64_t ldz, int k, const int *p1, const int *p2,
                           const double *s, int nfe, const int *fe, int nfo, const int *fo, void *He, void *Ho);
int grim_bor_mirror_asymmetry(grim_handle_t h, int n, const void *Z, int64_t ldz, const int *target,
                              const double *sign, double *out);
int grim_bor_mirror_split(grim_handle_t h, int nrhs, const void *B, int64_t ldb, int k, const int *p1, const int *p2,
                          const double *s, int nfe, const int *fe, int nfo, const int *fo, void *Be, void *Bo);
int grim_bor_mirror_join(grim_handle_t h, int nrhs, const void *Ye, const void *Yo, int k, const int *p1,
                         const int *p2, const double *s, int nfe, const int *fe, int nfo, const int *fo, void *X,
                         int64_t ldx);
int grim_bor_farfield_accumulate(grim_handle_t h, int nred, int ncol, const void *W, int64_t ldw, const void *X,
                                 int64_t ldx, void *amp);

/* Per-kernel profiling: while enabled, every launch records a CUDA event on the handle
 * stream; the report is JSON {"kernel": {"launches", "ms", "flops", "bytes"}} where a
 * kernel's time is the span from the previous event to its own (gaps included). */
int grim_profile_enable(grim_handle_t h, int enable);
int grim_profile_report(grim_handle_t h, char *buf, int len);

/* Free / total device memory in bytes (admission control). */
int grim_mem_info(grim_handle_t h, size_t *free_bytes, size_t *total_bytes);

/* Tile-shape overrides chosen by the autotuner (grim_20261007_b200.tuning), per handle;
 * value 0 restores the built-in rule.  GRIM_TUNE_SOLVE_BN: output-tile width (64 or 128)
 * of the tensor-core GEMMs of the packed-panel solve; GRIM_TUNE_GS_BLOCK: row block (64,
 * 128, 256 or 512) of the packed-panel solve; GRIM_TUNE_PIVOT: the pivot mode (GRIM_PIVOT_*) of
 * later factorizations on the handle (grim_getrf_grouped takes CERTIFIED or STATIC).  No
 * counterpart in the reference (its BLAS picks its own blocking and always pivots). */
#define GRIM_TUNE_SOLVE_BN 1
#define GRIM_TUNE_GS_BLOCK 2
#define GRIM_TUNE_PIVOT 3
int grim_set_tuning(grim_handle_t h, int key, int value);

#ifdef __cplusplus
}
#endif
#endif /* GRIMGPU_H */
