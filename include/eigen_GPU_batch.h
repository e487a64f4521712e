/*
 * C ABI of the B200 batched symmetric eigensolver (libeigenGbatch).
 *
 * Computes all eigenvalues and eigenvectors of L real symmetric n x n
 * matrices.  Matrix k is column-major at a + k*nm*n (only its upper
 * triangle is read); on return a holds the eigenvectors column by column
 * and w + k*n the eigenvalues (ascending by default).  All pointers except
 * the size-query target are device pointers owned by the caller; every call
 * is asynchronous on `stream` and allocates nothing.
 *
 * Drop-in replacement for RIKEN-RCCS/EigenG-Batched's eigen_GPU_batch.h.
 */
#ifndef EIGEN_GPU_BATCH_B200_H
#define EIGEN_GPU_BATCH_B200_H

#include <stddef.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

/*
 * Replaces eigen_GPU_batch_DP / eigen_GPU_batch_FP of the reference
 * (eigen_GPU_batch.h:26-30, defined at eigen_GPU_batch.cu:327-359).
 * Same arguments and behaviour: L matrices of order n (1 <= n <= nm,
 * 1 <= m <= n; n <= 1024 here), eigenvectors in a, eigenvalues in w,
 * workspace wk.
 * Workspace query: when wk == NULL the required workspace size in bytes is
 * written as a size_t through w, which must then be a HOST pointer
 * (0 for n == 1), exactly as eigen_GPU_batch.cu:332-339.  The size differs
 * from the reference's formula (eigen_GPU_batch.hpp:104-118), so callers
 * must use this query or eigen_GPU_batch_BufferSize_*.
 * Invalid arguments make the call a no-op (the reference discards the
 * status too); use eigen_GPU_batch_ex_* to receive it.
 */
void eigen_GPU_batch_DP(const int L, const int nm, const int n, const int m, double *a, double *w, double *wk,
                        const cudaStream_t stream);
void eigen_GPU_batch_FP(const int L, const int nm, const int n, const int m, float *a, float *w, float *wk,
                        const cudaStream_t stream);

/*
 * Workspace size in bytes for a call with these sizes on the current
 * device.  Counterpart of the header-only template
 * eigen_GPU_batch_BufferSize<T> (eigen_GPU_batch.hpp:104-118), exported so
 * that C callers need not go through the size-query mode above.
 */
cudaError_t eigen_GPU_batch_BufferSize_DP(const int L, const int nm, const int n, const int m, size_t *lwork);
cudaError_t eigen_GPU_batch_BufferSize_FP(const int L, const int nm, const int n, const int m, size_t *lwork);

/* Eigenvalue method of the extended entry point.  TQL2 is the reference's
 * default (USE_IMTQL 0, eigen_GPU_batch.cu:3); IMTQL2 its USE_IMTQL 1
 * variant; JACOBI the cyclic Jacobi path for n <= 32 (jac_tiled.hpp). */
#define EIGEN_GPU_BATCH_TQL2 0
#define EIGEN_GPU_BATCH_IMTQL2 1
#define EIGEN_GPU_BATCH_JACOBI 2

/* eigen_GPU_batch_opts.zmem: where the apply phase keeps the rows it rotates */
#define EIGEN_GPU_ZMEM_AUTO 0   /* tensor memory where a row fits (FP64 n <= 256,
                                   FP32 n <= 512), else shared memory, else the
                                   workspace */
#define EIGEN_GPU_ZMEM_SHARED 1 /* never tensor memory (same results, bit for bit) */

typedef struct eigen_GPU_batch_opts {
  int method;    /* EIGEN_GPU_BATCH_TQL2 (default), _IMTQL2 or _JACOBI */
  int sort;      /* 1: ascending eigenvalues (reference DO_SORT 1), 0: as computed */
  int max_sweep; /* QL sweeps per eigenvalue / Jacobi passes; <= 0 means 100 */
  int rec_cap;   /* rotation records kept per matrix; <= 0: the default
                    2n^2+4n+32.  A smaller value shrinks the workspace
                    (eigen_GPU_batch_ex_BufferSize_*); a matrix whose QL
                    rotations do not fit is finished by regenerating them
                    inside the apply phase, with identical results. */
  int chunk;     /* matrices per internal chunk; <= 0: automatic (workspace
                    about 8 GiB or 512 matrices).  Bounds the workspace. */
  int split;     /* n > 32: thread blocks sharing one matrix's rows in the
                    apply phase; <= 0: automatic (the fewest whose rows fit
                    in shared memory).  Larger values trade re-reads of the
                    rotation records for more warps per SM. */
  int zmem;      /* EIGEN_GPU_ZMEM_AUTO (0; any other value but
                    EIGEN_GPU_ZMEM_SHARED means the same) or EIGEN_GPU_ZMEM_SHARED */
  int ql_mpw;    /* QL phase: matrices per warp (one per lane), a power of
                    two 1..32; <= 0: automatic (about three warps per SM;
                    fewer per warp spread a small batch over more warps).
                    Solves that run concurrently on other streams do
                    better with 4..8: fewer warps then take issue slots
                    from the other solve's kernels.  Results do not
                    depend on it. */
} eigen_GPU_batch_opts;

/* Workspace bytes for eigen_GPU_batch_ex_* with these options (NULL:
 * defaults, equal to eigen_GPU_batch_BufferSize_*). */
cudaError_t eigen_GPU_batch_ex_BufferSize_DP(const int L, const int nm, const int n, const int m,
                                             const eigen_GPU_batch_opts *opts, size_t *lwork);
cudaError_t eigen_GPU_batch_ex_BufferSize_FP(const int L, const int nm, const int n, const int m,
                                             const eigen_GPU_batch_opts *opts, size_t *lwork);

/*
 * Extended form of eigen_GPU_batch_DP/FP (no reference counterpart: the
 * reference returns nothing and has no options).  lwork is the workspace
 * size in bytes (0: not checked); info, when not NULL, is a device array of
 * L ints that receives 0, or the 1-based index at which QL exceeded
 * max_sweep, or n+1 when Jacobi did not converge within max_sweep passes.
 * opts == NULL selects the reference defaults (tql2, sorted, 100 sweeps).
 * The JACOBI method needs no workspace (wk may be NULL).
 * Returns cudaErrorInvalidValue for bad sizes, a too small workspace or an
 * unknown method, otherwise the launch status.
 */
cudaError_t eigen_GPU_batch_ex_DP(const int L, const int nm, const int n, const int m, double *a, double *w, void *wk,
                                  const size_t lwork, int *info, const eigen_GPU_batch_opts *opts,
                                  const cudaStream_t stream);
cudaError_t eigen_GPU_batch_ex_FP(const int L, const int nm, const int n, const int m, float *a, float *w, void *wk,
                                  const size_t lwork, int *info, const eigen_GPU_batch_opts *opts,
                                  const cudaStream_t stream);

/*
 * One part of an eigen_GPU_batch_ex_* solve (no counterpart in the
 * reference): the phases selected by `phases` for matrices first ..
 * first+count-1 of the batch of L (count <= 0: to the end of the batch).
 * The phases of a matrix must run in order -- reduction, QL, apply --
 * each after the previous one has completed (same stream, or an event
 * between streams); parts for disjoint matrices may run concurrently.
 * Running all three over all matrices, in any split into parts, gives the
 * results of eigen_GPU_batch_ex_* bit for bit.  The workspace is the
 * whole batch's: eigen_GPU_batch_ex_BufferSize_* for (L, nm, n, m, opts),
 * with opts->chunk = 0 or >= L, and a plan that keeps the batch in one
 * chunk (otherwise cudaErrorInvalidValue; set opts->chunk = L to force
 * it).  Matrix k keeps its own workspace slot across the calls.  n = 1
 * and the JACOBI method have a single pass, run by the part that includes
 * EIGEN_GPU_STAGE_APPLY.  This lets a caller overlap host-device copies
 * of some matrices with the phases of others and run the latency-bound
 * QL phase over many matrices at once.
 */
#define EIGEN_GPU_STAGE_REDUCE 1 /* Householder tridiagonalization and Q */
#define EIGEN_GPU_STAGE_QL 2     /* QL iteration, rotation records */
#define EIGEN_GPU_STAGE_APPLY 4  /* rotations applied to Q, sort, output */
#define EIGEN_GPU_STAGE_ALL 7
cudaError_t eigen_GPU_batch_stage_DP(const int L, const int nm, const int n, const int m, double *a, double *w,
                                     void *wk, const size_t lwork, int *info, const eigen_GPU_batch_opts *opts,
                                     const int phases, const int first, const int count, const cudaStream_t stream);
cudaError_t eigen_GPU_batch_stage_FP(const int L, const int nm, const int n, const int m, float *a, float *w,
                                     void *wk, const size_t lwork, int *info, const eigen_GPU_batch_opts *opts,
                                     const int phases, const int first, const int count, const cudaStream_t stream);

/*
 * Solve without allocating (no counterpart in the reference).  For callers
 * that must not allocate device memory -- a plugin's enqueue that runs
 * under an allocator owned by a framework, a real-time loop where
 * allocation is not allowed -- and so cannot
 * provide the workspace of eigen_GPU_batch_DP.  Arguments as there
 * (tql2, sorted eigenvalues); info is an optional device array of L ints as
 * in eigen_GPU_batch_ex_DP.
 * The workspace is a fixed 64 MiB array in the library's device memory,
 * present on every GPU that loads the library until the process exits.
 * Large batches are processed in as many pieces as needed; a single matrix
 * must fit, which holds for n <= 1024 (the size limit of every entry point).
 * Limits and behaviour:
 *  - the first call on a device looks the array's address up
 *    (cudaGetSymbolAddress); make that first call before any stream capture;
 *    the address is then cached per device for the life of the process and
 *    stays valid only while that device's primary context lives -- after a
 *    cudaDeviceReset the next call would use a stale address, so do not call
 *    it after resetting a device;
 *  - every call uses the same array: calls that may overlap on the GPU
 *    (different streams, or different host threads without ordering) race
 *    and corrupt each other's results -- serialize them;
 *  - nothing in the array needs to start cleared; each call writes what it
 *    reads;
 *  - returns cudaErrorInvalidValue for invalid sizes, otherwise the launch
 *    status.
 */
cudaError_t eigen_GPU_batch_noalloc_DP(const int L, const int nm, const int n, const int m, double *a, double *w,
                                       int *info, const cudaStream_t stream);

/*
 * Mixed-precision solve refined to FP64 accuracy (no counterpart in the
 * reference's code; its README:165,169 lists tensor-core acceleration and
 * "half precision + iterative refinement" as future work).  Same inputs and
 * outputs as eigen_GPU_batch_DP (eigenvectors overwrite a, eigenvalues
 * ascending in w; 2 <= n <= 256 here, n = 1 trivially), computed as:
 *   1. shift by sigma = trace(A)/n and solve A - sigma I in FP32 with this
 *      library's FP32 path;
 *   2. refine the eigenvectors by Ogita-Aishima iterations whose products
 *      (A X, X^T A X, X^T X, X E) run on the int8 tensor cores as exact
 *      integer slice products (Ozaki's splitting, 8 slices for the FP64-
 *      accurate ones) accumulated in FP64; clusters of close eigenvalues
 *      (up to 32) are resolved by an FP64 Rayleigh-Ritz step;
 *   3. a matrix converges when n max|E_ij|^2, E the correction between
 *      clusters of its last update, is at most tol: the orthogonality defect
 *      and residual that update leaves are of that order; it then leaves the
 *      later iterations.
 * Matrices that do not converge within max_iter iterations, whose FP32
 * solve failed, or that have a cluster of more than 32 eigenvalues, are
 * solved again by the plain FP64 path (the fallback).  Results agree with
 * eigen_GPU_batch_DP's to FP64 accuracy (residual and orthogonality of
 * order 1e-15 relative to ||A||); equal eigenvalues are ordered by index.
 * info (device, L ints, optional): 0, or the plain path's status for a
 * matrix it solved, or -1 for a matrix left unsolved with fallback = 0.
 * iters (device, L ints, optional): refinement iterations used, 0 for a
 * matrix that went to the fallback.
 * The call reads the fallback count back to the host: it synchronizes
 * `stream` once before returning (and so cannot be captured in a CUDA
 * graph).  Workspace from eigen_GPU_batch_refine_BufferSize_DP.
 * Returns cudaErrorInvalidValue for invalid sizes or a too small
 * workspace, cudaErrorLaunchFailure if a tensor-core product's bounded wait
 * gave up, otherwise the launch status.
 */
typedef struct eigen_GPU_refine_opts {
  int max_iter; /* refinement iterations at most; <= 0: 3 */
  double tol;   /* convergence threshold on n max|E_ij|^2; <= 0: 1e-14 */
  int fallback; /* 1: unconverged matrices are solved by the plain FP64 path (the
                   default when opts == NULL); 0: they are left unsolved, info -1 */
  int chunk;    /* matrices per internal chunk; <= 0: automatic (about 16 GiB) */
} eigen_GPU_refine_opts;
cudaError_t eigen_GPU_batch_refine_BufferSize_DP(const int L, const int nm, const int n,
                                                const eigen_GPU_refine_opts *opts, size_t *lwork);
cudaError_t eigen_GPU_batch_refine_DP(const int L, const int nm, const int n, double *a, double *w, void *wk,
                                      const size_t lwork, int *info, int *iters, const eigen_GPU_refine_opts *opts,
                                      const cudaStream_t stream);

/*
 * Rayleigh products of a batch (no counterpart in the reference): for each
 * matrix k, with A_k the symmetric matrix whose upper triangle is at
 * a + k*nm*n and X_k the n x n matrix at x + k*nm*n (both column-major,
 * leading dimension nm),
 *   s + k*n*n  <-  X_k^T A_k X_k      g + k*n*n  <-  X_k^T X_k
 * (column-major, leading dimension n; either may be NULL).  The products
 * are computed on the int8 tensor cores as exact integer slice products
 * (Ozaki's splitting, eight slices) accumulated in FP64, so they carry
 * FP64 accuracy relative to |A||X| and |X||X|, like FP64 GEMMs: the
 * ingredients of an a-posteriori check or a refinement of eigenvectors X
 * (S nearly diagonal, G nearly I).  2 <= n <= 256.  Asynchronous on
 * stream; workspace from eigen_GPU_batch_rayleigh_BufferSize_DP.
 */
cudaError_t eigen_GPU_batch_rayleigh_BufferSize_DP(const int L, const int nm, const int n, size_t *lwork);
cudaError_t eigen_GPU_batch_rayleigh_DP(const int L, const int nm, const int n, const double *a, const double *x,
                                        double *s, double *g, void *wk, const size_t lwork,
                                        const cudaStream_t stream);

/*
 * Packed input (the "flexible data format" the reference's README:166 lists
 * as future work; no counterpart in its code): matrix k is the upper
 * triangle in LAPACK 'U' packed order, element (r, c), r <= c (0-based), at
 * ap[k*n(n+1)/2 + r + c(c+1)/2] -- half the input bytes of the full
 * layout.  ap is not modified; the eigenvectors go to z (column-major,
 * leading dimension ldz >= n, matrix k at z + k*ldz*n) and the eigenvalues
 * to w, exactly as eigen_GPU_batch_ex_* would leave them for the same
 * matrices.  Workspace, options and status as eigen_GPU_batch_ex_*
 * (eigen_GPU_batch_ex_BufferSize_* with nm = ldz gives lwork).
 */
cudaError_t eigen_GPU_batch_packed_DP(const int L, const int n, const double *ap, double *z, const int ldz,
                                      double *w, void *wk, const size_t lwork, int *info,
                                      const eigen_GPU_batch_opts *opts, const cudaStream_t stream);
cudaError_t eigen_GPU_batch_packed_FP(const int L, const int n, const float *ap, float *z, const int ldz, float *w,
                                      void *wk, const size_t lwork, int *info, const eigen_GPU_batch_opts *opts,
                                      const cudaStream_t stream);

/*
 * Packed solve with the accuracy gate in the same call (the reference's
 * eigen_GPU_check, eigen_GPU_check.cu:4-102, run on device as part of the
 * solve rather than as a second pass over a copy of A): as
 * eigen_GPU_batch_packed_*, then, on the same stream, per matrix in FP64
 * err1 = ||A Z - Z D||_F and err2 = ||Z^T Z - I||_F from the packed input
 * (which the solve leaves intact), z and w, and flags with the reference's
 * thresholds (bit 0: err1 > max(|w_1|,|w_n|) TOL, bit 1: err2 > n TOL;
 * TOL = EPS (2*512-1) sqrt(n+16) for FP64, eps (2*16-1) sqrt(n+16) for
 * FP32).  err1, err2 and flags are device arrays of L entries; any may be
 * NULL.  The norms and flags equal eigen_GPU_check_ex_*'s on the full
 * matrices bit for bit.
 */
cudaError_t eigen_GPU_batch_packed_check_DP(const int L, const int n, const double *ap, double *z, const int ldz,
                                            double *w, void *wk, const size_t lwork, int *info,
                                            const eigen_GPU_batch_opts *opts, double *err1, double *err2, int *flags,
                                            const cudaStream_t stream);
cudaError_t eigen_GPU_batch_packed_check_FP(const int L, const int n, const float *ap, float *z, const int ldz,
                                            float *w, void *wk, const size_t lwork, int *info,
                                            const eigen_GPU_batch_opts *opts, double *err1, double *err2, int *flags,
                                            const cudaStream_t stream);

/*
 * Interleaved layout (the reference's README:166 "flexible interleave data
 * format", not in its code): element (i, j) of matrix k (0-based) at
 * ai[(i + j*n)*L + k], i.e. the same element of every matrix contiguous, as
 * SIMD-per-matrix codes keep them; eigenvector element (i, j) returned the
 * same way in zi (may equal ai), eigenvalue j of matrix k at wi[j*L + k].
 * The batch is transposed on the device into the workspace, solved there
 * (results equal eigen_GPU_batch_ex_* on the same matrices) and transposed
 * back.  lwork from eigen_GPU_batch_interleaved_BufferSize_*.
 */
cudaError_t eigen_GPU_batch_interleaved_BufferSize_DP(const int L, const int n, const eigen_GPU_batch_opts *opts,
                                                      size_t *lwork);
cudaError_t eigen_GPU_batch_interleaved_BufferSize_FP(const int L, const int n, const eigen_GPU_batch_opts *opts,
                                                      size_t *lwork);
cudaError_t eigen_GPU_batch_interleaved_DP(const int L, const int n, const double *ai, double *zi, double *wi,
                                           void *wk, const size_t lwork, int *info,
                                           const eigen_GPU_batch_opts *opts, const cudaStream_t stream);
cudaError_t eigen_GPU_batch_interleaved_FP(const int L, const int n, const float *ai, float *zi, float *wi,
                                           void *wk, const size_t lwork, int *info,
                                           const eigen_GPU_batch_opts *opts, const cudaStream_t stream);

/*
 * Uneven batches (mixed sizes in one call; the reference API is
 * uniform-n, so its users group by n and call once per size).  Matrix k has
 * order n[k] (1..1024, n is a HOST array of L ints) and is stored
 * column-major with leading dimension n[k] at a + sum_{j<k} n[j]^2; its
 * eigenvalues go to w + sum_{j<k} n[j] and its status to info[k] (device,
 * optional).  The matrices are grouped by order, largest first, and cut
 * into waves whose workspaces fit an 8 GB budget together (opts->chunk > 0
 * also caps the matrices of a wave, and so the workspace).  In each wave
 * the groups' reductions run concurrently on internal streams, then one
 * persistent launch runs the QL phase of every matrix of the wave from a
 * device work queue (longest first, opts->ql_mpw matrices per warp, 4 by
 * default), then the groups' apply phases run concurrently again.  The call
 * is asynchronous with respect to the host except for small index copies
 * from host memory, and the caller's stream waits for all of it.  Results
 * equal eigen_GPU_batch_ex_* on each matrix, bit for bit.  Other options as
 * eigen_GPU_batch_ex_*; lwork from eigen_GPU_batch_uneven_BufferSize_*
 * with the same options.
 * Limits: the index lists are copied from pageable host memory, so a call
 * cannot be captured in a CUDA graph; the group streams are a pool per
 * device shared by every caller of the library, so concurrent uneven calls
 * (from other streams or host threads) serialize on them.
 */
cudaError_t eigen_GPU_batch_uneven_BufferSize_DP(const int L, const int *n, const eigen_GPU_batch_opts *opts,
                                                 size_t *lwork);
cudaError_t eigen_GPU_batch_uneven_BufferSize_FP(const int L, const int *n, const eigen_GPU_batch_opts *opts,
                                                 size_t *lwork);
cudaError_t eigen_GPU_batch_uneven_DP(const int L, const int *n, double *a, double *w, void *wk, const size_t lwork,
                                      int *info, const eigen_GPU_batch_opts *opts, const cudaStream_t stream);
cudaError_t eigen_GPU_batch_uneven_FP(const int L, const int *n, float *a, float *w, void *wk, const size_t lwork,
                                      int *info, const eigen_GPU_batch_opts *opts, const cudaStream_t stream);

/*
 * Symmetric matrix function of a solved batch (counterpart of the
 * reference's prototype symdmt.cu:5-80, z = a diag(d) a^T, and of the use
 * its README:171 names: powers such as the square root or the inverse):
 *   z_k = V_k diag(f(w_k)) V_k^T   for every matrix k,
 * with V_k at v + k*nm*n (eigenvectors as left by eigen_GPU_batch_*),
 * w_k at w + k*n and the full symmetric result at z + k*nm*n (padding rows
 * untouched).  func: EIGEN_GPU_FUNC_DIAG f(x) = x (w already holds f of
 * the eigenvalues, as symdmt), EIGEN_GPU_FUNC_POW f(x) = pow(x, p) (p = 0.5
 * square root, -1 inverse; NaN for negative x with non-integer p),
 * EIGEN_GPU_FUNC_EXP f(x) = exp(p x).  z must not alias v.  Asynchronous
 * on stream; returns cudaErrorInvalidValue for invalid arguments.
 */
#define EIGEN_GPU_FUNC_DIAG 0
#define EIGEN_GPU_FUNC_POW 1
#define EIGEN_GPU_FUNC_EXP 2
cudaError_t eigen_GPU_batch_symfunc_DP(const int L, const int nm, const int n, const double *v, const double *w,
                                       double *z, const int func, const double p, const cudaStream_t stream);
cudaError_t eigen_GPU_batch_symfunc_FP(const int L, const int nm, const int n, const float *v, const float *w,
                                       float *z, const int func, const double p, const cudaStream_t stream);

/*
 * Launch geometry of the reduction phase (phase 1, the matrix-parallel
 * kernel) of a default solve of L matrices of order n on the current
 * device, for the first chunk of the batch; counterpart of the reference's
 * header-only eigen_GPU_batch_get_Launch_params (eigen_GPU_batch.hpp:23-102),
 * which include/eigen_GPU_batch.hpp forwards here.  grpSZ: threads that own
 * one matrix; numGR: matrices per thread block (1 also for the cluster
 * form, where a matrix spans a cluster of ceil(n/32) blocks and grpSZ
 * counts the cluster's threads); numTH: threads per block; numTB: thread
 * blocks of the launch; sizeSH: dynamic shared memory bytes per block;
 * sizeL2: the device's L2 bytes.  cudaErrorInvalidValue for L < 1, n < 1
 * or n > 1024.
 */
cudaError_t eigen_GPU_batch_launch_params_DP(const int L, const int n, int *grpSZ, int *numTB, int *numGR,
                                             int *numTH, int *sizeSH, int *sizeL2);
cudaError_t eigen_GPU_batch_launch_params_FP(const int L, const int n, int *grpSZ, int *numTB, int *numGR,
                                             int *numTH, int *sizeSH, int *sizeL2);

/*
 * Tuned options (no counterpart in the reference, whose launch parameters
 * are fixed rules, eigen_GPU_batch.hpp:23-102): a table, per device and per
 * (element size, order n), of the options a solve then uses wherever the
 * caller leaves them automatic -- the apply phase's CTAs per matrix
 * (split), where its rows live (zmem), the QL phase's matrices per warp
 * (ql_mpw) and the phase-1 kernel (reduce).  split, zmem and ql_mpw change
 * speed, not results (bit for bit); reduce changes rounding (see below).
 * eigeng_b200/autotune.py measures the candidates on the device and writes
 * such a table.  eigen_GPU_batch_tune_set replaces the current device's
 * table by `count` entries (0 clears it); it is global to the process.
 * eigen_GPU_batch_tune_get returns the entry for (esize, n), or
 * cudaErrorInvalidValue when there is none.
 */
typedef struct eigen_GPU_tune_entry {
  int esize;  /* 4 (FP32) or 8 (FP64) */
  int n;      /* matrix order, 1..1024 */
  int split;  /* 0: automatic, else as eigen_GPU_batch_opts.split (1..32) */
  int zmem;   /* EIGEN_GPU_ZMEM_AUTO or EIGEN_GPU_ZMEM_SHARED */
  int ql_mpw; /* 0: automatic, else a power of two 1..32 */
  int reduce; /* phase-1 kernel: EIGEN_GPU_REDUCE_AUTO, _CTA or _CLUSTER */
} eigen_GPU_tune_entry;
/* phase-1 kernels: automatic (the one-CTA forms, measured faster on B200),
 * one CTA per matrix (registers for n <= 128, shared memory and a band in
 * global memory above), or a thread-block cluster holding the matrix in
 * distributed shared memory (32 < n <= 512, where the device can run it).
 * Unlike the other entries, the choice changes rounding (another summation
 * order), within the solver's accuracy. */
#define EIGEN_GPU_REDUCE_AUTO 0
#define EIGEN_GPU_REDUCE_CTA 1
#define EIGEN_GPU_REDUCE_CLUSTER 2
cudaError_t eigen_GPU_batch_tune_set(const eigen_GPU_tune_entry *entries, const int count);
cudaError_t eigen_GPU_batch_tune_get(const int esize, const int n, eigen_GPU_tune_entry *out);

/*
 * Phase timing (counterpart of the reference's compile-time TIMER,
 * eigen_GPU_batch.cu:157-244, which prints per-phase times from warp 0).
 * When set, every later solve on the calling process records, for chunk c
 * of the batch, events[4c] before phase 1 (tridiagonalization + Q),
 * events[4c+1] after it, events[4c+2] after phase 2 (QL) and events[4c+3]
 * after phase 3 (rotation apply + sort), on the call's stream, for the
 * chunks whose four events fit in nevents.  events == NULL turns it off.
 * The events are created and owned by the caller.  The setting is global
 * to the process: while it is on, every solve from any host thread or
 * stream records into the same events, so trace one solve at a time.
 */
cudaError_t eigen_GPU_batch_trace(cudaEvent_t *events, const int nevents);

#ifdef __cplusplus
}
#endif

#endif
