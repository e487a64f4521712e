/*
 * The learned warm start of the B200 batched symmetric eigensolver (no
 * counterpart in the reference, which solves every matrix from scratch).
 *
 * For batches drawn from a parameterised family
 *     A(theta) = A0 + sum_{j=1..4} theta_j E_j
 * (A0, E_j fixed symmetric n x n matrices), a small MLP maps the family
 * coordinates of a matrix to a prediction of C(theta) = V0^T V(theta), its
 * eigenvectors in the eigenbasis V0 of A0.  The network is trained on
 * eigenpairs this library computes for family members, by this library's
 * own kernels (tensor-core forward and backward products, Adam); the solve
 * polishes the warm start V0 C with FP32-accurate tensor-core products and
 * a Jacobi iteration, checks every matrix's residual, and solves those that
 * fail with the plain tridiagonal + QL path.
 *
 * All pointers are device pointers unless stated; every call is
 * asynchronous on `stream` unless stated.
 */
#ifndef EIGEN_GPU_LEARNED_B200_H
#define EIGEN_GPU_LEARNED_B200_H

#include <stddef.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

/*
 * The network: widths d0 -> d1 -> d2 -> d3 (each a multiple of 8, at least
 * 8), tanh on the two hidden layers, a linear output, mean squared error
 * loss.  One caller-allocated parameter buffer of eigen_GPU_mlp_size bytes
 * holds the FP32 weights and biases (flat, in the order W1 b1 W2 b2 W3 b3,
 * W_l row-major with shape out x in), their Adam moments and the BF16
 * copies the products read.  Inputs x are rows x d0 and outputs rows x d3
 * FP32 row-major; rows must be a multiple of 8.  The products run on the
 * tensor cores with BF16 operands and FP32 accumulation.
 */
cudaError_t eigen_GPU_mlp_size(const int d0, const int d1, const int d2, const int d3, size_t *bytes);
/* workspace bytes of eigen_GPU_mlp_forward/_gradient/_train_step for `rows` rows */
cudaError_t eigen_GPU_mlp_ws_size(const int d0, const int d1, const int d2, const int d3, const int rows,
                                  size_t *bytes);
/* weights uniform in +-sqrt(6 / (fan_in + fan_out)) from `seed`, biases and moments zero */
cudaError_t eigen_GPU_mlp_init(const int d0, const int d1, const int d2, const int d3, void *params,
                               const unsigned long long seed, const cudaStream_t stream);
/* y = MLP(x) */
cudaError_t eigen_GPU_mlp_forward(const int d0, const int d1, const int d2, const int d3, const void *params,
                                  const int rows, const float *x, float *y, void *ws, const size_t lws,
                                  const cudaStream_t stream);
/* grad (the flat FP32 layout) = gradient of mean((MLP(x) - t)^2) over all
 * rows x d3 entries; sse (optional, one double) += the sum of squared errors */
cudaError_t eigen_GPU_mlp_gradient(const int d0, const int d1, const int d2, const int d3, const void *params,
                                   const int rows, const float *x, const float *t, float *grad, double *sse,
                                   void *ws, const size_t lws, const cudaStream_t stream);
/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8, learning rate lr,
 * step counted from 1) on that gradient */
cudaError_t eigen_GPU_mlp_train_step(const int d0, const int d1, const int d2, const int d3, void *params,
                                     const int rows, const float *x, const float *t, const float lr, const int step,
                                     double *sse, void *ws, const size_t lws, const cudaStream_t stream);

/*
 * Training targets from solved family members: for matrix b with
 * eigenvectors V_b (column-major, leading dimension ldv, matrix b at
 * v + b*ldv*n) and the family's V0 (n x n column-major),
 *     c[b*n*n + j*n + k] = s_j (V0^T V_b)(k, j),
 * s_j = +1 or -1 making the entry of largest magnitude of column j positive
 * (eigenvector signs are arbitrary; the network learns one of them).
 * n <= 64.
 */
cudaError_t eigen_GPU_learned_targets_FP(const int L, const int n, const float *v, const int ldv, const float *v0,
                                         float *c, const cudaStream_t stream);

/* warm starts of eigen_GPU_batch_learned_FP */
#define EIGEN_GPU_WARM_NETWORK 0  /* V0 C, C predicted by the network */
#define EIGEN_GPU_WARM_BASIS 1    /* V0, the eigenvectors of A0 (no network) */
#define EIGEN_GPU_WARM_IDENTITY 2 /* I (no network, no family knowledge) */

typedef struct eigen_GPU_learned_opts {
  int warm;          /* EIGEN_GPU_WARM_*; 0 by default */
  int max_sweeps;    /* Jacobi sweeps at most; <= 0: 10 */
  double tol;        /* gate: max_j ||A x_j - w_j x_j|| / max|w| at most this; <= 0: 1e-6 */
  double jacobi_tol; /* Jacobi stops when off(B) <= jacobi_tol ||B||_F; <= 0: 1e-7 */
  int fallback;      /* 1 (default when opts == NULL): matrices that fail the gate are
                        solved by the plain path; 0: left unsolved, info -1 */
  int chunk;         /* matrices per internal chunk; <= 0: automatic (about 8 GiB) */
} eigen_GPU_learned_opts;

/*
 * Solve a batch of L FP32 family members (n x n, 8 <= n <= 64, n a multiple
 * of 8; column-major, leading dimension nm, upper triangle read) with the
 * learned warm start: eigenvectors overwrite a, eigenvalues ascending in w.
 * family: FP32, six n x n column-major matrices back to back: A0, E_1..E_4
 * and V0 (the eigenvectors of A0, in columns).  params: the network
 * (d0 = 16: the four family coordinates times ten, zero padded; d1, d2 its
 * hidden widths; d3 = n*n), as trained with eigen_GPU_mlp_train_step on
 * eigen_GPU_learned_targets_FP targets; unused for the other warm starts.
 * info (optional, L ints): 0, or the plain path's status for a matrix it
 * solved, -1 for a matrix left unsolved with fallback = 0.  sweeps
 * (optional, L ints): the Jacobi sweeps of a matrix that passed the gate,
 * -1 for one that went to the fallback.  resid (optional, L doubles): the
 * gate's relative residual of each matrix.  The call reads the fallback
 * count back: it synchronizes `stream` once before returning.  Workspace
 * from eigen_GPU_batch_learned_BufferSize_FP.  Returns
 * cudaErrorInvalidValue for invalid arguments or a too small workspace,
 * cudaErrorLaunchFailure when a tensor-core product's bounded wait gave up.
 */
cudaError_t eigen_GPU_batch_learned_BufferSize_FP(const int L, const int nm, const int n, const int d1, const int d2,
                                                  const eigen_GPU_learned_opts *opts, size_t *lwork);
cudaError_t eigen_GPU_batch_learned_FP(const int L, const int nm, const int n, float *a, float *w, const float *family,
                                       const void *params, const int d1, const int d2, void *wk, const size_t lwork,
                                       int *info, int *sweeps, double *resid, const eigen_GPU_learned_opts *opts,
                                       const cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif
