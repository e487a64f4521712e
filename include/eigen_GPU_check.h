/*
 * Accuracy gate of the B200 batched symmetric eigensolver.
 *
 * Per matrix, in FP64: err1 = ||A Z - Z D||_F and err2 = ||Z^T Z - I||_F
 * (off-diagonal terms counted twice), flagged against the reference's
 * tolerance TOL = eps*(2*512-1)*sqrt(n+16) (FP64) or eps*(2*16-1)*sqrt(n+16)
 * (FP32): bit 0 when err1 > max(|w_1|,|w_n|)*TOL, bit 1 when err2 > n*TOL.
 * A (a) is read through its upper triangle.
 */
#ifndef EIGEN_GPU_CHECK_B200_H
#define EIGEN_GPU_CHECK_B200_H

#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

/*
 * Replaces eigen_GPU_check_DP / eigen_GPU_check_FP of the reference
 * (eigen_GPU_check.h, defined at eigen_GPU_check.cu:183-197): a is the
 * pristine input copy, w the eigenvalues, z the eigenvectors.  As in the
 * reference the verdict is stored as four floats over the start of each
 * matrix of `a` (eigen_GPU_check.cu:76-80) and flagged matrices are printed
 * by a device-side printf on `stream`.
 */
void eigen_GPU_check_DP(const int L, const int nm, const int n, const int m, double *a, double *w, double *z,
                        const cudaStream_t stream);
void eigen_GPU_check_FP(const int L, const int nm, const int n, const int m, float *a, float *w, float *z,
                        const cudaStream_t stream);

/*
 * Non-destructive form (no reference counterpart): err1, err2 (double) and
 * flags (int) are device arrays of L entries, each may be NULL.
 */
cudaError_t eigen_GPU_check_ex_DP(const int L, const int nm, const int n, const int m, const double *a,
                                  const double *w, const double *z, double *err1, double *err2, int *flags,
                                  const cudaStream_t stream);
cudaError_t eigen_GPU_check_ex_FP(const int L, const int nm, const int n, const int m, const float *a,
                                  const float *w, const float *z, double *err1, double *err2, int *flags,
                                  const cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif
