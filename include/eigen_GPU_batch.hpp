/*
 * C++ interface of the B200 batched symmetric eigensolver, replacing the
 * reference's header-only eigen_GPU_batch.hpp (eigen_GPU_batch.hpp:23-157):
 * eigen_GPU_batch_get_Launch_params<T>, eigen_GPU_batch_BufferSize<T> and
 * eigen_GPU_batch<T> keep their names and signatures.  The workspace size
 * is this library's own (see eigen_GPU_batch_BufferSize_*), so code built
 * against the reference header must be rebuilt against this one.
 */
#ifndef EIGEN_GPU_BATCH_B200_HPP
#define EIGEN_GPU_BATCH_B200_HPP

#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "eigen_GPU_batch.h"

/*
 * Launch geometry of the solver's matrix-parallel reduction phase on the
 * current device (reference: eigen_GPU_batch.hpp:23-102), exactly as the
 * library launches it: grpSZ threads own one matrix (a warp for n <= 32,
 * a CTA of 32*NB*NB threads for the register form at 32 < n <= 128, NB =
 * ceil(n/32), else the CTA form), numGR matrices per block of numTH
 * threads, numTB blocks for the first chunk of the batch, sizeSH bytes of
 * dynamic shared memory per block, sizeL2 the device's L2 size.
 */
template <class T>
cudaError_t eigen_GPU_batch_get_Launch_params(const int L, const int n, int &grpSZ_, int &numTB_, int &numGR_,
                                              int &numTH_, int &sizeSH_, int &sizeL2_)
{
  if (std::is_same<T, double>::value)
    return eigen_GPU_batch_launch_params_DP(L, n, &grpSZ_, &numTB_, &numGR_, &numTH_, &sizeSH_, &sizeL2_);
  if (std::is_same<T, float>::value)
    return eigen_GPU_batch_launch_params_FP(L, n, &grpSZ_, &numTB_, &numGR_, &numTH_, &sizeSH_, &sizeL2_);
  grpSZ_ = numTB_ = numGR_ = numTH_ = sizeSH_ = sizeL2_ = 0;
  return cudaErrorInvalidValue;
}

/* Workspace size in bytes (reference: eigen_GPU_batch.hpp:104-118). */
template <class T>
cudaError_t eigen_GPU_batch_BufferSize(const int L, const int nm, const int n, const int m, T *a, T *w,
                                       size_t *lwork)
{
  (void)a;
  (void)w;
  if (std::is_same<T, double>::value) return eigen_GPU_batch_BufferSize_DP(L, nm, n, m, lwork);
  if (std::is_same<T, float>::value) return eigen_GPU_batch_BufferSize_FP(L, nm, n, m, lwork);
  if (lwork) *lwork = 0;
  return cudaErrorInvalidValue;
}

/* Solve (reference: eigen_GPU_batch.hpp:120-157). */
template <class T>
void eigen_GPU_batch(const int L, const int nm, const int n, const int m, T *a, T *w, T *wk,
                     const cudaStream_t stream = NULL)
{
  if (std::is_same<T, float>::value)
    eigen_GPU_batch_FP(L, nm, n, m, (float *)a, (float *)w, (float *)wk, stream);
  if (std::is_same<T, double>::value)
    eigen_GPU_batch_DP(L, nm, n, m, (double *)a, (double *)w, (double *)wk, stream);
}

#endif
