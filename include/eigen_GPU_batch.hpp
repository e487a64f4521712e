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
 * Launch geometry of the solver's matrix-parallel phases on the current
 * device (reference: eigen_GPU_batch.hpp:23-102).  grpSZ: threads that own
 * one matrix (a warp for n <= 32, a CTA of ceil(n/32)*32 threads above);
 * numGR: matrices per thread block; numTH: threads per block; numTB: blocks
 * per launch; sizeSH: 0 (dynamic shared memory is sized internally);
 * sizeL2: the device's L2 size.
 */
template <class T>
cudaError_t eigen_GPU_batch_get_Launch_params(const int L, const int n, int &grpSZ_, int &numTB_, int &numGR_,
                                              int &numTH_, int &sizeSH_, int &sizeL2_)
{
  grpSZ_ = numTB_ = numGR_ = numTH_ = sizeSH_ = sizeL2_ = 0;
  if (L < 1 || n < 1) return cudaErrorInvalidValue;
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  int l2 = 0;
  err = cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev);
  if (err != cudaSuccess) return err;
  if (n <= 32) {
    grpSZ_ = 32;
    numGR_ = 4;
    numTH_ = 128;
    numTB_ = (L + 3) / 4;
  } else {
    grpSZ_ = std::min(1024, ((n + 31) / 32) * 32);
    numGR_ = 1;
    numTH_ = grpSZ_;
    numTB_ = L;
  }
  sizeSH_ = 0;
  sizeL2_ = l2;
  return cudaSuccess;
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
