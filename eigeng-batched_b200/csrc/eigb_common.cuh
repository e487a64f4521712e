// Common device helpers of the B200 batched symmetric eigensolver.
//
// Storage convention everywhere: column-major, element (r, c) of a matrix
// with leading dimension ld at p[r + c*ld] (0-based).  Matrix k of a batch
// starts at a + k*nm*n and its eigenvalues at w + k*n, as in the reference
// (eigen_GPU_batch.cu:89-90, eigen_GPU_batch.hpp:104-118).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

namespace eigb {

template <class T> struct Num;
template <> struct Num<double> {
  static __host__ __device__ constexpr double eps() { return 2.220446049250313080847e-16; }
  // QL deflation tolerance factor of the reference, tql2_tiled.hpp:8
  static __host__ __device__ constexpr double tolmul() { return 512.0; }
};
template <> struct Num<float> {
  static __host__ __device__ constexpr float eps() { return 1.1920928955078125e-07f; }
  static __host__ __device__ constexpr float tolmul() { return 16.0f; }
};

// 1/sqrt(x): CUDA's double rsqrt (1 ulp) and the correctly rounded float
// intrinsic.
// (host versions exist so that the scalar recurrences can be unit-tested on
// the CPU; the host rsqrt is 1/sqrt)
__host__ __device__ __forceinline__ double rsq(double x)
{
#ifdef __CUDA_ARCH__
  return rsqrt(x);
#else
  return 1.0 / sqrt(x);
#endif
}
__host__ __device__ __forceinline__ float rsq(float x)
{
#ifdef __CUDA_ARCH__
  return __frsqrt_rn(x);
#else
  return 1.0f / sqrtf(x);
#endif
}
__host__ __device__ __forceinline__ double sqr_t(double x) { return sqrt(x); }
__host__ __device__ __forceinline__ float sqr_t(float x) { return sqrtf(x); }
__host__ __device__ __forceinline__ double fabs_t(double x) { return fabs(x); }
__host__ __device__ __forceinline__ float fabs_t(float x) { return fabsf(x); }
__host__ __device__ __forceinline__ double fmax_t(double x, double y) { return fmax(x, y); }
__host__ __device__ __forceinline__ float fmax_t(float x, float y) { return fmaxf(x, y); }
__host__ __device__ __forceinline__ double copysign_t(double x, double y) { return copysign(x, y); }
__host__ __device__ __forceinline__ float copysign_t(float x, float y) { return copysignf(x, y); }

// Products that must not be fused into a neighbouring addition: the QL
// recurrences are written with explicit fma() and these, so that every copy
// of a recurrence rounds identically whatever the compiler's contraction.
__host__ __device__ __forceinline__ double mul_rn(double a, double b)
{
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
__host__ __device__ __forceinline__ float mul_rn(float a, float b)
{
#ifdef __CUDA_ARCH__
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}

// Zero guard used wherever the reference divides by a possibly vanishing
// product (misc_gpu.hpp:474-509 flip0to1).
template <class T> __host__ __device__ __forceinline__ T flip0to1(T x) { return x == T(0) ? T(1) : x; }

// Plane rotation for (a, b): r = hypot(a, b), c = a/r, s = b/r, with one
// reciprocal square root instead of a square root and two divisions.  For
// a = b = 0 it returns the identity (c = 1, s = 0, r = 0).  Like the
// reference's pythag (misc_gpu.hpp:533-548) the squares are formed
// unscaled, so |a|,|b| must stay below sqrt(overflow threshold).
template <class T>
__host__ __device__ __forceinline__ void givens(T a, T b, T &c, T &s, T &r)
{
  const T sig = fma(a, a, mul_rn(b, b));
  if (sig > T(0)) {
    const T y = rsq(sig);
    c = a * y;
    s = b * y;
    r = sig * y;
  } else {
    c = T(1);
    s = T(0);
    r = T(0);
  }
}

// sqrt(p*p + 1) without overflow for large |p| (the shift of tql2/imtql2,
// reference pythag1, misc_gpu.hpp:514-530).
template <class T>
__host__ __device__ __forceinline__ T hypot1(T p)
{
  const T ap = fabs_t(p);
  const T big = T(sizeof(T) == 8 ? 1e150 : 1e18);
  return ap > big ? ap : sqr_t(fma(p, p, T(1)));
}

// Rotation records: a record is (c, s); a segment header carries two ints
// (top rotation index i0, number of rotations that follow).  A segment
// applies rotations i0, i0-1, ..., i0-cnt+1, rotation i acting on columns
// (i, i+1) of Z:  z_{i+1} <- s z_i + c z_{i+1},  z_i <- c z_i - s z_{i+1}
// (tql2_tiled.hpp:116-121 chain order).
template <class T> struct __align__(2 * sizeof(T)) Rec { T c, s; };

union Bits64 { double d; long long i; };
union Bits32 { float f; int i; };
__host__ __device__ __forceinline__ Rec<double> make_hdr(int i0, int cnt, double)
{
  Bits64 a, b;
  a.i = i0;
  b.i = cnt;
  Rec<double> h;
  h.c = a.d;
  h.s = b.d;
  return h;
}
__host__ __device__ __forceinline__ Rec<float> make_hdr(int i0, int cnt, float)
{
  Bits32 a, b;
  a.i = i0;
  b.i = cnt;
  Rec<float> h;
  h.c = a.f;
  h.s = b.f;
  return h;
}
__host__ __device__ __forceinline__ int hdr_i0(const Rec<double> &h) { Bits64 a; a.d = h.c; return (int)a.i; }
__host__ __device__ __forceinline__ int hdr_cnt(const Rec<double> &h) { Bits64 a; a.d = h.s; return (int)a.i; }
__host__ __device__ __forceinline__ int hdr_i0(const Rec<float> &h) { Bits32 a; a.f = h.c; return a.i; }
__host__ __device__ __forceinline__ int hdr_cnt(const Rec<float> &h) { Bits32 a; a.f = h.s; return a.i; }

// Asynchronous global -> shared copy of B bytes (B = 4, 8 or 16, both
// addresses aligned to B), completed by cp_async_wait_all().  Host builds
// (unit tests) copy at once.
template <int B> __host__ __device__ __forceinline__ void cp_async(void *dst_smem, const void *src)
{
#ifdef __CUDA_ARCH__
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(B) : "memory");
#else
  memcpy(dst_smem, src, B);
#endif
}
__host__ __device__ __forceinline__ void cp_async_commit()
{
#ifdef __CUDA_ARCH__
  asm volatile("cp.async.commit_group;\n" ::: "memory");
#endif
}
__host__ __device__ __forceinline__ void cp_async_wait_all()
{
#ifdef __CUDA_ARCH__
  asm volatile("cp.async.wait_all;\n" ::: "memory");
#endif
}

// Per-matrix status block in the workspace.
struct Meta {
  int nrec;      // records written by the QL pass
  int overflow;  // 1: record capacity exceeded, the apply pass regenerates
  int ierr;      // 0 or the failing QL index (1-based, as the reference)
  int pad;
};

template <class T>
__device__ __forceinline__ T warp_sum(T x)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

__device__ __forceinline__ int warp_min_int(int x)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = min(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}

// A team is the set of threads that cooperate on one matrix: one warp
// (several independent matrices per CTA) or the whole CTA.
struct WarpTeam {
  int rank;  // 0..31
  __device__ WarpTeam() : rank(threadIdx.x & 31) {}
  __device__ __forceinline__ int size() const { return 32; }
  __device__ __forceinline__ void sync() const { __syncwarp(); }
  // Sum over the warp, result in every lane; the trailing __syncwarp orders
  // the shared-memory accesses around it like the CTA barrier does.
  template <class T> __device__ __forceinline__ T sum(T x, T *)
  {
    x = warp_sum(x);
    __syncwarp();
    return x;
  }
};

struct CtaTeam {
  int rank;
  int nthr;
  int flip;
  __device__ CtaTeam() : rank(threadIdx.x), nthr(blockDim.x), flip(0) {}
  __device__ __forceinline__ int size() const { return nthr; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
  // Sum over the CTA, result in every thread.  `red` holds 2*32 slots; the
  // two halves alternate so back-to-back reductions need one barrier each.
  template <class T> __device__ __forceinline__ T sum(T x, T *red)
  {
    x = warp_sum(x);
    T *buf = red + (flip ? 32 : 0);
    flip ^= 1;
    if ((rank & 31) == 0) buf[rank >> 5] = x;
    __syncthreads();
    const int nw = (nthr + 31) >> 5;
    T s = T(0);
    for (int k = 0; k < nw; k++) s += buf[k];
    return s;
  }
  // A sum split around a barrier the caller places: post() (called by whole
  // warps) stores the warp's sum of x in buf[warp]; after the next sync(),
  // total() adds the slots of warps w0 .. w0+nw-1.  `id` names the buffer
  // for the host emulation of a team, which keeps one slot per thread.
  template <class T> __device__ __forceinline__ void post(T x, T *buf, int) const
  {
    x = warp_sum(x);
    if ((rank & 31) == 0) buf[rank >> 5] = x;
  }
  // post(0) without the shuffles
  template <class T> __device__ __forceinline__ void post_zero(T *buf, int) const
  {
    if ((rank & 31) == 0) buf[rank >> 5] = T(0);
  }
  // within one warp: the sum of post() in every lane, lane src's x, a warp barrier
  template <class T> __device__ __forceinline__ T wsum(T x) const { return warp_sum(x); }
  template <class T> __device__ __forceinline__ T shfl(T x, const int src) const
  {
    return __shfl_sync(0xffffffffu, x, src);
  }
  __device__ __forceinline__ void sync_warp() const { __syncwarp(); }
  template <class T> __device__ __forceinline__ T total(const T *buf, int, const int w0, const int nw) const
  {
    T s = T(0);
    for (int k = 0; k < nw; k++) s += buf[w0 + k];
    return s;
  }
};

}  // namespace eigb
