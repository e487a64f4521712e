// Symmetric matrix function of a solved batch: Z = V diag(f(w)) V^T.
//
// The reference ships this as a prototype, symdmt.cu:5-80 (z(i,j) =
// sum_k a(i,k) d(k) a(j,k), one warp per matrix, d supplied by the
// caller); its README:171 names the use: powers such as the square root or
// the inverse of a matrix right after its eigendecomposition (LETKF
// transforms, main.cpp:68-167).  Here f is applied on the fly:
//   SYMF_DIAG: f(x) = x         (d given by the caller in w, as symdmt)
//   SYMF_POW:  f(x) = pow(x, p) (p = 1/2 square root, -1 inverse, ...)
//   SYMF_EXP:  f(x) = exp(p x)
//
// One CTA computes one 64 x 64 tile of Z for one matrix; only tiles on or
// above the diagonal are computed and each off-diagonal tile is also
// stored transposed (Z is symmetric).  The k loop stages 16-column panels
// of V (rows of the tile) and of V scaled by f(w) (columns of the tile) in
// shared memory, coalesced from the column-major V; each of the 256
// threads accumulates a 4 x 4 register tile (rows and columns 16 apart,
// so that a warp's shared-memory reads and its stores of Z are
// contiguous).  FP64 on B200 runs SIMT FMAs at the rate of its FP64 tensor
// path, so no tensor-core form is used.
#pragma once
#include "eigb_common.cuh"

namespace eigb {

enum { SYMF_DIAG = 0, SYMF_POW = 1, SYMF_EXP = 2 };

constexpr int SF_TILE = 64;  // tile of Z per CTA
constexpr int SF_KC = 16;    // k panel
constexpr int SF_LDP = SF_TILE + 4;

template <class T> __device__ __forceinline__ T symf_apply(const int func, const T x, const T p)
{
  if (func == SYMF_POW) return pow(x, p);
  if (func == SYMF_EXP) return exp(p * x);
  return x;
}

// upper-triangular tile index t -> (ti, tj), ti <= tj, row-major over the
// upper triangle of an nt x nt tile grid
__host__ __device__ __forceinline__ void symf_tile(int t, const int nt, int &ti, int &tj)
{
  ti = 0;
  while (t >= nt - ti) {
    t -= nt - ti;
    ti++;
  }
  tj = ti + t;
}

template <class T>
__global__ void __launch_bounds__(256) k_symfunc(const long L, const int nm, const int n, const T *__restrict__ v,
                                                 const T *__restrict__ w, T *__restrict__ z, const int func,
                                                 const T p, const int ntiles)
{
  __shared__ __align__(16) T Vi[SF_KC][SF_LDP];  // V(tile rows, k)
  __shared__ __align__(16) T Vj[SF_KC][SF_LDP];  // f(w_k) V(tile columns, k)
  __shared__ T fw[SF_KC];
  const long k = blockIdx.x / ntiles;
  if (k >= L) return;
  const int nt = (n + SF_TILE - 1) / SF_TILE;
  int ti, tj;
  symf_tile((int)(blockIdx.x % ntiles), nt, ti, tj);
  const int i0 = ti * SF_TILE, j0 = tj * SF_TILE;
  const T *V = v + (size_t)k * nm * n;
  const T *W = w + (size_t)k * n;
  T *Z = z + (size_t)k * nm * n;
  const int t = threadIdx.x;
  const int tr = t % 16, tc = t / 16;  // rows tr + 16x, columns tc + 16y of the tile (x, y < 4)
  T acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = T(0);

  for (int kc = 0; kc < n; kc += SF_KC) {
    if (t < SF_KC) fw[t] = (kc + t < n) ? symf_apply(func, W[kc + t], p) : T(0);
    __syncthreads();  // fw ready; the previous panel is consumed
    // panel loads: 16 columns x 64 rows each, 4 elements per thread per panel
#pragma unroll
    for (int q = 0; q < (SF_KC * SF_TILE) / 256; q++) {
      const int e = t + 256 * q;
      const int rr = e % SF_TILE, cc = e / SF_TILE;
      const int kk = kc + cc;
      const bool kin = kk < n;
      const int ri = i0 + rr, rj = j0 + rr;
      Vi[cc][rr] = (kin && ri < n) ? V[ri + (size_t)kk * nm] : T(0);
      Vj[cc][rr] = (kin && rj < n) ? fw[cc] * V[rj + (size_t)kk * nm] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < SF_KC; c++) {
      T a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        a[u] = Vi[c][tr + 16 * u];  // 16 consecutive rows per warp: one wavefront
        b[u] = Vj[c][tc + 16 * u];
      }
#pragma unroll
      for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) acc[x][y] = fma(a[x], b[y], acc[x][y]);
    }
  }
  // Z(i, j) = Z(j, i) = acc for i <= j (every element of an off-diagonal
  // tile; the upper half of a diagonal tile), so Z is exactly symmetric
#pragma unroll
  for (int y = 0; y < 4; y++) {
    const int j = j0 + tc + 16 * y;
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const int i = i0 + tr + 16 * x;
      if (i < n && j < n && i <= j) {
        Z[i + (size_t)j * nm] = acc[x][y];
        if (i != j) Z[j + (size_t)i * nm] = acc[x][y];
      }
    }
  }
}

}  // namespace eigb
