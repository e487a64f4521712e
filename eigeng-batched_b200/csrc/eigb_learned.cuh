// The learned warm start (no counterpart in the reference): for a batch of
// FP32 matrices from a parameterised family A(theta) = A0 + sum_j theta_j E_j
// (j = 1..4), a small MLP (eigb_mlp.cuh) predicts C(theta) = V0^T V(theta),
// the eigenvectors of A(theta) in the eigenbasis V0 of A0; X0 = V0 C is the
// warm start.  A polish then makes it exact to the FP32 tolerance:
//   S = X0^T A X0, G = X0^T X0       int8 tensor-core products, 4 slices
//                                   (FP32-level accuracy, eigb_oz.cuh)
//   G = L L^T (FP64 Cholesky), B = L^-1 S L^-T, cyclic Jacobi on B with the
//   round-robin parallel ordering (n/2 disjoint rotations per round, n-1
//   rounds per sweep) until off(B) <= tol_j ||B||, Y = L^-T V
//                                   (k_lw_polish, FP64, one CTA per matrix)
//   X = X0 Y                        int8 tensor-core product, 4 slices
//   gate: max_j ||A x_j - mu_j x_j|| <= tol ||A||, FP64 from one more
//   product A X                     (k_lw_gate)
// Matrices that fail the gate are solved by the plain tridiagonal + QL path.
// The warm start can also be V0 itself or the identity (the method without
// the network), which the ablation compares.
#pragma once
#include <stdint.h>

#include "eigb_mlp.cuh"
#include "eigb_refine.cuh"

namespace eigb {

constexpr int LW_NMAX = 64;
constexpr int LW_THETA = 4;
constexpr int LW_D0 = 16;  // network input width: 4 parameters, zero padded to a multiple of 8

// prep for FP32 input: full symmetric FP64 copy of the upper triangle
// (leading dimension nm -> n), one CTA per matrix
__global__ void __launch_bounds__(256) k_lw_prep(const float *__restrict__ a, const int nm, const int n,
                                                 double *__restrict__ af)
{
  const long b = blockIdx.x;
  const float *A = a + (size_t)b * nm * n;
  double *F = af + (size_t)b * n * n;
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    const int r = idx % n, c = idx / n;
    F[idx] = (double)(r <= c ? A[(size_t)c * nm + r] : A[(size_t)r * nm + c]);
  }
}

// Gram matrix of the E_j and its inverse (FP64, 4 x 4), from the family
// buffer [A0 | E_1..E_4 | V0] (each n x n, column-major, symmetric)
__global__ void k_lw_gram(const int n, const float *__restrict__ fam, double *__restrict__ ginv)
{
  __shared__ double g[LW_THETA][LW_THETA];
  __shared__ double red[8];
  const size_t nn = (size_t)n * n;
  for (int j = 0; j < LW_THETA; j++)
    for (int k = 0; k <= j; k++) {
      double s = 0.0;
      for (size_t i = threadIdx.x; i < nn; i += blockDim.x)
        s += (double)fam[(1 + j) * nn + i] * (double)fam[(1 + k) * nn + i];
      s = blk_sum(s, red);
      if (threadIdx.x == 0) g[j][k] = g[k][j] = s;
      __syncthreads();
    }
  if (threadIdx.x == 0) {  // Gauss-Jordan on the SPD 4 x 4
    double m[LW_THETA][2 * LW_THETA];
    for (int i = 0; i < LW_THETA; i++)
      for (int j = 0; j < 2 * LW_THETA; j++) m[i][j] = j < LW_THETA ? g[i][j] : (j - LW_THETA == i ? 1.0 : 0.0);
    for (int c = 0; c < LW_THETA; c++) {
      const double pv = m[c][c];
      for (int j = 0; j < 2 * LW_THETA; j++) m[c][j] /= pv;
      for (int i = 0; i < LW_THETA; i++)
        if (i != c) {
          const double f = m[i][c];
          for (int j = 0; j < 2 * LW_THETA; j++) m[i][j] -= f * m[c][j];
        }
    }
    for (int i = 0; i < LW_THETA; i++)
      for (int j = 0; j < LW_THETA; j++) ginv[i * LW_THETA + j] = m[i][j + LW_THETA];
  }
}

// network input of each matrix: 10 theta (theta = Gram^-1 <A - A0, E_j>,
// the least-squares coordinates in the family), zero padded to LW_D0
__global__ void __launch_bounds__(256) k_lw_features(const int n, const double *__restrict__ af,
                                                     const float *__restrict__ fam, const double *__restrict__ ginv,
                                                     float *__restrict__ feat)
{
  __shared__ double red[8];
  __shared__ double bj[LW_THETA];
  const long b = blockIdx.x;
  const size_t nn = (size_t)n * n;
  const double *A = af + b * nn;
  for (int j = 0; j < LW_THETA; j++) {
    double s = 0.0;
    for (size_t i = threadIdx.x; i < nn; i += blockDim.x) s += (A[i] - (double)fam[i]) * (double)fam[(1 + j) * nn + i];
    s = blk_sum(s, red);
    if (threadIdx.x == 0) bj[j] = s;
  }
  __syncthreads();
  if (threadIdx.x < LW_D0) {
    double th = 0.0;
    if (threadIdx.x < LW_THETA)
      for (int k = 0; k < LW_THETA; k++) th += ginv[threadIdx.x * LW_THETA + k] * bj[k];
    feat[b * LW_D0 + threadIdx.x] = (float)(10.0 * th);
  }
}

// warm starts without the network: X0 = V0 (mode 1) or I (mode 2), per
// matrix column-major
__global__ void k_lw_fill(const long L, const int n, const int mode, const float *__restrict__ v0,
                          float *__restrict__ x0)
{
  const size_t nn = (size_t)n * n;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < L * (long)nn; i += (long)gridDim.x * blockDim.x) {
    const size_t e = (size_t)i % nn;
    x0[i] = mode == 1 ? v0[e] : ((e % n) == (e / n) ? 1.0f : 0.0f);
  }
}

// V0 as the BF16 right operand of the warm-start product: rows i, K index k
__global__ void k_lw_v0rows(const int n, const float *__restrict__ v0, bf16 *__restrict__ out)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * n; i += gridDim.x * blockDim.x) {
    const int r = i / n, k = i % n;
    out[i] = __float2bfloat16_rn(v0[(size_t)k * n + r]);  // V0(r, k)
  }
}

// ------------------------------------------------------------------ polish
// One CTA (256 threads) per matrix, n <= LW_NMAX; dynamic shared memory
// lw_polish_smem(n).  S, G: X0^T A X0 and X0^T X0 (FP64, column-major,
// symmetric up to rounding).  Writes Y (FP64, column-major, columns in
// ascending order of the eigenvalues mu), mu, and the sweeps it took
// (-1: G was not positive definite; the gate then fails the matrix).
__host__ __device__ inline int lw_ld(int n) { return n + 1; }
// two n x ld matrices (B; L, then V), so that three CTAs share an SM: the
// Cholesky factor waits in the output buffer Y while V is rotated
__host__ __device__ inline size_t lw_polish_smem(int n)
{
  return sizeof(double) * (2 * (size_t)n * lw_ld(n) + 2 * (size_t)n + 64) + sizeof(int) * (3 * (size_t)n + 2) + 64;
}

__global__ void __launch_bounds__(256) k_lw_polish(const int n, const double *__restrict__ S,
                                                   const double *__restrict__ G, double *__restrict__ Y,
                                                   double *__restrict__ mu, int *__restrict__ sweeps,
                                                   const int max_sweeps, const double tol_j)
{
  extern __shared__ __align__(16) unsigned char lp_smem[];
  const int ld = lw_ld(n);
  double *Bm = reinterpret_cast<double *>(lp_smem);  // n x ld, row-major: B[i*ld + j]
  double *Lm = Bm + (size_t)n * ld;                   // the Cholesky factor ...
  double *Vm = Lm;                                    // ... then the rotations
  double *cs = Vm + (size_t)n * ld;                   // 2 per pair
  double *red = cs + 2 * n;
  int *perm = reinterpret_cast<int *>(red + 64);
  int *pq = perm + n;                                  // the pairs of a round, 2 per pair
  __shared__ int bad;
  const long b = blockIdx.x;
  const int tid = threadIdx.x;
  const double *Sb = S + (size_t)b * n * n, *Gb = G + (size_t)b * n * n;
  if (tid == 0) bad = 0;
  for (int idx = tid; idx < n * n; idx += 256) {
    const int i = idx % n, j = idx / n;
    Bm[i * ld + j] = 0.5 * (Sb[(size_t)j * n + i] + Sb[(size_t)i * n + j]);
    Lm[i * ld + j] = 0.5 * (Gb[(size_t)j * n + i] + Gb[(size_t)i * n + j]);
  }
  __syncthreads();
  // Cholesky G = L L^T in place (lower triangle of Lm), left-looking
  for (int j = 0; j < n; j++) {
    double t = 0.0;
    const int i = tid;
    if (i >= j && i < n) {
      t = Lm[i * ld + j];
      for (int k = 0; k < j; k++) t -= Lm[i * ld + k] * Lm[j * ld + k];
      if (i == j) {
        if (!(t > 0.0)) bad = 1;
        Lm[j * ld + j] = sqrt(fmax(t, 1e-300));
      }
    }
    __syncthreads();
    if (i > j && i < n) Lm[i * ld + j] = t / Lm[j * ld + j];
    __syncthreads();
  }
  // B <- L^-1 B (columns in parallel), then B <- B L^-T (rows in parallel)
  for (int i = 0; i < n; i++) {
    if (tid < n) {
      double s = Bm[i * ld + tid];
      for (int k = 0; k < i; k++) s -= Lm[i * ld + k] * Bm[k * ld + tid];
      Bm[i * ld + tid] = s / Lm[i * ld + i];
    }
    __syncthreads();
  }
  for (int j = 0; j < n; j++) {
    if (tid < n) {
      double s = Bm[tid * ld + j];
      for (int k = 0; k < j; k++) s -= Bm[tid * ld + k] * Lm[j * ld + k];
      Bm[tid * ld + j] = s / Lm[j * ld + j];
    }
    __syncthreads();
  }
  // L aside in this matrix's output slot (row-major, n x n) until the
  // back substitution; its shared-memory area takes V
  double *Yb = Y + (size_t)b * n * n;
  for (int idx = tid; idx < n * n; idx += 256) Yb[idx] = Lm[(idx / n) * ld + idx % n];
  __syncthreads();
  for (int idx = tid; idx < n * n; idx += 256) {
    const int i = idx / n, j = idx % n;
    Vm[i * ld + j] = (i == j) ? 1.0 : 0.0;
    if (i < j) {  // symmetrize
      const double v = 0.5 * (Bm[i * ld + j] + Bm[j * ld + i]);
      Bm[i * ld + j] = v;
      Bm[j * ld + i] = v;
    }
  }
  __syncthreads();
  // Jacobi sweeps, round-robin ordering over np = n rounded up to even
  const int np = (n + 1) & ~1, m = np - 1, half = np / 2;
  // this thread's 2 x 2 blocks of B (pairs ka, kb) and entries of V (pair,
  // row), the same in every round: index arithmetic out of the loop
  constexpr int LW_BPT = (LW_NMAX / 2) * (LW_NMAX / 2) / 256, LW_VPT = (LW_NMAX / 2) * LW_NMAX / 256;
  int bka[LW_BPT], bkb[LW_BPT], vk[LW_VPT], vl[LW_VPT];
#pragma unroll
  for (int j = 0; j < LW_BPT; j++) {
    const int idx = tid + 256 * j;
    bka[j] = idx < half * half ? idx / half : -1;
    bkb[j] = idx < half * half ? idx % half : 0;
  }
#pragma unroll
  for (int j = 0; j < LW_VPT; j++) {
    const int idx = tid + 256 * j;
    vk[j] = idx < half * n ? idx / n : -1;
    vl[j] = idx < half * n ? idx % n : 0;
  }
  int sw = 0;
  for (; sw < max_sweeps; sw++) {
    double off = 0.0, dg = 0.0;
    for (int idx = tid; idx < n * n; idx += 256) {
      const int i = idx / n, j = idx % n;
      const double v = Bm[i * ld + j];
      if (i != j) off += v * v;
      else dg += v * v;
    }
    off = blk_sum(off, red);
    dg = blk_sum(dg, red);
    if (off <= tol_j * tol_j * dg) break;
    for (int r = 0; r < m; r++) {
      if (tid < half) {  // pair tid of round r
        int p = tid == 0 ? r : (r + tid) % m, q = tid == 0 ? m : (r - tid + m) % m;
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        double c = 1.0, s = 0.0;
        if (q < n) {
          const double app = Bm[p * ld + p], aqq = Bm[q * ld + q], apq = Bm[p * ld + q];
          if (fabs(apq) > 1e-300) {
            const double th = (aqq - app) / (2.0 * apq);
            const double t = (fabs(th) > 1e150) ? 0.5 / th : copysign(1.0, th) / (fabs(th) + sqrt(fma(th, th, 1.0)));
            c = 1.0 / sqrt(fma(t, t, 1.0));
            s = t * c;
          }
        }
        cs[2 * tid] = c;
        cs[2 * tid + 1] = s;
        pq[2 * tid] = p;
        pq[2 * tid + 1] = q;
      }
      __syncthreads();
      // B <- J^T B J in one pass: the pairs are disjoint, so entry (i, j)
      // depends only on the 2 x 2 block of the pairs of i and of j; the
      // rows are rotated first, then the columns, as two separate passes
      // over B would (same operations, same order)
#pragma unroll
      for (int jb = 0; jb < LW_BPT; jb++) {
        const int ka = bka[jb], kb = bkb[jb];
        if (ka < 0) continue;
        const int p = pq[2 * ka], q = pq[2 * ka + 1], p2 = pq[2 * kb], q2 = pq[2 * kb + 1];
        if (q < n && q2 < n) {
          const double ca = cs[2 * ka], sa = cs[2 * ka + 1], cb = cs[2 * kb], sb = cs[2 * kb + 1];
          const double b00 = Bm[p * ld + p2], b01 = Bm[p * ld + q2], b10 = Bm[q * ld + p2], b11 = Bm[q * ld + q2];
          const double r00 = ca * b00 - sa * b10, r10 = sa * b00 + ca * b10;  // rows p, q
          const double r01 = ca * b01 - sa * b11, r11 = sa * b01 + ca * b11;
          Bm[p * ld + p2] = cb * r00 - sb * r01;  // columns p2, q2
          Bm[p * ld + q2] = sb * r00 + cb * r01;
          Bm[q * ld + p2] = cb * r10 - sb * r11;
          Bm[q * ld + q2] = sb * r10 + cb * r11;
        } else if (q2 < n) {  // pair ka is the dummy of odd n: p < n, only the columns turn
          const double cb = cs[2 * kb], sb = cs[2 * kb + 1];
          const double b0 = Bm[p * ld + p2], b1 = Bm[p * ld + q2];
          Bm[p * ld + p2] = cb * b0 - sb * b1;
          Bm[p * ld + q2] = sb * b0 + cb * b1;
        } else if (q < n) {  // pair kb is the dummy: only the rows turn
          const double ca = cs[2 * ka], sa = cs[2 * ka + 1];
          const double b0 = Bm[p * ld + p2], b1 = Bm[q * ld + p2];
          Bm[p * ld + p2] = ca * b0 - sa * b1;
          Bm[q * ld + p2] = sa * b0 + ca * b1;
        } else {  // both dummies: entry (p, p2), untouched
        }
      }
      // columns p, q of V
#pragma unroll
      for (int jv = 0; jv < LW_VPT; jv++) {
        const int k = vk[jv], l = vl[jv];
        if (k < 0) continue;
        const int p = pq[2 * k], q = pq[2 * k + 1];
        if (q < n) {
          const double c = cs[2 * k], s = cs[2 * k + 1];
          const double vp = Vm[l * ld + p], vq = Vm[l * ld + q];
          Vm[l * ld + p] = c * vp - s * vq;
          Vm[l * ld + q] = s * vp + c * vq;
        }
      }
      __syncthreads();
    }
  }
  // ascending eigenvalues (ties by index)
  for (int i = tid; i < n; i += 256) {
    const double li = Bm[i * ld + i];
    int rk = 0;
    for (int j = 0; j < n; j++) {
      const double lj = Bm[j * ld + j];
      rk += (lj < li || (lj == li && j < i)) ? 1 : 0;
    }
    perm[rk] = i;
  }
  __syncthreads();
  // Y = L^-T V (back substitution, columns in parallel, each in place over
  // its column of V), column q of Y holds eigenvector perm[q]; L comes back
  // into B's area once B's diagonal, the eigenvalues, has been read
  double muq = 0.0;
  if (tid < n) muq = Bm[perm[tid] * ld + perm[tid]];
  __syncthreads();  // B is free
  double *L2 = Bm;
  for (int idx = tid; idx < n * n; idx += 256) L2[(idx / n) * ld + idx % n] = Yb[idx];
  __syncthreads();  // the output slot is free
  if (tid < n) {
    const int col = perm[tid];
    for (int i = n - 1; i >= 0; i--) {
      double s = Vm[i * ld + col];
      for (int k = i + 1; k < n; k++) s -= L2[k * ld + i] * Vm[k * ld + col];
      Vm[i * ld + col] = s / L2[i * ld + i];
    }
    mu[(size_t)b * n + tid] = muq;
  }
  __syncthreads();
  for (int idx = tid; idx < n * n; idx += 256) {
    const int i = idx % n, q = idx / n;
    Yb[(size_t)q * n + i] = Vm[i * ld + perm[q]];
  }
  if (tid == 0) sweeps[b] = bad ? -1 : sw;
}

// ------------------------------------------------------------------- gate
// res_j = ||(A X)_j - mu_j x_j|| / max|mu|; pass when max_j res_j <= tol.
// Passing matrices get their eigenvectors (FP32, leading dimension nm) and
// eigenvalues; failing ones go to the fallback list.
__global__ void __launch_bounds__(256) k_lw_gate(const int n, const int nm, const double *__restrict__ AX,
                                                 const double *__restrict__ X, const double *__restrict__ mu,
                                                 const int *__restrict__ sweeps, const double tol,
                                                 float *__restrict__ a, float *__restrict__ w, int *__restrict__ info,
                                                 int *__restrict__ sweeps_out, double *__restrict__ res_out,
                                                 int *__restrict__ fb_list, int *__restrict__ fb_count,
                                                 const long gofs)
{
  __shared__ double red[8];
  const long b = blockIdx.x;
  const double *AXb = AX + (size_t)b * n * n, *Xb = X + (size_t)b * n * n, *mb = mu + (size_t)b * n;
  double am = 0.0;
  for (int j = threadIdx.x; j < n; j += 256) am = fmax(am, fabs(mb[j]));
  am = blk_max(am, red);
  double worst = 0.0;
  // one column per warp
  const int warp = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int j = warp; j < n; j += 8) {
    double s = 0.0;
    for (int i = l; i < n; i += 32) {
      const double d = AXb[(size_t)j * n + i] - mb[j] * Xb[(size_t)j * n + i];
      s += d * d;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    worst = fmax(worst, sqrt(s));
  }
  worst = blk_max(worst, red) / fmax(am, 1e-300);
  const bool pass = sweeps[b] >= 0 && worst <= tol;  // NaN fails
  if (threadIdx.x == 0 && res_out) res_out[gofs + b] = worst;
  if (!pass) {
    if (threadIdx.x == 0) {
      fb_list[atomicAdd(fb_count, 1)] = (int)(gofs + b);
      if (sweeps_out) sweeps_out[gofs + b] = -1;
    }
    return;
  }
  float *A = a + (size_t)(gofs + b) * nm * n;
  for (int idx = threadIdx.x; idx < n * n; idx += 256) {
    const int i = idx % n, j = idx / n;
    A[(size_t)j * nm + i] = (float)Xb[(size_t)j * n + i];
  }
  for (int j = threadIdx.x; j < n; j += 256) w[(size_t)(gofs + b) * n + j] = (float)mb[j];
  if (threadIdx.x == 0) {
    if (info) info[gofs + b] = 0;
    if (sweeps_out) sweeps_out[gofs + b] = sweeps[b];
  }
}

}  // namespace eigb

namespace eigb {
// training targets: c_b[j*n + k] = s_j (V0^T V_b)(k, j), s_j = +-1 making
// the entry of largest magnitude in column j positive; one CTA per matrix
// (V_b column-major with leading dimension ldv)
__global__ void __launch_bounds__(256) k_lw_targets(const int n, const float *__restrict__ v, const int ldv,
                                                    const float *__restrict__ v0, float *__restrict__ c)
{
  extern __shared__ __align__(16) unsigned char lt_smem[];
  float *sv0 = reinterpret_cast<float *>(lt_smem);  // n x n
  float *sv = sv0 + n * n;                          // n x n
  const long b = blockIdx.x;
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
    sv0[i] = v0[i];
    sv[i] = v[(size_t)b * ldv * n + (size_t)(i / n) * ldv + (i % n)];
  }
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    float best = 0.0f;
    for (int k = 0; k < n; k++) {
      float s = 0.0f;
      for (int i = 0; i < n; i++) s = fmaf(sv0[k * n + i], sv[j * n + i], s);
      if (fabsf(s) > fabsf(best)) best = s;
    }
    const float sg = best < 0.0f ? -1.0f : 1.0f;
    for (int k = 0; k < n; k++) {
      float s = 0.0f;
      for (int i = 0; i < n; i++) s = fmaf(sv0[k * n + i], sv[j * n + i], s);
      c[(size_t)b * n * n + (size_t)j * n + k] = sg * s;
    }
  }
}
}  // namespace eigb
