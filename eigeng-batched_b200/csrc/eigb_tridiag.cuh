// Phase 1: Householder tridiagonalization and explicit formation of Q^T.
//
// Method: the reference's bottom-up reduction (tred1_tiled.hpp:42-205,
// hhsy2tr.hpp:53-300): for column i = n-1 .. 1 (0-based) the reflector
// u = A(0:i-1, i) with pivot u_{i-1} := u_{i-1} - anorm,
// anorm = -sign(||u||, u_{i-1}), beta = 1/flip0to1(u_pivot*anorm), so that
// H_i = I + beta u u^T and A <- H_i A H_i = A + u w^T + w u^T with
// w = beta A u + (beta/2)(u^T beta A u) u.
//
// Instead of keeping the reflectors for a back-transformation of the final
// eigenvectors (hhtr2sy_tiled.hpp, 2n^3 flops), this phase accumulates
// M = Q^T = H_1 H_2 ... H_{n-1} in place over the reflector storage
// (4/3 n^3 flops); the QL rotations are later applied to Q directly, which
// gives the same eigenvectors Q * Z_T up to rounding.
//
// Thread mapping: the team (one warp, or the whole CTA) owns the rows of
// the full symmetric n x n matrix S (column-major, leading dimension ld):
// thread t owns rows t, t + size, ..., t + (R-1)*size.  Every access S[r +
// k*ld] of a team at fixed k touches consecutive rows, i.e. consecutive
// addresses in shared memory (conflict-free) or in global memory
// (coalesced).
#pragma once
#include "eigb_common.cuh"

namespace eigb {

// On entry S holds the full symmetric matrix (both triangles).  On exit
// d_out[0:n] = diagonal, e_out[0:n] = off-diagonal (e_out[k] couples k and
// k+1, e_out[n-1] = 0, the reference's convention tred1_tiled.hpp:207-212)
// and S holds M = Q^T with A = Q T Q^T.
//   beta_s, pv: n-element scratch in shared memory; red: 72 slots (64 for
//   team reductions, red[64] carries the reflector pivot to the team).
template <class T, int R, class Team>
__host__ __device__ void tridiag_qt(Team &tm, T *S, const int ld, const int n, T *d_out, T *e_out,
                           T *beta_s, T *pv, T *red)
{
  const int nt = tm.size();
  const int t = tm.rank;

  for (int i = n - 1; i >= 1; --i) {
    // ---- reflector from column i (rows 0..i-1) ----
    T ur[R];
    T ss = T(0);
#pragma unroll
    for (int j = 0; j < R; j++) {
      const int r = t + j * nt;
      ur[j] = (r < i) ? S[r + (size_t)i * ld] : T(0);
      ss = fma(ur[j], ur[j], ss);
      // the owner of row i-1 publishes the pivot; the barrier in sum()
      // orders it after the previous step's updates of that row
      if (r == i - 1) red[64] = ur[j];
    }
    const T sig = tm.sum(ss, red);
    const T ulast = red[64];
    const T anorm = -copysign_t(sqr_t(sig), ulast);
    const T ul = ulast - anorm;
    const T beta = T(1) / flip0to1(ul * anorm);
#pragma unroll
    for (int j = 0; j < R; j++) {
      const int r = t + j * nt;
      if (r == i - 1) {
        ur[j] = ul;
        S[r + (size_t)i * ld] = ul;  // reflector pivot stored back
      }
    }
    if (t == 0) {
      e_out[i - 1] = anorm;
      beta_s[i] = beta;
    }

    // ---- p = beta * A(0:i-1, 0:i-1) u ----
    T p[R];
#pragma unroll
    for (int j = 0; j < R; j++) p[j] = T(0);
    {
      const T *ucol = S + (size_t)i * ld;
      for (int k = 0; k < i - 1; k++) {
        const T uk = ucol[k];
        const T *sk = S + (size_t)k * ld;
#pragma unroll
        for (int j = 0; j < R; j++) {
          const int r = t + j * nt;
          if (r < i) p[j] = fma(sk[r], uk, p[j]);
        }
      }
      const T *sk = S + (size_t)(i - 1) * ld;
#pragma unroll
      for (int j = 0; j < R; j++) {
        const int r = t + j * nt;
        if (r < i) {
          p[j] = fma(sk[r], ul, p[j]);
          p[j] *= beta;
          pv[r] = p[j];
        }
      }
    }
    T pu = T(0);
#pragma unroll
    for (int j = 0; j < R; j++) pu = fma(p[j], ur[j], pu);
    const T alpha = tm.sum(pu, red) * (beta * T(0.5));

    // ---- A += u w^T + w u^T, w = p + alpha u (both triangles) ----
    {
      T wr[R];
#pragma unroll
      for (int j = 0; j < R; j++) wr[j] = fma(alpha, ur[j], p[j]);
      const T *ucol = S + (size_t)i * ld;
      for (int k = 0; k < i; k++) {
        const T uk = ucol[k];
        const T wk = fma(alpha, uk, pv[k]);
        T *sk = S + (size_t)k * ld;
#pragma unroll
        for (int j = 0; j < R; j++) {
          const int r = t + j * nt;
          if (r < i) sk[r] = fma(wk, ur[j], fma(uk, wr[j], sk[r]));
        }
      }
    }
    // the barrier in the next step's first sum() orders these updates
  }
  tm.sync();
#pragma unroll
  for (int j = 0; j < R; j++) {
    const int r = t + j * nt;
    if (r < n) d_out[r] = S[r + (size_t)r * ld];
  }
  if (t == 0) e_out[n - 1] = T(0);
  tm.sync();

  // ---- M = H_1 H_2 ... H_{n-1}, built in the leading k x k block ----
  if (t == 0) S[0] = T(1);
  for (int k = 1; k < n; k++) {
    const T bk = beta_s[k];
    const T *ucol = S + (size_t)k * ld;  // reflector k, rows 0..k-1
#pragma unroll
    for (int j = 0; j < R; j++) {
      const int r = t + j * nt;
      // extend M_{k-1} by e_{k-1}: column k-1 (rows < k-1) and row k-1
      if (r < k - 1) S[r + (size_t)(k - 1) * ld] = T(0);
      if (r == k - 1)
        for (int c = 0; c < k; c++) S[r + (size_t)c * ld] = (c == k - 1) ? T(1) : T(0);
    }
    // M <- M + beta (M u) u^T, row-local
    T q[R];
#pragma unroll
    for (int j = 0; j < R; j++) q[j] = T(0);
    for (int c = 0; c < k; c++) {
      const T uc = ucol[c];
      const T *sc = S + (size_t)c * ld;
#pragma unroll
      for (int j = 0; j < R; j++) {
        const int r = t + j * nt;
        if (r < k) q[j] = fma(sc[r], uc, q[j]);
      }
    }
#pragma unroll
    for (int j = 0; j < R; j++) q[j] *= bk;
    for (int c = 0; c < k; c++) {
      const T uc = ucol[c];
      T *sc = S + (size_t)c * ld;
#pragma unroll
      for (int j = 0; j < R; j++) {
        const int r = t + j * nt;
        if (r < k) sc[r] = fma(q[j], uc, sc[r]);
      }
    }
    tm.sync();  // column k is overwritten by the next extension
  }
#pragma unroll
  for (int j = 0; j < R; j++) {
    const int r = t + j * nt;
    if (r < n - 1) S[r + (size_t)(n - 1) * ld] = T(0);
    if (r == n - 1)
      for (int c = 0; c < n; c++) S[r + (size_t)c * ld] = (c == n - 1) ? T(1) : T(0);
  }
  tm.sync();
}

}  // namespace eigb
