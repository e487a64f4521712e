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
// the full symmetric n x n matrix S (column-major, leading dimension ld).
// The team's nt threads form SPLIT groups of nr = nt/SPLIT threads; thread
// t owns row r = t % nr and, within every row operation, the h-th of SPLIT
// contiguous column ranges, h = t / nr.  nr is a multiple of 32, so a warp
// has one h and 32 consecutive rows: at fixed column k it touches
// consecutive addresses (shared memory: conflict-free; global: coalesced).
#pragma once
#include "eigb_common.cuh"

namespace eigb {

// Column range [lo, hi) of part h of [0, len) split in SPLIT pieces.
template <int SPLIT>
__host__ __device__ __forceinline__ void split_range(int len, int h, int &lo, int &hi)
{
  if (SPLIT == 1) {
    lo = 0;
    hi = len;
  } else {
    const int q = (len + SPLIT - 1) / SPLIT;
    lo = min(len, h * q);
    hi = min(len, lo + q);
  }
}

// sum_{k in [lo,hi)} S[r + k*ld] * v[k] with four independent accumulators
template <class T>
__host__ __device__ __forceinline__ T dot_col(const T *__restrict__ Sr, const int ld, const T *__restrict__ v,
                                              int lo, const int hi)
{
  T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
  int off = lo * ld;
  for (; lo + 4 <= hi; lo += 4, off += 4 * ld) {
    a0 = fma(Sr[off], v[lo], a0);
    a1 = fma(Sr[off + ld], v[lo + 1], a1);
    a2 = fma(Sr[off + 2 * ld], v[lo + 2], a2);
    a3 = fma(Sr[off + 3 * ld], v[lo + 3], a3);
  }
  for (; lo < hi; lo++, off += ld) a0 = fma(Sr[off], v[lo], a0);
  return (a0 + a1) + (a2 + a3);
}

// The update loops below load a batch of row elements before storing any:
// a store to Sr[k] followed by the load of Sr[k+1] cannot be reordered by
// the compiler, which would otherwise expose one full memory latency per
// element (L2 latency for the part of the matrix in global memory).
constexpr int TQ_BATCH = 8;

// Sr[k] += u_k * wr + (alpha u_k + p_k) * ur for k in [lo, hi)
template <class T>
__host__ __device__ __forceinline__ void rank2_row(T *__restrict__ Sr, const size_t ld, const T *__restrict__ u,
                                                   const T *__restrict__ pv, const T alpha, const T ur, const T wr,
                                                   int lo, const int hi)
{
  for (; lo + TQ_BATCH <= hi; lo += TQ_BATCH) {
    T a[TQ_BATCH];
#pragma unroll
    for (int q = 0; q < TQ_BATCH; q++) a[q] = Sr[(size_t)(lo + q) * ld];
#pragma unroll
    for (int q = 0; q < TQ_BATCH; q++) {
      const T uk = u[lo + q];
      const T wk = fma(alpha, uk, pv[lo + q]);
      Sr[(size_t)(lo + q) * ld] = fma(wk, ur, fma(uk, wr, a[q]));
    }
  }
  for (; lo < hi; lo++) {
    const T uk = u[lo];
    const T wk = fma(alpha, uk, pv[lo]);
    Sr[(size_t)lo * ld] = fma(wk, ur, fma(uk, wr, Sr[(size_t)lo * ld]));
  }
}

// Sr[k] += q u_k for k in [lo, hi)
template <class T>
__host__ __device__ __forceinline__ void axpy_row(T *__restrict__ Sr, const size_t ld, const T *__restrict__ u,
                                                  const T q, int lo, const int hi)
{
  for (; lo + TQ_BATCH <= hi; lo += TQ_BATCH) {
    T a[TQ_BATCH];
#pragma unroll
    for (int j = 0; j < TQ_BATCH; j++) a[j] = Sr[(size_t)(lo + j) * ld];
#pragma unroll
    for (int j = 0; j < TQ_BATCH; j++) Sr[(size_t)(lo + j) * ld] = fma(q, u[lo + j], a[j]);
  }
  for (; lo < hi; lo++) Sr[(size_t)lo * ld] = fma(q, u[lo], Sr[(size_t)lo * ld]);
}

// Reflectors applied per barrier in the formation of M.
constexpr int TQ_QB = 4;

// a[j] += sum_{c in [lo,hi)} Sr[c] U[j][c] for the TQ_QB reflectors in U
// (row stride nu): every element of the row is loaded once for all four
template <class T>
__host__ __device__ __forceinline__ void dot4_row(const T *__restrict__ Sr, const size_t ld, const T *__restrict__ U,
                                                  const int nu, int lo, const int hi, T (&a)[TQ_QB])
{
  for (; lo + TQ_BATCH <= hi; lo += TQ_BATCH) {
    T m[TQ_BATCH];
#pragma unroll
    for (int q = 0; q < TQ_BATCH; q++) m[q] = Sr[(size_t)(lo + q) * ld];
#pragma unroll
    for (int q = 0; q < TQ_BATCH; q++)
#pragma unroll
      for (int j = 0; j < TQ_QB; j++) a[j] = fma(m[q], U[j * nu + lo + q], a[j]);
  }
  for (; lo < hi; lo++) {
    const T m = Sr[(size_t)lo * ld];
#pragma unroll
    for (int j = 0; j < TQ_QB; j++) a[j] = fma(m, U[j * nu + lo], a[j]);
  }
}

// Sr[c] += sum_j q[j] U[j][c] for c in [lo, hi)
template <class T>
__host__ __device__ __forceinline__ void axpy4_row(T *__restrict__ Sr, const size_t ld, const T *__restrict__ U,
                                                   const int nu, const T (&q)[TQ_QB], int lo, const int hi)
{
  for (; lo + TQ_BATCH <= hi; lo += TQ_BATCH) {
    T m[TQ_BATCH];
#pragma unroll
    for (int x = 0; x < TQ_BATCH; x++) m[x] = Sr[(size_t)(lo + x) * ld];
#pragma unroll
    for (int x = 0; x < TQ_BATCH; x++) {
      T v = m[x];
#pragma unroll
      for (int j = 0; j < TQ_QB; j++) v = fma(q[j], U[j * nu + lo + x], v);
      Sr[(size_t)(lo + x) * ld] = v;
    }
  }
  for (; lo < hi; lo++) {
    T v = Sr[(size_t)lo * ld];
#pragma unroll
    for (int j = 0; j < TQ_QB; j++) v = fma(q[j], U[j * nu + lo], v);
    Sr[(size_t)lo * ld] = v;
  }
}

// Storage of tridiag_qt: element (r, c) is S[r + c*ld] (shared memory) when
// r < B and c < B, else G[r + c*ldg] (global memory).  B = n keeps the whole
// matrix in shared memory, B = 0 none of it; in between, the leading B x B
// block (where the bottom-up reduction spends its last steps, and the
// formation of M its first) is on chip and only the outer band goes to
// memory.  Column i < B lies entirely in S (its rows are < i), column
// i >= B entirely in G.
template <class T> struct HybridRow {
  T *s;    // row r in S: element (r, k) at s[k*ld] for k < lim
  T *g;    // row r in G: element (r, k) at g[k*ldg] for k >= lim
  int ld, ldg, lim;
  __host__ __device__ __forceinline__ T &at(int k) const
  {
    return (k < lim) ? s[(size_t)k * ld] : g[(size_t)k * ldg];
  }
};

// On entry the storage holds the full symmetric matrix (both triangles).
// On exit d_out[0:n] = diagonal, e_out[0:n] = off-diagonal (e_out[k]
// couples k and k+1, e_out[n-1] = 0, the reference's convention
// tred1_tiled.hpp:207-212) and the storage holds M = Q^T with A = Q T Q^T.
// Shared scratch: beta_s[n], pv[n], part[TQ_QB*SPLIT*nr], red[72] (64 for
// team reductions, red[64] carries the reflector pivot to the team),
// ubuf[TQ_QB*n] and gram[3n] for the formation of M.
template <class T, int SPLIT, class Team>
__host__ __device__ void tridiag_qt(Team &tm, T *S, const int ld, T *G, const int ldg, const int B, const int n,
                                    T *d_out, T *e_out, T *beta_s, T *pv, T *part, T *red, T *ubuf, T *gram)
{
  const int nt = tm.size();
  const int nr = nt / SPLIT;
  const int t = tm.rank;
  const int r = t % nr;
  const int h = t / nr;
  const HybridRow<T> row{S + r, G + r, ld, ldg, (r < B) ? B : 0};
  T *Sr = row.s;
  T *Gr = row.g;
  const int Br = row.lim;  // first column of row r held in G

  for (int i = n - 1; i >= 1; --i) {
    T *ucol = (i < B) ? S + (size_t)i * ld : G + (size_t)i * ldg;  // reflector: column i, rows 0..i-1
    // ---- reflector ----
    // Column i was last updated (previous step) by the threads whose column
    // range held i; only they read it before the barrier.
    const int hs = (SPLIT == 1) ? 0 : i / ((i + SPLIT) / SPLIT);
    T ur = (r < i && h == hs) ? ucol[r] : T(0);
    if (r == i - 1 && h == hs) red[64] = ur;  // pivot, ordered by the barrier in sum()
    const T sig = tm.sum(ur * ur, red);
    const T ulast = red[64];
    const T anorm = -copysign_t(sqr_t(sig), ulast);
    const T ul = ulast - anorm;
    const T beta = T(1) / flip0to1(ul * anorm);
    ur = (r < i - 1) ? ucol[r] : ((r == i - 1) ? ul : T(0));
    if (r == i - 1 && h == 0) ucol[i - 1] = ul;  // reflector pivot stored back
    if (t == 0) {
      e_out[i - 1] = anorm;
      beta_s[i] = beta;
    }
    int lo, hi;
    split_range<SPLIT>(i, h, lo, hi);

    // ---- p = beta * A(0:i-1, 0:i-1) u (this thread's column range) ----
    if (r < i) {
      // column i-1 of u is the new pivot ul: ucol[i-1] is being rewritten
      const int hi1 = min(hi, i - 1);
      T pp = dot_col(Sr, ld, ucol, lo, min(hi1, Br)) + dot_col(Gr, ldg, ucol, max(lo, Br), hi1);
      if (lo <= i - 1 && i - 1 < hi) pp = fma(row.at(i - 1), ul, pp);
      if (SPLIT > 1) part[h * nr + r] = pp;
      else pv[r] = pp * beta;
    }
    if (SPLIT > 1) {
      tm.sync();
      if (r < i && h == 0) {
        T pp = T(0);
#pragma unroll
        for (int q = 0; q < SPLIT; q++) pp += part[q * nr + r];
        pv[r] = pp * beta;
      }
    }
    // p_r of this row (all SPLIT threads of the row hold the same value)
    T pr = T(0);
    if (r < i) {
      if (SPLIT > 1) {
#pragma unroll
        for (int q = 0; q < SPLIT; q++) pr += part[q * nr + r];
        pr *= beta;
      } else {
        pr = pv[r];
      }
    }
    const T alpha = tm.sum(h == 0 ? pr * ur : T(0), red) * (beta * T(0.5));

    // ---- A += u w^T + w u^T, w = p + alpha u (both triangles, own columns) ----
    if (r < i) {
      const T wr = fma(alpha, ur, pr);
      const int mid = max(lo, min(hi, Br));
      rank2_row(Sr, (size_t)ld, ucol, pv, alpha, ur, wr, lo, mid);
      rank2_row(Gr, (size_t)ldg, ucol, pv, alpha, ur, wr, mid, hi);
    }
    // the barrier in the next step's first sum() orders these updates
  }
  tm.sync();
  if (r < n && h == 0) d_out[r] = row.at(r);
  if (t == 0) e_out[n - 1] = T(0);
  tm.sync();

  // ---- M = H_1 H_2 ... H_{n-1}, built in the leading k x k block ----
  // Step k extends M_{k-1} by e_{k-1} (row and column k-1) and applies
  // H_k from the right: M <- M + beta_k (M u) u^T, u = column k.  TQ_QB
  // steps per block: the block's reflectors are copied aside (the
  // extensions overwrite their columns), all its extensions are applied
  // first (H_k leaves row and column k-1 alone, so they commute), then with
  // a_j = M u_j for the M before the block,
  //   q_j = beta_j (a_j + sum_{i<j} q_i (u_i . u_j)),  M += sum_j q_j u_j^T,
  // from the Gram entries gram[3k + d - 1] = u_k . u_{k+d} computed here.
  // Every thread writes only entries of its own row and column range.
  for (int idx = t; idx < 3 * n; idx += nt) {
    const int k = idx / 3, dd = idx % 3 + 1;
    T g = T(0);
    if (k >= 1 && k + dd < n) {
      const T *uk = (k < B) ? S + (size_t)k * ld : G + (size_t)k * ldg;
      const T *uj = (k + dd < B) ? S + (size_t)(k + dd) * ld : G + (size_t)(k + dd) * ldg;
      for (int q = 0; q < k; q++) g = fma(uk[q], uj[q], g);
    }
    gram[idx] = g;
  }
  for (int k0 = 1; k0 < n; k0 += TQ_QB) {
    const int kl = min(k0 + TQ_QB - 1, n - 1);  // last step of the block
    for (int idx = t; idx < TQ_QB * n; idx += nt) {
      const int j = idx / n, q = idx % n, k = k0 + j;
      T v = T(0);
      if (k <= kl && q < k) v = ((k < B) ? S + (size_t)k * ld : G + (size_t)k * ldg)[q];
      ubuf[idx] = v;
    }
    tm.sync();  // the block's reflectors are aside; their columns may change
    // this thread's columns for the whole block: the extensions, the
    // products and the update below touch the same entries
    int lo, hi;
    split_range<SPLIT>(kl, h, lo, hi);
    for (int k = k0; k <= kl; k++) {
      if (r < k - 1) {
        if (lo <= k - 1 && k - 1 < hi) row.at(k - 1) = T(0);
      } else if (r == k - 1) {  // row k-1 of the extension (M_0 = [1] for k = 1)
        for (int c = lo; c < min(hi, k); c++) row.at(c) = (c == k - 1) ? T(1) : T(0);
      }
    }
    const int mid = max(lo, min(hi, Br));
    T a[TQ_QB];
#pragma unroll
    for (int j = 0; j < TQ_QB; j++) a[j] = T(0);
    if (r < kl) {
      dot4_row(Sr, (size_t)ld, ubuf, n, lo, mid, a);
      dot4_row(Gr, (size_t)ldg, ubuf, n, mid, hi, a);
      if (SPLIT > 1) {
#pragma unroll
        for (int j = 0; j < TQ_QB; j++) part[(j * SPLIT + h) * nr + r] = a[j];
      }
    }
    if (SPLIT > 1) tm.sync();
    if (r < kl) {
      if (SPLIT > 1) {
#pragma unroll
        for (int j = 0; j < TQ_QB; j++) {
          T x = T(0);
#pragma unroll
          for (int s2 = 0; s2 < SPLIT; s2++) x += part[(j * SPLIT + s2) * nr + r];
          a[j] = x;
        }
      }
      T q[TQ_QB];
#pragma unroll
      for (int j = 0; j < TQ_QB; j++) {
        T x = a[j];
#pragma unroll
        for (int i2 = 0; i2 < j; i2++) x = fma(q[i2], gram[3 * (k0 + i2) + (j - i2) - 1], x);
        q[j] = (k0 + j <= kl) ? beta_s[k0 + j] * x : T(0);
      }
      axpy4_row(Sr, (size_t)ld, ubuf, n, q, lo, mid);
      axpy4_row(Gr, (size_t)ldg, ubuf, n, q, mid, hi);
    }
    tm.sync();  // ubuf and part are reused by the next block
  }
  if (r < n) {
    int lo, hi;
    split_range<SPLIT>(n, h, lo, hi);
    if (r < n - 1) {
      if (lo <= n - 1 && n - 1 < hi) row.at(n - 1) = T(0);
    } else {
      for (int c = lo; c < hi; c++) row.at(c) = (c == n - 1) ? T(1) : T(0);
    }
  }
  tm.sync();
}

}  // namespace eigb
