// Phase 3: several consecutive sweeps applied to one row in one pass.
//
// The QL recurrence emits its rotations as segments: rotations i0, i0-1,
// ..., i0-L+1, rotation i acting on columns (i, i+1) of a row of Z
// (z_{i+1} <- s z_i + c z_{i+1}, z_i <- c z_i - s z_{i+1}).  Consecutive
// sweeps usually share their top index i0 (the block end m) and each
// reaches no lower than the one before (l only grows), so K of them can
// run as a K-stage pipeline: sweep j trails sweep j-1 by one column and
// takes that sweep's output for a column as its input.  Each column is
// loaded once and stored once for all K sweeps, and a thread carries K
// independent rotation chains instead of one.
//
// Exactness: every element receives the same operations in the same
// order as with the sweeps applied one after another.  A sweep that has
// not reached a column yet, or has passed its last rotation, acts as the
// identity on the wave (its carried value moves on unchanged); the first
// K-1 steps fill the pipeline and the last K steps drain it.
//
// Used by the tensor-memory apply (k3_tmem) for rows of 128 or more; the
// row accessor below lets the host-side unit tests run the same code on
// memory.  The shared-memory and workspace forms (k3_cta) keep their
// pairs of sweeps (seg_apply_pair), measured faster there.
#pragma once
#include "eigb_common.cuh"

namespace eigb {

// Sweeps applied per pass at most.
constexpr int K3_GROUP = 8;

// Row accessor for a row in memory: element c at z[c*cs] (CS > 0: the
// stride known at compile time).
template <class T, int CS> struct RowMem {
  T *z;
  int cs_rt;
  __host__ __device__ __forceinline__ int cs() const { return CS > 0 ? CS : cs_rt; }
  __host__ __device__ __forceinline__ T ld(const int c) const { return z[c * cs()]; }
  __host__ __device__ __forceinline__ void st(const int c, const T v) const { z[c * cs()] = v; }
  // v[u] = column c - u
  __host__ __device__ __forceinline__ void ld8(const int c, T (&v)[8]) const
  {
#pragma unroll
    for (int u = 0; u < 8; u++) v[u] = z[(c - u) * cs()];
  }
  __host__ __device__ __forceinline__ void begin() const {}
};

// One step of sweep j of a group at rotation i with the wave value v
// (column i after the sweeps before j): a rotation inside the sweep's
// range, else the identity (the carried value moves on).
#define EIGB_GSTEP(J, I, V)                                 \
  {                                                         \
    const int i_ = (I);                                     \
    if (i_ >= b[J]) {                                       \
      const Rec<T> r_ = rp[J][t - i_];                      \
      const T y_ = fma(r_.c, h[J], r_.s * (V));             \
      h[J] = fma(-r_.s, h[J], r_.c * (V));                  \
      V = y_;                                               \
    } else {                                                \
      const T y_ = h[J];                                    \
      h[J] = V;                                             \
      V = y_;                                               \
    }                                                       \
  }

// K sweeps with the common top t and lengths L[0] >= L[1] >= ... >= 1
// (records rp[j][0 .. L[j]) for rotations t, t-1, ...).
template <class T, int K, class Row>
__host__ __device__ __forceinline__ void seg_apply_group(const Row &row, const Rec<T> *const (&rp)[K], const int t,
                                                         const int (&L)[K])
{
  row.begin();
  int b[K];  // last rotation of each sweep
#pragma unroll
  for (int j = 0; j < K; j++) b[j] = t - L[j] + 1;
  T h[K];  // carried value of each sweep
  h[0] = row.ld(t + 1);
#pragma unroll
  for (int j = 1; j < K; j++) h[j] = T(0);
  int x = t;  // column entering sweep 0 at this step; sweep j works at rotation x + j
  // fill: sweep s+1 takes the wave's value as its first carried value
#pragma unroll
  for (int s = 0; s < K - 1; s++, x--) {
    T v = (x >= b[0]) ? row.ld(x) : T(0);
#pragma unroll
    for (int j = 0; j < K; j++) {
      if (j <= s) EIGB_GSTEP(j, x + j, v)
      else if (j == s + 1) h[j] = v;
    }
  }
  // steady state: every sweep inside its range (x + j >= b[j] for all j),
  // no branches, U columns loaded at a time (before any of their stores: a
  // store lands K columns above the column that entered)
  int xs = b[0];
#pragma unroll
  for (int j = 1; j < K; j++) xs = max(xs, b[j] - j);
  // The next block's columns are loaded before this block is applied (they
  // lie below all of this block's stores).
  constexpr int U = 8;
  T v8[U];
  bool have = x - (U - 1) >= xs;
  if (have) row.ld8(x, v8);
  while (have) {
    const int xn = x - U;
    const bool hn = xn - (U - 1) >= xs;
    T n8[U];
    if (hn) row.ld8(xn, n8);
#pragma unroll
    for (int u = 0; u < U; u++) {
      T v = v8[u];
#pragma unroll
      for (int j = 0; j < K; j++) {
        const Rec<T> r = rp[j][t - (x - u + j)];
        const T y = fma(r.c, h[j], r.s * v);
        h[j] = fma(-r.s, h[j], r.c * v);
        v = y;
      }
      row.st(x - u + K, v);
    }
    x = xn;
    have = hn;
#pragma unroll
    for (int u = 0; u < U; u++) v8[u] = n8[u];
  }
  // the rest, and the drain (no column below b[0] is read: the wave carries
  // a zero there, which only ever passes through identities)
  for (; x >= b[0] - K; x--) {
    T v = (x >= b[0]) ? row.ld(x) : T(0);
#pragma unroll
    for (int j = 0; j < K; j++) EIGB_GSTEP(j, x + j, v)
    row.st(x + K, v);
  }
}
#undef EIGB_GSTEP

// The sweeps of rbuf[q ..) that form a group with the one at q: the same
// top, non-increasing lengths >= 1, all complete within used.  Returns the
// group size k (1..KG <= K3_GROUP), their record starts and lengths, and the
// position after the group.  (The loop is unrolled with fixed indices, so
// the arrays stay in registers.)
template <class T, int KG>
__host__ __device__ __forceinline__ int seg_group(const Rec<T> *rbuf, const int q, const int used, int &i0,
                                                  const Rec<T> *(&rp)[K3_GROUP], int (&L)[K3_GROUP], int &qnext)
{
  const Rec<T> hd = rbuf[q];
  i0 = hdr_i0(hd);
  L[0] = hdr_cnt(hd);
  rp[0] = rbuf + q + 1;
  int k = 1, qn = q + 1 + L[0];
#pragma unroll
  for (int g = 1; g < K3_GROUP; g++) {
    L[g] = 0;
    rp[g] = rp[0];
    if (g < KG && k == g && L[g - 1] >= 1 && qn < used) {
      const Rec<T> h2 = rbuf[qn];
      const int l2 = hdr_cnt(h2);
      if (hdr_i0(h2) == i0 && l2 >= 1 && l2 <= L[g - 1] && qn + 1 + l2 <= used) {
        L[g] = l2;
        rp[g] = rbuf + qn + 1;
        qn += 1 + l2;
        k++;
      }
    }
  }
  qnext = qn;
  return k;
}

// seg_apply_group for the first K of the sweeps found by seg_group
template <class T, int K, class Row>
__host__ __device__ __forceinline__ void group_call(const Row &row, const Rec<T> *const (&rp)[K3_GROUP], const int i0,
                                                   const int (&L)[K3_GROUP])
{
  const Rec<T> *r[K];
  int l[K];
#pragma unroll
  for (int j = 0; j < K; j++) {
    r[j] = rp[j];
    l[j] = L[j];
  }
  seg_apply_group<T, K>(row, r, i0, l);
}

// Applies the complete segments of rbuf[0..used) to one row: groups of up
// to KG sweeps through seg_apply_group, single sweeps through `single`
// (a functor taking the records, the top index and the length).
template <class T, int KG, class Row, class Single>
__host__ __device__ __forceinline__ void apply_grouped(const Rec<T> *rbuf, const int used, const Row &row,
                                                       const Single &single)
{
  int q = 0;
  while (q < used) {
    int i0, qn, L[K3_GROUP];
    const Rec<T> *rp[K3_GROUP];
    const int k = seg_group<T, KG>(rbuf, q, used, i0, rp, L, qn);
    switch (k) {  // k <= KG: the larger cases are compiled only where they can occur
      case 1: single(rp[0], i0, L[0]); break;
      case 2: group_call<T, 2>(row, rp, i0, L); break;
      case 3: if (KG >= 3) group_call<T, (KG >= 3 ? 3 : 2)>(row, rp, i0, L); break;
      case 4: if (KG >= 4) group_call<T, (KG >= 4 ? 4 : 2)>(row, rp, i0, L); break;
      case 5: if (KG >= 5) group_call<T, (KG >= 5 ? 5 : 2)>(row, rp, i0, L); break;
      case 6: if (KG >= 6) group_call<T, (KG >= 6 ? 6 : 2)>(row, rp, i0, L); break;
      case 7: if (KG >= 7) group_call<T, (KG >= 7 ? 7 : 2)>(row, rp, i0, L); break;
      default: if (KG >= 8) group_call<T, (KG >= 8 ? 8 : 2)>(row, rp, i0, L); break;
    }
    q = qn;
  }
}

}  // namespace eigb
