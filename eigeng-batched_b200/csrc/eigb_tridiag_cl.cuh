// Phase 1 on a thread-block cluster: the matrix in distributed shared memory.
//
// Same method as eigb_tridiag.cuh (the reference's bottom-up Householder
// reduction, tred1_tiled.hpp:42-205, then M = Q^T = H_1 ... H_{n-1} built in
// place over the reflectors), for 128 < n <= 512, where one CTA's shared
// memory cannot hold the matrix: a cluster of cn = ceil(n / 32) CTAs holds
// it, CTA c the 32 consecutive full rows 32c .. 32c+31 (column-major slab,
// leading dimension 33, element (r, k) at S[(r - 32c) + 33 k]).  Every row
// operation of the method (the product A u, the rank-2 update, the
// formation's products and updates) is local to the row's owner; what
// crosses the cluster is small:
//   step i   the reflector u (column i) and p = beta A u, i values each,
//            stored by their owners into every CTA's copy (double buffered
//            by the parity of i), and two scalars (u.u and u.p) as one
//            partial per CTA; two cluster barriers per step;
//   block    the formation's QB reflectors, pulled from their owners into
//            every CTA, one cluster barrier per block;
//   once     the Gram entries u_k . u_{k+d} as partials per CTA.
// The cluster barriers are the hardware's (barrier.cluster arrive/wait
// through cooperative groups): every thread of every CTA takes the same
// sequence of them, and the kernel ends with one, so no CTA leaves while
// another may still read its shared memory.  No spin waits.
//
// Within a CTA, warp h owns column range h of SPLIT (split_range, as in
// eigb_tridiag.cuh) and lane l row 32c + l; a warp's accesses at one column
// are 32 consecutive rows (conflict-free).
#pragma once
#include <cooperative_groups.h>

#include "eigb_common.cuh"
#include "eigb_tridiag.cuh"

namespace eigb {

constexpr int CL_ROWS = 32;     // rows per CTA
constexpr int CL_LDS = 33;      // slab leading dimension
constexpr int CL_QB = TQ_QB;    // reflectors per formation block
constexpr int CL_MAX_CN = 16;   // n <= 512

__host__ __device__ inline int cl_cn(int n) { return (n + CL_ROWS - 1) / CL_ROWS; }

// Shared-memory layout (elements of T): slab, beta, then a union of the
// reduction's buffers and the formation's.
struct ClLayout {
  int slab, beta, uni;                       // offsets
  int u, pv, red, part;                      // reduction (relative to uni)
  int gp, gram, ub, fpart;                   // formation (relative to uni)
  int total;
};
template <int SPLIT> __host__ __device__ inline ClLayout cl_layout(int n)
{
  const int cn = cl_cn(n);
  auto ev = [](int x) { return (x + 1) & ~1; };  // keep 16-byte alignment for T = double pairs
  ClLayout L;
  L.slab = 0;
  L.beta = ev(CL_LDS * n);
  L.uni = L.beta + ev(n);
  L.u = 0;
  L.pv = L.u + 2 * n;
  L.red = L.pv + 2 * n;
  L.part = L.red + ev(4 * cn);
  const int ured = L.part + SPLIT * CL_ROWS;
  L.gram = 0;
  L.ub = L.gram + ev(3 * n);
  L.gp = L.ub;  // the Gram partials live in the reflector buffer until the first block
  L.fpart = L.ub + ev(CL_QB * n > 3 * n ? CL_QB * n : 3 * n);
  const int uform = L.fpart + CL_QB * SPLIT * CL_ROWS;
  L.total = L.uni + (ured > uform ? ured : uform);
  return L;
}
template <class T, int SPLIT> __host__ __device__ inline size_t cl_smem_bytes(int n)
{
  return sizeof(T) * (size_t)cl_layout<SPLIT>(n).total;
}

template <class T> __device__ __forceinline__ T cl_warp_sum(T v)
{
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// A (n x n, leading dimension nm, upper triangle used; or the packed upper
// triangle Ap) -> d, e and Q in A.  One cluster per matrix; called by all
// threads of all its CTAs.
template <class T, int SPLIT>
__device__ void tridiag_qt_cluster(T *A, const int nm, const int n, T *d_out, T *e_out, const T *Ap, T *sm)
{
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int cn = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const int t = threadIdx.x;
  const int NT = 32 * SPLIT;
  const int rl = t & 31, h = t >> 5;
  const int r0 = rank * CL_ROWS;
  const int r = r0 + rl;
  const bool own = r < n;  // lanes past the last row carry zeros and skip row work
  const ClLayout LY = cl_layout<SPLIT>(n);
  T *S = sm + LY.slab;
  T *Sr = S + rl;
  T *beta_s = sm + LY.beta;
  T *U = sm + LY.uni + LY.u;      // [2][n]
  T *PV = sm + LY.uni + LY.pv;    // [2][n]
  T *RED = sm + LY.uni + LY.red;  // [2 parity][2 kind][cn]
  T *PART = sm + LY.uni + LY.part;

  // ---- the slab: rows r0 .. r0+31 of the full symmetric matrix ----
  for (int idx = t; idx < CL_ROWS * n; idx += NT) {  // upper part, k >= r: column k, rows consecutive
    const int l = idx % CL_ROWS, k = idx / CL_ROWS, rr = r0 + l;
    if (rr < n && k >= rr) S[l + CL_LDS * k] = Ap ? Ap[rr + (size_t)k * (k + 1) / 2] : A[rr + (size_t)k * nm];
  }
  for (int idx = t; idx < CL_ROWS * n; idx += NT) {  // lower part, k < r: element (k, r) of column r
    const int k = idx % n, l = idx / n, rr = r0 + l;
    if (rr < n && k < rr) S[l + CL_LDS * k] = Ap ? Ap[k + (size_t)rr * (rr + 1) / 2] : A[k + (size_t)rr * nm];
  }
  for (int idx = t; idx < CL_ROWS * n; idx += NT) {  // padding rows of the last CTA: zero
    const int l = idx % CL_ROWS, k = idx / CL_ROWS;
    if (r0 + l >= n) S[l + CL_LDS * k] = T(0);
  }
  cl.sync();

  // ---- reduction, i = n-1 .. 1 ----
  for (int i = n - 1; i >= 1; --i) {
    const int b = i & 1;
    T *ub = U + b * n, *pb = PV + b * n, *rs = RED + (2 * b) * cn, *ra = RED + (2 * b + 1) * cn;
    // A: column i (last updated by the warp whose range held i in step i+1)
    // goes to every CTA's copy of u, with the partial of u.u
    const int hs = (SPLIT == 1) ? 0 : i / ((i + SPLIT) / SPLIT);
    if (h == hs) {
      const T ur = (own && r < i) ? Sr[CL_LDS * i] : T(0);
      if (own && r < i)
        for (int c = 0; c < cn; c++) cl.map_shared_rank(ub, c)[r] = ur;
      const T s = cl_warp_sum(ur * ur);
      if (rl == 0)
        for (int c = 0; c < cn; c++) cl.map_shared_rank(rs, c)[rank] = s;
    }
    cl.sync();
    // B: the reflector, then p = beta A u for this CTA's rows
    T sig = T(0);
    for (int c = 0; c < cn; c++) sig += rs[c];
    const T ulast = ub[i - 1];
    const T anorm = -copysign_t(sqr_t(sig), ulast);
    const T ul = ulast - anorm;
    const T beta = T(1) / flip0to1(ul * anorm);
    if (h == hs && own && r == i - 1) Sr[CL_LDS * i] = ul;  // reflector pivot stored back
    if (t == 0) {
      beta_s[i] = beta;
      if (rank == 0) e_out[i - 1] = anorm;
    }
    int lo, hi;
    split_range<SPLIT>(i, h, lo, hi);
    if (own && r < i) {
      const int hi1 = min(hi, i - 1);
      T pp = dot_col(Sr, CL_LDS, ub, lo, hi1);
      if (lo <= i - 1 && i - 1 < hi) pp = fma(Sr[CL_LDS * (i - 1)], ul, pp);
      PART[h * CL_ROWS + rl] = pp;
    }
    __syncthreads();  // every thread has read ulast: u_{i-1} may become the pivot
    if (t == 0) ub[i - 1] = ul;  // read again only after the cluster barrier
    if (h == 0) {
      T pr = T(0), x = T(0);
      if (own && r < i) {
#pragma unroll
        for (int q = 0; q < SPLIT; q++) pr += PART[q * CL_ROWS + rl];
        pr *= beta;
        for (int c = 0; c < cn; c++) cl.map_shared_rank(pb, c)[r] = pr;
        x = (r == i - 1 ? ul : ub[r]) * pr;
      }
      const T s = cl_warp_sum(x);
      if (rl == 0)
        for (int c = 0; c < cn; c++) cl.map_shared_rank(ra, c)[rank] = s;
    }
    cl.sync();
    // C: A += u w^T + w u^T on this CTA's rows, w = p + alpha u
    T al = T(0);
    for (int c = 0; c < cn; c++) al += ra[c];
    const T alpha = al * (beta * T(0.5));
    if (own && r < i) {
      const T ur = ub[r];
      const T wr = fma(alpha, ur, pb[r]);
      rank2_row(Sr, (size_t)CL_LDS, ub, pb, alpha, ur, wr, lo, hi);
    }
  }
  __syncthreads();
  if (h == 0 && own) d_out[r] = Sr[CL_LDS * r];
  if (t == 0 && rank == 0) e_out[n - 1] = T(0);

  // ---- M = H_1 ... H_{n-1} (the formation of eigb_tridiag.cuh) ----
  T *GP = sm + LY.uni + LY.gp;
  T *GRAM = sm + LY.uni + LY.gram;
  T *UB = sm + LY.uni + LY.ub;        // [CL_QB][n]
  T *FPART = sm + LY.uni + LY.fpart;  // [CL_QB][SPLIT][32]
  // partials of gram[3k + d - 1] = u_k . u_{k+d} over this CTA's rows
  for (int idx = t; idx < 3 * n; idx += NT) {
    const int k = idx / 3, dd = idx % 3 + 1;
    T g = T(0);
    if (k >= 1 && k + dd < n)
      for (int l = 0; l < CL_ROWS && r0 + l < k; l++) g = fma(S[l + CL_LDS * k], S[l + CL_LDS * (k + dd)], g);
    GP[idx] = g;
  }
  cl.sync();
  for (int idx = t; idx < 3 * n; idx += NT) {
    T g = T(0);
    for (int c = 0; c < cn; c++) g += cl.map_shared_rank(GP, c)[idx];
    GRAM[idx] = g;
  }
  cl.sync();  // every CTA has read the partials: their buffer takes the reflectors
  for (int k0 = 1; k0 < n; k0 += CL_QB) {
    const int kl = min(k0 + CL_QB - 1, n - 1);
    T *ubk = UB;
    // the block's reflectors from their owners (columns k0 .. kl are no
    // longer written by anyone: earlier blocks touch columns < k0)
    for (int idx = t; idx < CL_QB * n; idx += NT) {
      const int j = idx / n, q = idx % n, k = k0 + j;
      T v = T(0);
      if (k <= kl && q < k) v = cl.map_shared_rank(S, q / CL_ROWS)[(q % CL_ROWS) + CL_LDS * k];
      ubk[idx] = v;
    }
    cl.sync();  // every CTA has its copy before the extensions overwrite the columns
    int lo, hi;
    split_range<SPLIT>(kl, h, lo, hi);
    if (own) {
      for (int k = k0; k <= kl; k++) {
        if (r < k - 1) {
          if (lo <= k - 1 && k - 1 < hi) Sr[CL_LDS * (k - 1)] = T(0);
        } else if (r == k - 1) {
          for (int c = lo; c < min(hi, k); c++) Sr[CL_LDS * c] = (c == k - 1) ? T(1) : T(0);
        }
      }
    }
    T a[CL_QB];
#pragma unroll
    for (int j = 0; j < CL_QB; j++) a[j] = T(0);
    if (own && r < kl) {
      dot4_row(Sr, (size_t)CL_LDS, ubk, n, lo, hi, a);
#pragma unroll
      for (int j = 0; j < CL_QB; j++) FPART[(j * SPLIT + h) * CL_ROWS + rl] = a[j];
    }
    __syncthreads();
    if (own && r < kl) {
#pragma unroll
      for (int j = 0; j < CL_QB; j++) {
        T x = T(0);
#pragma unroll
        for (int s2 = 0; s2 < SPLIT; s2++) x += FPART[(j * SPLIT + s2) * CL_ROWS + rl];
        a[j] = x;
      }
      T q[CL_QB];
#pragma unroll
      for (int j = 0; j < CL_QB; j++) {
        T x = a[j];
#pragma unroll
        for (int i2 = 0; i2 < j; i2++) x = fma(q[i2], GRAM[3 * (k0 + i2) + (j - i2) - 1], x);
        q[j] = (k0 + j <= kl) ? beta_s[k0 + j] * x : T(0);
      }
      axpy4_row(Sr, (size_t)CL_LDS, ubk, n, q, lo, hi);
    }
    __syncthreads();  // UB and FPART are rewritten by the next block
  }
  {
    int lo, hi;
    split_range<SPLIT>(n, h, lo, hi);
    if (own) {
      if (r < n - 1) {
        if (lo <= n - 1 && n - 1 < hi) Sr[CL_LDS * (n - 1)] = T(0);
      } else {
        for (int c = lo; c < hi; c++) Sr[CL_LDS * c] = (c == n - 1) ? T(1) : T(0);
      }
    }
  }
  __syncthreads();
  // Q = M^T: A(c, r) = M(r, c), column r of A contiguous
  for (int idx = t; idx < CL_ROWS * n; idx += NT) {
    const int c = idx % n, l = idx / n, rr = r0 + l;
    if (rr < n) A[c + (size_t)rr * nm] = S[l + CL_LDS * c];
  }
  cl.sync();
}

}  // namespace eigb
