// Batch kernels of the B200 eigensolver.
//
//   k_n1           n == 1 (eigen_GPU_batch.cu:36-54): w = a(1,1), a(1,1) = 1
//   k1_warp        phase 1 for n <= 32: one warp per matrix, 4 per CTA
//   k1_cl          phase 1 for 32 < n <= 512 on a thread-block cluster, the
//                  matrix in the cluster's distributed shared memory
//   k1_reg<NB>     phase 1 for 32 < n <= 128: one CTA per matrix, the matrix
//                  in registers (eigb_tridiag_reg.cuh)
//   k1_cta<SPLIT>  phase 1 for larger n: one CTA per matrix; the leading
//                  block that fits is staged in shared memory, the rest is
//                  reduced in place in global memory
//   k2_ql          phase 2: QL on (d, e), one matrix per thread
//   k3_warp        phase 3 for n <= 32: rotations applied to Q held in
//                  registers (one row per lane), selection-sort emulation,
//                  permuted write-back
//   k3_cta<SM>     phase 3 for n > 32: rows of Z in shared memory (a
//                  matrix's rows split over CTAs when needed) or, for the
//                  largest FP64 sizes, Z in the workspace
//   k3_tmem        phase 3 for n > 32 with rows of up to 512 32-bit
//                  columns: rows of Z in tensor memory
//   k_jacobi_warp  cyclic Jacobi for n <= 32 (jac_tiled.hpp:3-152)
//   k_check_w      FP64 residual / orthogonality gate (eigen_GPU_check.cu)
//                  on the FP64 tensor cores, one warp per matrix for
//                  n <= 32; k_check_cta (one CTA per matrix, n <= 64) and
//                  k_check_tc (128 x 128 tiles, above) the larger forms
#pragma once
#include <stdio.h>

#include "eigb_apply.cuh"
#include "eigb_common.cuh"
#include "eigb_ql.cuh"
#include "eigb_symfunc.cuh"
#include "eigb_tmem.cuh"
#include "eigb_tridiag.cuh"
#include "eigb_tridiag_cl.cuh"
#include "eigb_tridiag_reg.cuh"

namespace eigb {

// Kernel parameters (one struct for all phases; pointers already offset to
// the current chunk of matrices).
template <class T> struct KP {
  T *a;          // matrices, column-major, leading dimension nm
  T *w;          // eigenvalues, n per matrix
  T *d, *e;      // workspace: tridiagonal, n per matrix each
  Rec<T> *rec;   // workspace: rotation records, rcap per matrix
  Meta *meta;    // workspace: per-matrix status
  T *zs;         // workspace: n*n per matrix when Z does not fit in shared memory
  int k1b;       // phase 1 (CTA form): leading block kept in shared memory
  int zrows;     // phase 3 with Z in shared memory: rows per CTA ...
  int zsplit;    // ... and CTAs per matrix
  int k2mpw;     // phase 2: matrices per warp (1..32)
  const T *ap;   // packed upper-triangle input (nullptr: the upper triangle of a)
  // uneven batches: matrix k of a launch is matrix kid[k] of the caller's
  // batch, at a + aoff[kid[k]] (leading dimension nm = n), eigenvalues at
  // w + woff[kid[k]], status at info[kid[k]]; nullptr: matrix k at
  // a + k nm n, w + k n, info + k
  const int *kid;
  const long long *aoff, *woff;
  int *info;     // optional per-matrix status for the caller (may be null)
  long Lc;       // matrices in this chunk
  int n, nm;
  int rcap;
  int method;    // QL_TQL2 / QL_IMTQL2
  int max_sweep;
  int sort;
};

template <class T> __device__ __forceinline__ T *mat_ptr(const KP<T> &p, long k)
{
  return p.kid ? p.a + p.aoff[p.kid[k]] : p.a + (size_t)k * p.nm * p.n;
}
template <class T> __device__ __forceinline__ T *val_ptr(const KP<T> &p, long k)
{
  return p.kid ? p.w + p.woff[p.kid[k]] : p.w + (size_t)k * p.n;
}
template <class T> __device__ __forceinline__ void put_info(const KP<T> &p, long k, int v)
{
  if (p.info) p.info[p.kid ? p.kid[k] : k] = v;
}

// Packed upper triangle (LAPACK 'U' order): element (r, c), r <= c, at
// ap[r + c(c+1)/2]; matrix k starts at ap + k n(n+1)/2.
__host__ __device__ __forceinline__ size_t packed_size(int n) { return (size_t)n * (n + 1) / 2; }
__host__ __device__ __forceinline__ int packed_at(int r, int c) { return r + c * (c + 1) / 2; }

constexpr int K1W_NW = 4;       // warps (matrices) per CTA in k1_warp
constexpr int K2_MAX_WARPS = 8; // warps per CTA in k2_ql at most
constexpr int K1W_LD = 33;      // padded leading dimension, odd
constexpr int K3W_NW = 4;       // warps per CTA in k3_warp
constexpr int K3W_CH = 128;     // records staged per warp

// per warp: S (K1W_LD x 32), beta[32], pv[32], red[72], ubuf[4*32], gram[3*32]
template <class T> __host__ __device__ constexpr int k1w_slot() { return K1W_LD * 32 + 32 + 32 + 72 + 128 + 96; }

// threads per row in k1_cta (column ranges split across warps).  FP64
// 128 < n <= 240 takes two, which with a smaller leading block in shared
// memory (k1c_block) leaves room for two or three CTAs per SM: measured on
// B200, phase 1 in ms at four per row / two per row: n=136 20.6 / 15.9,
// n=160 27.8 / 23.5, n=192 47.8 / 41.7, n=224 34.5 / 32.4 (L=2048), n=240
// 44.2 / 42.6; at n=256 52.4 against 51.0, so four stay there.
// FP32 likewise gains from more CTAs per SM (with k1c_block's smaller
// blocks): phase 1 in ms, the largest block at four / two per row against
// the kept form: n=144 18.4 -> 11.5 (one per row, 64 x 64), n=192 32.2 ->
// 24.9 (one, 64), n=256 37.8 -> 31.6 (two, 128), n=384 75.1 -> 62.2 (two,
// 128), n=512 97.5 -> 79.8 (one, 128).
template <class T> __host__ __device__ constexpr int k1_split(int n)
{
  return sizeof(T) == 8 ? (n <= 240 ? 2 : (n <= 256 ? 4 : (n <= 512 ? 2 : 1)))
                        : (n <= 128 ? 4 : (n <= 224 ? 1 : (n <= 448 ? 2 : 1)));
}

// ---------------------------------------------------------------- n == 1
template <class T>
__global__ void k_n1(const KP<T> p)
{
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < p.Lc; k += (long)gridDim.x * blockDim.x) {
    T *A = mat_ptr(p, k);
    *val_ptr(p, k) = p.ap ? p.ap[k] : A[0];
    A[0] = T(1);
    put_info(p, k, 0);
  }
}

// ---------------------------------------------------------------- phase 1
template <class T>
__global__ void __launch_bounds__(32 * K1W_NW) k1_warp(const KP<T> p)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int wid = threadIdx.x >> 5;
  const long k = (long)blockIdx.x * K1W_NW + wid;
  if (k >= p.Lc) return;  // uniform per warp; no CTA barrier is used below
  T *S = reinterpret_cast<T *>(smem_raw) + wid * k1w_slot<T>();
  T *beta_s = S + K1W_LD * 32;
  T *pv = beta_s + 32;
  T *red = pv + 32;
  T *ubuf = red + 72;
  T *gram = ubuf + 128;
  WarpTeam tm;
  const int n = p.n, nm = p.nm, r = tm.rank;
  T *A = mat_ptr(p, k);
  const T *Ap = p.ap ? p.ap + (size_t)k * packed_size(n) : nullptr;
  for (int c = 0; c < n; c++)
    if (r <= c) S[r + c * K1W_LD] = Ap ? Ap[packed_at(r, c)] : A[r + (size_t)c * nm];
  __syncwarp();
  for (int c = 0; c < n; c++)
    if (r > c && r < n) S[r + c * K1W_LD] = S[c + r * K1W_LD];
  __syncwarp();
  tridiag_qt<T, 1>(tm, S, K1W_LD, S, K1W_LD, n, n, p.d + k * n, p.e + k * n, beta_s, pv, pv, red, ubuf, gram);
  if (r < n)
    for (int c = 0; c < n; c++) A[r + (size_t)c * nm] = S[r + c * K1W_LD];
}

// Shared-memory elements of k1_cta: red[72], beta[n], pv[n],
// part[TQ_QB*nthreads], ubuf[TQ_QB*n], gram[3n] and the leading B x B block
// of the matrix (leading dimension B|1).
__host__ __device__ inline size_t k1c_smem_elems(int n, int nthreads, int B)
{
  return 72 + 2 * (size_t)n + (size_t)TQ_QB * nthreads + (size_t)(TQ_QB + 3) * n + (size_t)B * (size_t)(B | 1);
}

// One CTA per matrix; the leading p.k1b x p.k1b block of the matrix is
// worked on in shared memory and the rest in place in a (all of it in
// shared memory when p.k1b = n).  On exit a holds Q (A = Q T Q^T): its rows
// are what phase 3 rotates.
template <class T, int SPLIT>
__global__ void __launch_bounds__(1024) k1_cta(const KP<T> p)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long k = blockIdx.x;
  const int n = p.n, nm = p.nm, t = threadIdx.x, nt = blockDim.x;
  const int B = p.k1b, ld = B | 1;
  T *A = mat_ptr(p, k);
  T *sm = reinterpret_cast<T *>(smem_raw);
  T *red = sm;          // 72
  T *beta_s = sm + 72;  // n
  T *pv = beta_s + n;   // n
  T *part = pv + n;     // TQ_QB * nt
  T *ubuf = part + TQ_QB * nt;  // TQ_QB * n
  T *gram = ubuf + TQ_QB * n;   // 3n
  T *S = gram + 3 * n;  // B x B
  // full symmetric matrix from the upper triangle: the leading block in S
  // (coalesced reads), the outer band mirrored in place (or, from a packed
  // input, written to a in both triangles)
  const T *Ap = p.ap ? p.ap + (size_t)k * packed_size(n) : nullptr;
  for (int idx = t; idx < B * B; idx += nt) {
    const int r = idx % B, c = idx / B;
    if (r <= c) S[r + c * ld] = Ap ? Ap[packed_at(r, c)] : A[r + (size_t)c * nm];
  }
  for (long idx = t; idx < (long)n * n; idx += nt) {
    const int r = (int)(idx % n), c = (int)(idx / n);
    if (Ap) {
      if (r >= B || c >= B) A[r + (size_t)c * nm] = Ap[r <= c ? packed_at(r, c) : packed_at(c, r)];
    } else if (r > c && r >= B) {
      A[r + (size_t)c * nm] = A[c + (size_t)r * nm];
    }
  }
  __syncthreads();
  for (int idx = t; idx < B * B; idx += nt) {
    const int r = idx % B, c = idx / B;
    if (r > c) S[r + c * ld] = S[c + r * ld];
  }
  __syncthreads();
  CtaTeam tm;
  tridiag_qt<T, SPLIT>(tm, S, ld, A, nm, B, n, p.d + k * n, p.e + k * n, beta_s, pv, part, red, ubuf, gram);
  // the storage holds M = Q^T; a receives Q: the leading block transposed
  // out of S, the outer band transposed in place (pairs (r, c), (c, r)
  // both lie outside the block)
  for (long idx = t; idx < (long)n * n; idx += nt) {
    const int r = (int)(idx % n), c = (int)(idx / n);
    if (r < B && c < B) {
      A[r + (size_t)c * nm] = S[c + r * ld];
    } else if (r < c) {
      const T x = A[r + (size_t)c * nm];
      A[r + (size_t)c * nm] = A[c + (size_t)r * nm];
      A[c + (size_t)r * nm] = x;
    }
  }
}

// Register-resident phase 1 for 32 < n <= 32*NB, one CTA of NB*NB warps
// per matrix (eigb_tridiag_reg.cuh).
// CTAs of k1_reg wanted per SM (registers are bounded accordingly): the
// step chain is latency-bound, and more matrices per SM pay even where the
// tighter bound costs spills.  Measured on B200 (phase 1, ms):
//   FP32 n=64: 18.8 (1 CTA/SM bound) -> 8.5 (8); n=96: 14.7 (2) -> 10.2 (3);
//   n=128: 5.7 (1) -> 4.1 (2).  FP64 n=64: 6.6 (2) -> 4.4 (4); n=96: 13.0
//   (1) -> 9.9 (2); n=128: 8.4 (1), 19.9 with 2.
template <class T> __host__ __device__ constexpr int k1r_min_blocks(int nb)
{
  return sizeof(T) == 4 ? (nb == 2 ? 8 : (nb == 3 ? 3 : 2)) : (nb == 2 ? 4 : (nb == 3 ? 2 : 1));
}

template <class T, int NB>
__global__ void __launch_bounds__(32 * NB * NB, k1r_min_blocks<T>(NB)) k1_reg(const KP<T> p)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long k = blockIdx.x;
  CtaTeam tm;
  tridiag_qt_reg<T, NB>(tm, mat_ptr(p, k), p.nm, p.n, p.d + k * p.n, p.e + k * p.n,
                        reinterpret_cast<T *>(smem_raw), p.ap ? p.ap + (size_t)k * packed_size(p.n) : nullptr);
}

// Phase 1 on a cluster of cl_cn(n) CTAs per matrix, the matrix in their
// distributed shared memory (eigb_tridiag_cl.cuh); 32 < n <= 512.
// SPLIT warps per CTA, one column range each; two CTAs per SM by registers.
constexpr int K1CL_SPLIT = 16;
template <class T, int SPLIT = K1CL_SPLIT>
__global__ void __launch_bounds__(32 * SPLIT, 1024 / (32 * SPLIT)) k1_cl(const KP<T> p)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long k = blockIdx.x / cl_cn(p.n);
  tridiag_qt_cluster<T, SPLIT>(mat_ptr(p, k), p.nm, p.n, p.d + k * p.n, p.e + k * p.n,
                               p.ap ? p.ap + (size_t)k * packed_size(p.n) : nullptr,
                               reinterpret_cast<T *>(smem_raw));
}

// ---------------------------------------------------------------- phase 2
template <class T>
__global__ void __launch_bounds__(K2_MAX_WARPS * 32) k2_ql(const KP<T> p)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // lanes 0 .. k2mpw-1 of each warp run one matrix each: fewer matrices
  // per warp spread a small batch over more warps (the chains are serial,
  // so time follows the slowest lane of a warp, and lanes diverge)
  const int mpw = p.k2mpw;
  const int lane = threadIdx.x & 31;
  if (lane >= mpw) return;  // no barriers in this kernel
  const int st = (blockDim.x >> 5) * mpw;  // matrices per block
  const int slot = (threadIdx.x >> 5) * mpw + lane;
  const long k = (long)blockIdx.x * st + slot;
  if (k >= p.Lc) return;
  const int n = p.n;
  T *dd = reinterpret_cast<T *>(smem_raw) + slot;
  T *ee = dd + (size_t)n * st;
  const T *din = p.d + k * n;
  const T *ein = p.e + k * n;
  for (int i = 0; i < n; i++) {
    dd[(size_t)i * st] = din[i];
    ee[(size_t)i * st] = ein[i];
  }
  Rec<T> *out = p.rec + (size_t)k * p.rcap;
  int ierr = 0;
  const int nr = (p.method == QL_IMTQL2) ? ql_imtql2_fast(dd, ee, st, n, out, p.rcap, p.max_sweep, &ierr)
                                         : ql_tql2_fast(dd, ee, st, n, out, p.rcap, p.max_sweep, &ierr);
  Meta mt;
  mt.nrec = nr < 0 ? 0 : nr;
  mt.pad = 0;
  if (nr < 0) {
    mt.overflow = 1;
    mt.ierr = 0;
  } else {
    mt.overflow = 0;
    mt.ierr = ierr;
    // unsorted eigenvalues over e (no longer needed): phase 3 reads them
    // from there in every CTA of the matrix, and writes w sorted
    T *wo = p.e + k * n;
    for (int i = 0; i < n; i++) wo[i] = dd[(size_t)i * st];
  }
  p.meta[k] = mt;
}

// ---------------------------------------------------------------- sorting
// Permutation of the reference's DO_SORT selection sort (tql2_tiled.hpp:
// 149-176): for distinct, non-NaN eigenvalues it is the ascending order,
// computed here by ranks in parallel; with ties or NaNs the serial
// first-strict-minimum/swap procedure is replayed exactly.
template <class T>
__device__ void select_sort_serial(const int n, T *dwork, int *pos)
{
  for (int i = 0; i < n; i++) pos[i] = i;
  for (int l = 0; l < n - 1; l++) {
    T dl = dwork[l];
    int il = l;
    for (int j = l + 1; j < n; j++) {
      const T dj = dwork[j];
      if (dl > dj) {
        dl = dj;
        il = j;
      }
    }
    if (il != l) {
      const int t = pos[l];
      pos[l] = pos[il];
      pos[il] = t;
      dwork[il] = dwork[l];
      dwork[l] = dl;
    }
  }
}

// ---------------------------------------------------------------- phase 3, n <= 32
#define EIGB_ROT(I)                                   \
  {                                                   \
    const Rec<T> rr = *rp++;                          \
    const T h0 = z[I], h1 = z[I + 1];                 \
    z[I + 1] = fma(rr.c, h1, rr.s * h0);              \
    z[I] = fma(-rr.s, h1, rr.c * h0);                 \
    if (--mm == 0) break;                             \
  }

template <class T>
__device__ __forceinline__ void apply_duff32(T (&z)[32], int cur, int mm, const Rec<T> *rp)
{
  // rotations cur, cur-1, ..., cur-mm+1 (mm >= 1, 0 <= cur <= 30)
  switch (cur) {
    case 30: EIGB_ROT(30) case 29: EIGB_ROT(29) case 28: EIGB_ROT(28) case 27: EIGB_ROT(27)
    case 26: EIGB_ROT(26) case 25: EIGB_ROT(25) case 24: EIGB_ROT(24) case 23: EIGB_ROT(23)
    case 22: EIGB_ROT(22) case 21: EIGB_ROT(21) case 20: EIGB_ROT(20) case 19: EIGB_ROT(19)
    case 18: EIGB_ROT(18) case 17: EIGB_ROT(17) case 16: EIGB_ROT(16) case 15: EIGB_ROT(15)
    case 14: EIGB_ROT(14) case 13: EIGB_ROT(13) case 12: EIGB_ROT(12) case 11: EIGB_ROT(11)
    case 10: EIGB_ROT(10) case 9: EIGB_ROT(9) case 8: EIGB_ROT(8) case 7: EIGB_ROT(7)
    case 6: EIGB_ROT(6) case 5: EIGB_ROT(5) case 4: EIGB_ROT(4) case 3: EIGB_ROT(3)
    case 2: EIGB_ROT(2) case 1: EIGB_ROT(1) case 0: EIGB_ROT(0)
    default: break;
  }
}
#undef EIGB_ROT

template <class T> struct K3WSlot {
  Rec<T> rbuf[K3W_CH];
  T sd[32], se[32], sdd[32];
  int inv[32], pos[32];
  int ierr, nrec, done;
};

// Writes sorted eigenvalues and the eigenvector columns of one matrix held
// one row per lane (z[c] = Z(lane, c)).
template <class T>
__device__ __forceinline__ void k3w_writeback(const KP<T> &p, K3WSlot<T> &sl, const long k, const T (&z)[32],
                                              const T dr, const int ierr)
{
  const int n = p.n, nm = p.nm, r = threadIdx.x & 31;
  int inv = r;
  if (p.sort && ierr == 0) {
    int cnt = 0;
    bool bad = (r < n) && (dr != dr);
    for (int q = 0; q < n; q++) {
      const T dq = __shfl_sync(0xffffffffu, dr, q);
      cnt += (dq < dr) ? 1 : 0;
      bad |= (r < n) && (q != r) && (dq == dr);
    }
    inv = cnt;
    if (__any_sync(0xffffffffu, bad)) {
      if (r < n) sl.sdd[r] = dr;
      __syncwarp();
      if (r == 0) {
        select_sort_serial(n, sl.sdd, sl.pos);
        for (int j = 0; j < n; j++) sl.inv[sl.pos[j]] = j;
      }
      __syncwarp();
      inv = (r < n) ? sl.inv[r] : r;
    }
  }
  T *A = mat_ptr(p, k);
#pragma unroll
  for (int c = 0; c < 32; c++) {
    const int dst = __shfl_sync(0xffffffffu, inv, c);
    if (c < n && r < n) A[r + (size_t)dst * nm] = z[c];
  }
  if (r < n) val_ptr(p, k)[inv] = dr;
  if (r == 0) put_info(p, k, ierr);
}

template <class T>
__global__ void __launch_bounds__(32 * K3W_NW) k3_warp(const KP<T> p)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int wid = threadIdx.x >> 5;
  const long k = (long)blockIdx.x * K3W_NW + wid;
  if (k >= p.Lc) return;
  K3WSlot<T> &sl = reinterpret_cast<K3WSlot<T> *>(smem_raw)[wid];
  const int n = p.n, nm = p.nm, r = threadIdx.x & 31;
  const T *A = mat_ptr(p, k);
  // Z = Q: phase 1 left M = Q^T in a, so Z(r, c) = M(c, r) = a[c + r*nm]
  T z[32];
#pragma unroll
  for (int c = 0; c < 32; c++) z[c] = (r < n && c < n) ? A[c + (size_t)r * nm] : T(0);

  const Meta mt = p.meta[k];
  int cur = 0, rem = 0;
  // applies one staged chunk of records (segments may continue across chunks)
  auto apply = [&](const Rec<T> *b, int nr) {
    int q = 0;
    while (q < nr) {
      if (rem == 0) {
        const Rec<T> h = b[q++];
        cur = hdr_i0(h);
        rem = hdr_cnt(h);
        continue;
      }
      const int mm = min(rem, nr - q);
      apply_duff32(z, cur, mm, b + q);
      q += mm;
      rem -= mm;
      cur -= mm;
    }
  };
  T dr;
  int ierr;
  if (!mt.overflow) {
    const Rec<T> *src = p.rec + (size_t)k * p.rcap;
    for (int base = 0; base < mt.nrec; base += K3W_CH) {
      const int cnt = min(K3W_CH, mt.nrec - base);
      for (int q = r; q < cnt; q += 32) sl.rbuf[q] = src[base + q];
      __syncwarp();
      apply(sl.rbuf, cnt);
      __syncwarp();
    }
    dr = (r < n) ? p.e[k * n + r] : T(0);
    ierr = mt.ierr;
  } else {
    // capacity exceeded in phase 2: regenerate the rotations in small chunks
    if (r < n) {
      sl.sd[r] = p.d[k * n + r];
      sl.se[r] = p.e[k * n + r];
    }
    __syncwarp();
    QLGen<T> g;
    g.pc = PC_START;
    while (true) {
      if (r == 0) {
        sl.nrec = ql_run(p.method, g, DEView<T>{sl.sd, sl.se, 1}, n, sl.rbuf, K3W_CH, p.max_sweep);
        sl.done = (g.pc == PC_DONE);
        sl.ierr = g.ierr;
      }
      __syncwarp();
      const int nr = sl.nrec;
      const int done = sl.done;
      apply(sl.rbuf, nr);
      __syncwarp();
      if (done) break;
    }
    dr = (r < n) ? sl.sd[r] : T(0);
    ierr = sl.ierr;
  }
  k3w_writeback(p, sl, k, z, dr, ierr);
}

// ---------------------------------------------------------------- phase 3, n > 32
// Records staged per buffer in k3_cta (two buffers, one being filled while
// the other is applied): room for two whole segments.
// Records per buffer: room for `sweeps` whole sweeps (and their headers),
// since a sweep is applied only once it is complete in the buffer and a
// group of sweeps (eigb_apply.cuh) only when all of it is.
__host__ __device__ inline int k3c_chunk(int n, int sweeps = 2) { return ((sweeps * (n + 1) + 63) / 64) * 64; }

template <class T> __host__ __device__ inline size_t k3c_fixed_bytes(int n, int sweeps = 2)
{
  size_t b = sizeof(Rec<T>) * 2 * (size_t)k3c_chunk(n, sweeps) + sizeof(T) * (3 * (size_t)n + 64) +
             sizeof(int) * (2 * (size_t)n + 8);
  return (b + 15) & ~(size_t)15;
}

// rows: rows of Z held in shared memory by one CTA (0: Z in the workspace)
template <class T> __host__ __device__ inline size_t k3c_smem_bytes(int n, int rows)
{
  return k3c_fixed_bytes<T>(n) + sizeof(T) * (size_t)rows * (size_t)(n | 1);
}

// Rotations K3_U at a time: the columns and records of the next block are
// loaded before the stores of the current one, so their latency overlaps
// the rotation chain (which only waits for one fma per rotation).
constexpr int K3_U = 8;

#define EIGB_CHAIN(R, Z, OUT)                     \
  {                                               \
    const T y_ = fma((R).c, h, (R).s * (Z));      \
    h = fma(-(R).s, h, (R).c * (Z));              \
    OUT = y_;                                     \
  }

// block of K3_U columns starting COFF below p, and its records from rp[RI]
#define EIGB_LOAD(ZB, RB, COFF, RI)                  \
  {                                                  \
    _Pragma("unroll") for (int u = 0; u < K3_U; u++) \
    {                                                \
      ZB[u] = p[-((COFF) + u) * cs];                 \
      RB[u] = rp[(RI) + u];                          \
    }                                                \
  }
// a block: the products that do not depend on the carried value first,
// then the chain, in which each rotation waits for a single fma
#define EIGB_BLOCK(ZB, RB)                                       \
  {                                                              \
    T cz_[K3_U], sz_[K3_U];                                      \
    _Pragma("unroll") for (int u = 0; u < K3_U; u++)             \
    {                                                            \
      cz_[u] = RB[u].c * ZB[u];                                  \
      sz_[u] = RB[u].s * ZB[u];                                  \
    }                                                            \
    _Pragma("unroll") for (int u = 0; u < K3_U; u++)             \
    {                                                            \
      const T y_ = fma(RB[u].c, h, sz_[u]);                      \
      h = fma(-RB[u].s, h, cz_[u]);                              \
      p[(1 - u) * cs] = y_;                                      \
    }                                                            \
    p -= K3_U * cs;                                              \
  }

// One segment: rotations i0, i0-1, ..., i0-len+1 (records rp[0..len)) on a
// row whose column c is zr[c*cs].  Rotation i replaces (z_i, z_{i+1}) by
// (c z_i - s z_{i+1}, s z_i + c z_{i+1}); z_{i+1} is carried in h, which
// enters as column i0+1 and leaves as column i0-len+1.  Blocks of K3_U
// rotations alternate between two register sets: while one block is
// applied, the next one's columns and records are already being loaded
// (they lie below every column the current block stores).
// seg_apply_h takes z_{i0+1} as the carried value h instead of loading it
// (a sweep that continues another one's pass).
template <class T, int CS>
__host__ __device__ __forceinline__ void seg_apply_h(T *__restrict__ zr, const int cs_rt,
                                                     const Rec<T> *__restrict__ rp, const int i0, const int len,
                                                     T h)
{
  const int cs = CS > 0 ? CS : cs_rt;
  T *p = zr + i0 * cs;  // column of the next rotation's z_i (rotation j of the segment)
  int j = 0;
  if (len >= K3_U) {
    T za[K3_U], zb[K3_U];
    Rec<T> ra[K3_U], rb[K3_U];
    EIGB_LOAD(za, ra, 0, 0)  // invariant: za/ra hold block j, j + K3_U <= len, p at rotation j
    for (; j + 3 * K3_U <= len; j += 2 * K3_U) {
      EIGB_LOAD(zb, rb, K3_U, j + K3_U)
      EIGB_BLOCK(za, ra)
      EIGB_LOAD(za, ra, K3_U, j + 2 * K3_U)  // p is at rotation j + K3_U now
      EIGB_BLOCK(zb, rb)
    }
    if (j + 2 * K3_U <= len) {
      EIGB_LOAD(zb, rb, K3_U, j + K3_U)
      EIGB_BLOCK(za, ra)
      EIGB_BLOCK(zb, rb)
      j += 2 * K3_U;
    } else {
      EIGB_BLOCK(za, ra)
      j += K3_U;
    }
  }
  for (; j < len; j++, p -= cs) {
    const T z0 = p[0];
    EIGB_CHAIN(rp[j], z0, p[cs])
  }
  p[cs] = h;
}
template <class T, int CS>
__host__ __device__ __forceinline__ void seg_apply(T *__restrict__ zr, const int cs_rt,
                                                   const Rec<T> *__restrict__ rp, const int i0, const int len)
{
  const int cs = CS > 0 ? CS : cs_rt;
  seg_apply_h<T, CS>(zr, cs_rt, rp, i0, len, zr[(i0 + 1) * cs]);
}
#undef EIGB_LOAD
#undef EIGB_BLOCK
#undef EIGB_CHAIN

// End of the last complete segment (header + rotations) in rbuf[0..cnt).
template <class T> __host__ __device__ __forceinline__ int seg_walk(const Rec<T> *rbuf, const int cnt)
{
  int q = 0;
  while (q < cnt) {
    const int L = hdr_cnt(rbuf[q]);
    if (L < 0 || q + 1 + L > cnt) break;
    q += 1 + L;
  }
  return q;
}


#define EIGB_PAIR_STEP(X, RA, RB, OUT)               \
  {                                                  \
    const T ya_ = fma((RA).c, ha, (RA).s * (X));     \
    ha = fma(-(RA).s, ha, (RA).c * (X));             \
    const T yb_ = fma((RB).c, hb, (RB).s * ya_);     \
    hb = fma(-(RB).s, hb, (RB).c * ya_);             \
    OUT = yb_;                                       \
  }

// Two consecutive sweeps from the same top i0, the first over rotations
// i0 .. i0-la+1 (records ra[0..la)), the second over i0 .. i0-len+1
// (records rb[0..len), len <= la), as a two-stage pipeline on one row: the
// second sweep trails the first by one column and takes the first's output
// from registers, so each column they share is loaded and stored once for
// both (half the shared-memory traffic of two seg_apply calls) and the two
// fma chains are independent within a step; past the second sweep's end
// the first continues alone (seg_apply_h).  Same result, rotation by
// rotation, as seg_apply(ra) followed by seg_apply(rb).
template <class T, int CS>
__host__ __device__ __forceinline__ void seg_apply_pair(T *__restrict__ zr, const int cs_rt,
                                                        const Rec<T> *__restrict__ ra, const int la,
                                                        const Rec<T> *__restrict__ rb, const int i0, const int len)
{
  const int cs = CS > 0 ? CS : cs_rt;
  T *p = zr + i0 * cs;
  T ha = p[cs];
  T hb;
  {  // first sweep, rotation i0: its output z_{i0+1} is the second sweep's carry
    const T x = p[0];
    const Rec<T> r = ra[0];
    hb = fma(r.c, ha, r.s * x);
    ha = fma(-r.s, ha, r.c * x);
  }
  p -= cs;  // at column i0 - j for step j: first sweep rotation i0-j, second i0-j+1
  int j = 1;
  constexpr int U = 4;
  if (len - 1 >= 2 * U) {
    T x[U], xn[U];
    Rec<T> a[U], b[U], an[U], bn[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      x[u] = p[-u * cs];
      a[u] = ra[j + u];
      b[u] = rb[j - 1 + u];
    }
    for (; j + 2 * U <= len; j += U) {
#pragma unroll
      for (int u = 0; u < U; u++) {  // next block, below every store of this one
        xn[u] = p[-(U + u) * cs];
        an[u] = ra[j + U + u];
        bn[u] = rb[j - 1 + U + u];
      }
#pragma unroll
      for (int u = 0; u < U; u++) EIGB_PAIR_STEP(x[u], a[u], b[u], p[(2 - u) * cs])
      p -= U * cs;
#pragma unroll
      for (int u = 0; u < U; u++) {
        x[u] = xn[u];
        a[u] = an[u];
        b[u] = bn[u];
      }
    }
    // j + U <= len: the block in registers is inside the segment
#pragma unroll
    for (int u = 0; u < U; u++) EIGB_PAIR_STEP(x[u], a[u], b[u], p[(2 - u) * cs])
    p -= U * cs;
    j += U;
  }
  for (; j < len; j++, p -= cs) {
    const T x0 = p[0];
    EIGB_PAIR_STEP(x0, ra[j], rb[j - 1], p[2 * cs])
  }
  if (la == len) {  // second sweep, last rotation i0-len+1, on the first's last value
    const Rec<T> r = rb[len - 1];
    p[2 * cs] = fma(r.c, hb, r.s * ha);
    p[cs] = fma(-r.s, hb, r.c * ha);
  } else {  // the first sweep's rotation i0-len, then the second's last, then the first alone
    const T x0 = p[0];
    const Rec<T> a = ra[len], b = rb[len - 1];
    const T ya = fma(a.c, ha, a.s * x0);
    ha = fma(-a.s, ha, a.c * x0);
    p[2 * cs] = fma(b.c, hb, b.s * ya);
    p[cs] = fma(-b.s, hb, b.c * ya);
    seg_apply_h<T, CS>(zr, cs_rt, ra + len + 1, i0 - len - 1, la - len - 1, ha);
  }
}
#undef EIGB_PAIR_STEP

// Applies the segments of rbuf[0..used) (complete, as found by seg_walk) to
// one row; two consecutive segments from the same top, the second no
// longer than the first (consecutive sweeps of the QL recurrence nest this
// way), go through seg_apply_pair.
template <class T, int CS>
__host__ __device__ __forceinline__ void apply_segments(const Rec<T> *rbuf, const int used, T *zr, const int cs)
{
  int q = 0;
  while (q < used) {
    const Rec<T> hd = rbuf[q];
    const int L = hdr_cnt(hd), i0 = hdr_i0(hd);
    const int q2 = q + 1 + L;
    if (L >= 1 && q2 < used) {
      const Rec<T> h2 = rbuf[q2];
      const int L2 = hdr_cnt(h2);
      if (hdr_i0(h2) == i0 && L2 >= 1 && L2 <= L) {  // complete within used (seg_walk)
        seg_apply_pair<T, CS>(zr, cs, rbuf + q + 1, L, rbuf + q2 + 1, i0, L2);
        q = q2 + 1 + L2;
        continue;
      }
    }
    seg_apply<T, CS>(zr, cs, rbuf + q + 1, i0, L);
    q = q2;
  }
}

template <class T, bool SM, int RPT>
__device__ __forceinline__ void apply_chunk(const Rec<T> *rbuf, const int used, const int cs, const bool (&own)[RPT],
                                            T *const (&zr)[RPT])
{
#pragma unroll
  for (int j = 0; j < RPT; j++)
    if (own[j]) {
      if (SM) apply_segments<T, 1>(rbuf, used, zr[j], 1);
      else apply_segments<T, 0>(rbuf, used, zr[j], cs);
    }
}

// Phase 1 leaves Q in a; rotations act on the rows of Q independently, so
// with Z in shared memory a matrix's rows are split over p.zsplit CTAs of
// p.zrows rows each (every CTA reads all records and only its own rows of
// a, and writes only those rows back).
// Z layout: in shared memory row-major, Z(r, c) at Z[r*(n|1) + c] (each
// thread walks its own contiguous row; at a fixed column the warp touches
// rows with an odd stride: conflict-free).  In the workspace (large n)
// column-major, Z(r, c) at Z[r + c*n], so that a warp's accesses at a fixed
// column are coalesced.
template <class T, bool SM, int RPT>
__global__ void __launch_bounds__(SM ? 256 : 512, 1) k3_cta(const KP<T> p)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int zsplit = SM ? p.zsplit : 1;
  const long k = blockIdx.x / zsplit;
  const int n = p.n, nm = p.nm, t = threadIdx.x, nt = blockDim.x;
  const int r0 = SM ? (int)(blockIdx.x % zsplit) * p.zrows : 0;
  const int nrow = SM ? min(p.zrows, n - r0) : n;
  const int ch = k3c_chunk(n);
  Rec<T> *rbuf = reinterpret_cast<Rec<T> *>(smem_raw);  // two buffers of ch records
  T *sd = reinterpret_cast<T *>(rbuf + 2 * ch);
  T *se = sd + n;
  T *sdd = se + n;
  T *red = sdd + n;
  int *inv = reinterpret_cast<int *>(red + 64);
  int *pos = inv + n;
  int *sflag = pos + n;  // [0] nrec, [1] done, [2] ierr
  T *Z;
  int rs, cs;  // element (r, c) at Z[r*rs + c*cs]
  if (SM) {
    Z = reinterpret_cast<T *>(smem_raw + k3c_fixed_bytes<T>(n));
    rs = n | 1;
    cs = 1;
  } else {
    Z = p.zs + (size_t)k * n * n;
    rs = 1;
    cs = n;
  }
  T *A = mat_ptr(p, k);
  const Meta mt = p.meta[k];
  if (!mt.overflow) {  // first chunk of records, copied while Z is loaded
    const Rec<T> *src = p.rec + (size_t)k * p.rcap;
    const int cnt = min(ch, mt.nrec);
    for (int q = t; q < cnt; q += nt) cp_async<sizeof(Rec<T>)>(rbuf + q, src + q);
    cp_async_commit();
  }
  // Z = rows r0 .. r0+nrow-1 of Q
  for (int idx = t; idx < nrow * n; idx += nt) {
    const int rr = idx % nrow, c = idx / nrow;
    Z[rr * rs + c * cs] = A[r0 + rr + (size_t)c * nm];
  }
  cp_async_wait_all();
  __syncthreads();

  bool own[RPT];
  T *zr[RPT];
#pragma unroll
  for (int j = 0; j < RPT; j++) {
    own[j] = t + j * nt < nrow;
    zr[j] = Z + (own[j] ? t + j * nt : 0) * rs;
  }
  if (!mt.overflow) {
    // double buffer: the next chunk is copied in while this one is applied
    const Rec<T> *src = p.rec + (size_t)k * p.rcap;
    int base = 0, cur = 0;
    while (base < mt.nrec) {
      Rec<T> *rb = rbuf + cur * ch;
      const int cnt = min(ch, mt.nrec - base);
      const int used = seg_walk(rb, cnt);
      const int nb = base + (used > 0 ? used : cnt);  // a segment is at most n records: used > 0
      if (nb < mt.nrec) {
        Rec<T> *nx = rbuf + (cur ^ 1) * ch;
        const int ncnt = min(ch, mt.nrec - nb);
        for (int q = t; q < ncnt; q += nt) cp_async<sizeof(Rec<T>)>(nx + q, src + nb + q);
        cp_async_commit();
      }
      apply_chunk<T, SM, RPT>(rb, used, cs, own, zr);
      cp_async_wait_all();
      __syncthreads();
      base = nb;
      cur ^= 1;
    }
    for (int c = t; c < n; c += nt) sd[c] = p.e[k * n + c];
    if (t == 0) sflag[2] = mt.ierr;
  } else {
    // capacity exceeded in phase 2: regenerate in chunks (segments are
    // closed at every chunk end, so each chunk is self-contained)
    for (int c = t; c < n; c += nt) {
      sd[c] = p.d[k * n + c];
      se[c] = p.e[k * n + c];
    }
    __syncthreads();
    QLGen<T> g;
    g.pc = PC_START;
    while (true) {
      if (t == 0) {
        sflag[0] = ql_run(p.method, g, DEView<T>{sd, se, 1}, n, rbuf, ch, p.max_sweep);
        sflag[1] = (g.pc == PC_DONE);
        sflag[2] = g.ierr;
      }
      __syncthreads();
      const int nr = sflag[0];
      const int done = sflag[1];
      apply_chunk<T, SM, RPT>(rbuf, nr, cs, own, zr);
      __syncthreads();
      if (done) break;
    }
  }
  __syncthreads();
  const int ierr = sflag[2];
  // sort permutation (inverse: destination column of each source column)
  bool bad = false;
  for (int c = t; c < n; c += nt) {
    inv[c] = c;
    if (p.sort && ierr == 0) {
      const T dc = sd[c];
      int cnt = 0;
      bad |= (dc != dc);
      for (int q = 0; q < n; q++) {
        const T dq = sd[q];
        cnt += (dq < dc) ? 1 : 0;
        bad |= (q != c) && (dq == dc);
      }
      inv[c] = cnt;
    }
  }
  if (__syncthreads_or(bad)) {
    if (t == 0) {
      for (int c = 0; c < n; c++) sdd[c] = sd[c];
      select_sort_serial(n, sdd, pos);
      for (int j = 0; j < n; j++) inv[pos[j]] = j;
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < RPT; j++)
    if (own[j]) {
      const int row = t + j * nt;
      for (int c = 0; c < n; c++) A[r0 + row + (size_t)inv[c] * nm] = Z[row * rs + c * cs];
    }
  if (r0 == 0) {
    for (int c = t; c < n; c += nt) val_ptr(p, k)[inv[c]] = sd[c];
    if (t == 0) put_info(p, k, ierr);
  }
}

// ---------------------------------------------------------------- phase 3, Z in tensor memory
// Sweeps per record buffer of k3_tmem: a full group and the next sweep
// (shared memory is not what limits that kernel).
constexpr int K3_TM_SWEEPS = K3_GROUP + 1;

// One part of k3_tmem: rows r0 .. r0+zrows-1 of one matrix, applied by the
// pn threads pt = 0 .. pn-1 of the part (row r0+pt in tensor memory at z0),
// with the shared-memory scratch of k3_cta (records double buffer, d, e,
// sort permutation; no Z) at ps and named barrier id bar.  Same steps and
// the same arithmetic as k3_cta.
template <class T, int KG>
__device__ __forceinline__ void k3_tmem_part(const KP<T> &p, const long part, const int pt, const int pn,
                                             const int bar, unsigned char *ps, const uint32_t z0)
{
  const long k = part / p.zsplit;
  const int n = p.n, nm = p.nm;
  const int r0 = (int)(part % p.zsplit) * p.zrows;
  const int nrow = min(p.zrows, n - r0);
  const int ch = k3c_chunk(n, K3_TM_SWEEPS);
  Rec<T> *rbuf = reinterpret_cast<Rec<T> *>(ps);  // two buffers of ch records
  T *sd = reinterpret_cast<T *>(rbuf + 2 * ch);
  T *se = sd + n;
  T *sdd = se + n;
  T *red = sdd + n;
  int *inv = reinterpret_cast<int *>(red + 64);
  int *pos = inv + n;
  int *sflag = pos + n;  // [0] nrec, [1] done, [2] ierr
  T *A = mat_ptr(p, k);
  const Meta mt = p.meta[k];
  const Rec<T> *src = p.rec + (size_t)k * p.rcap;
  if (!mt.overflow) {  // first chunk of records, copied while Z is loaded
    const int cnt = min(ch, mt.nrec);
    for (int q = pt; q < cnt; q += pn) cp_async<sizeof(Rec<T>)>(rbuf + q, src + q);
    cp_async_commit();
  }
  // row r0+pt of Q into tensor memory (zeros in lanes past the last row)
  const bool mine = pt < nrow;
  {
    const T *Ar = A + r0 + pt;
    int c = 0;
    for (; c + 8 <= n; c += 8) {
      T v[8];
#pragma unroll
      for (int u = 0; u < 8; u++) v[u] = mine ? Ar[(size_t)(c + u) * nm] : T(0);
#pragma unroll
      for (int u = 0; u < 8; u++) tmem_st1(tmem_at<T>(z0, c + u), v[u]);
    }
    for (; c < n; c++) tmem_st1(tmem_at<T>(z0, c), mine ? Ar[(size_t)c * nm] : T(0));
  }
  cp_async_wait_all();
  part_sync(bar, pn);

  if (!mt.overflow) {
    // double buffer: the next chunk is copied in while this one is applied
    int base = 0, cur = 0;
    while (base < mt.nrec) {
      Rec<T> *rb = rbuf + cur * ch;
      const int cnt = min(ch, mt.nrec - base);
      const int used = seg_walk(rb, cnt);
      const int nb = base + (used > 0 ? used : cnt);  // a segment is at most n records: used > 0
      if (nb < mt.nrec) {
        Rec<T> *nx = rbuf + (cur ^ 1) * ch;
        const int ncnt = min(ch, mt.nrec - nb);
        for (int q = pt; q < ncnt; q += pn) cp_async<sizeof(Rec<T>)>(nx + q, src + nb + q);
        cp_async_commit();
      }
      apply_segments_tm<T, KG>(rb, used, z0);
      cp_async_wait_all();
      part_sync(bar, pn);
      base = nb;
      cur ^= 1;
    }
    for (int c = pt; c < n; c += pn) sd[c] = p.e[k * n + c];
    if (pt == 0) sflag[2] = mt.ierr;
  } else {
    // capacity exceeded in phase 2: regenerate in chunks (segments are
    // closed at every chunk end, so each chunk is self-contained)
    for (int c = pt; c < n; c += pn) {
      sd[c] = p.d[k * n + c];
      se[c] = p.e[k * n + c];
    }
    part_sync(bar, pn);
    QLGen<T> g;
    g.pc = PC_START;
    while (true) {
      if (pt == 0) {
        sflag[0] = ql_run(p.method, g, DEView<T>{sd, se, 1}, n, rbuf, ch, p.max_sweep);
        sflag[1] = (g.pc == PC_DONE);
        sflag[2] = g.ierr;
      }
      part_sync(bar, pn);
      const int nr = sflag[0];
      const int done = sflag[1];
      apply_segments_tm<T, KG>(rbuf, nr, z0);
      part_sync(bar, pn);
      if (done) break;
    }
  }
  part_sync(bar, pn);
  const int ierr = sflag[2];
  // sort permutation (inverse: destination column of each source column)
  bool bad = false;
  for (int c = pt; c < n; c += pn) {
    inv[c] = c;
    if (p.sort && ierr == 0) {
      const T dc = sd[c];
      int cnt = 0;
      bad |= (dc != dc);
      for (int q = 0; q < n; q++) {
        const T dq = sd[q];
        cnt += (dq < dc) ? 1 : 0;
        bad |= (q != c) && (dq == dc);
      }
      inv[c] = cnt;
    }
  }
  if (part_sync_or(bar, pn, bad)) {
    if (pt == 0) {
      for (int c = 0; c < n; c++) sdd[c] = sd[c];
      select_sort_serial(n, sdd, pos);
      for (int j = 0; j < n; j++) inv[pos[j]] = j;
    }
    part_sync(bar, pn);
  }
  tmem_wait_st();  // the last segment's stores
  {
    T *Ar = A + r0 + pt;
    int c = 0;
    for (; c + 8 <= n; c += 8) {
      T v[8];
      tmem_ld8(tmem_at<T>(z0, c + 7), v);  // v[u] = column c+7-u
#pragma unroll
      for (int u = 0; u < 8; u++)
        if (mine) Ar[(size_t)inv[c + 7 - u] * nm] = v[u];
    }
    for (; c < n; c++) {
      const T v = tmem_ld1((const T *)nullptr, tmem_at<T>(z0, c));
      if (mine) Ar[(size_t)inv[c] * nm] = v;
    }
  }
  if (r0 == 0) {
    for (int c = pt; c < n; c += pn) val_ptr(p, k)[inv[c]] = sd[c];
    if (pt == 0) put_info(p, k, ierr);
  }
}

// Phase 3 with Z in tensor memory (eigb_tmem.cuh), for rows of at most
// 512 32-bit columns.  A CTA of at most four warps applies blockDim.x /
// (32 wpp) parts, wpp warps each (two parts of two warps where a part has
// at most 64 rows, so that all four lane quarters of its columns are in
// use).  Warp w keeps its 32 rows in the lanes of its sub-partition,
// 32*(w % 4) .., in the acols columns the CTA allocates.  The host sizes
// the CTA's shared memory in proportion to acols, so the CTAs that share an
// SM never hold more than its 512 columns together.
template <class T, int KG>
__global__ void __launch_bounds__(128, 1) k3_tmem(const KP<T> p, const int wpp, const int acols)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t tbase;
  const int t = threadIdx.x, w = t >> 5;
  const int pn = 32 * wpp;  // threads of a part
  const int parts = blockDim.x / pn;
  const int g = t / pn;
  const long part = (long)blockIdx.x * parts + g;
  if (w == 0) tmem_alloc(&tbase, acols);
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  const uint32_t z0 = tbase + ((uint32_t)(32 * (w & 3)) << 16);
  if (part < p.Lc * (long)p.zsplit)  // uniform per part
    k3_tmem_part<T, KG>(p, part, t - g * pn, pn, parts == 1 ? 0 : 1 + g,
                    smem_raw + (size_t)g * k3c_fixed_bytes<T>(p.n, K3_TM_SWEEPS), z0);
  // every tensor memory access of the CTA is complete (loads wait in
  // place, stores before the read-out); the allocating warp frees
  tmem_fence_before();
  __syncthreads();
  if (w == 0) {
    tmem_fence_after();
    tmem_dealloc(tbase, acols);
  }
}

// ---------------------------------------------------------------- Jacobi, n <= 32
template <class T> struct JacSlot {
  T As[32 * 33];
  T Zs[32 * 33];
  T sdd[32];
  int inv[32], pos[32];
};

template <class T>
__global__ void __launch_bounds__(32 * K1W_NW) k_jacobi_warp(const KP<T> p)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int wid = threadIdx.x >> 5;
  const long k = (long)blockIdx.x * K1W_NW + wid;
  if (k >= p.Lc) return;
  JacSlot<T> &sl = reinterpret_cast<JacSlot<T> *>(smem_raw)[wid];
  T *As = sl.As, *Zs = sl.Zs;
  const int n = p.n, nm = p.nm, r = threadIdx.x & 31;
  const bool own = r < n;
  T *A = mat_ptr(p, k);
  // full symmetric matrix from the upper triangle; Z = I
  for (int c = 0; c < 32; c++) {
    T v = T(0);
    if (own && c < n) {
      if (p.ap) v = p.ap[(size_t)k * packed_size(n) + (r <= c ? packed_at(r, c) : packed_at(c, r))];
      else v = (r <= c) ? A[r + (size_t)c * nm] : A[c + (size_t)r * nm];
    }
    As[r + c * 33] = v;
    Zs[r + c * 33] = (r == c) ? T(1) : T(0);
  }
  __syncwarp();
  T wr = As[r + r * 33];
  As[r + r * 33] = T(0);
  __syncwarp();
  const T tol = T(sizeof(T) == 4 ? 1e-10 : 1e-20);  // jac_tiled.hpp:71
  int converged = 0;
  for (int pass = 0; pass < p.max_sweep; pass++) {
    int stable = 1;
    for (int i0 = 0; i0 < n; i0++) {
      // two arg-max searches, lower index wins ties (jac_tiled.hpp:38-64)
      T x = own ? fabs_t(As[r + i0 * 33]) : T(-1);
      int ii = r;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const T xo = __shfl_xor_sync(0xffffffffu, x, o);
        const int io = __shfl_xor_sync(0xffffffffu, ii, o);
        if (xo > x || (xo == x && io < ii)) {
          x = xo;
          ii = io;
        }
      }
      T y = own ? fabs_t(As[r + ii * 33]) : T(-1);
      int jj = r;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const T yo = __shfl_xor_sync(0xffffffffu, y, o);
        const int jo = __shfl_xor_sync(0xffffffffu, jj, o);
        if (yo > y || (yo == y && jo < jj)) {
          y = yo;
          jj = jo;
        }
      }
      const int i = min(ii, jj), j = max(ii, jj);
      if (i == j) continue;
      T aij = As[j + i * 33];
      const T aii = __shfl_sync(0xffffffffu, wr, i);
      const T ajj = __shfl_sync(0xffffffffu, wr, j);
      if (fabs_t(aij) < (fabs_t(aii) + fabs_t(ajj)) * tol) continue;
      // rotation, jac_tiled.hpp:79-95
      const T alpha = T(2) * aij;
      const T beta = ajj - aii;
      const T tt = alpha / (beta + copysign_t(hypot(alpha, beta), beta));
      const T c = T(1) / hypot1(tt);
      const T s = c * tt;
      const T cc = c * c, ss = s * s, cs = -(c * s);
      aij = ((c - s) * (c + s) * aij) + cs * beta;
      const T wi = ((cc * aii) + ss * ajj) + cs * alpha;
      const T wj = (aii + ajj) - wi;
      __syncwarp();
      if (own) {
        const T aki = As[r + i * 33], akj = As[r + j * 33];
        if (r != i && r != j) {
          const T bki = c * aki - s * akj;
          const T bkj = s * aki + c * akj;
          As[i + r * 33] = bki;
          As[j + r * 33] = bkj;
          As[r + i * 33] = bki;
          As[r + j * 33] = bkj;
        } else {
          As[r + (i + j - r) * 33] = aij;
        }
        const T zki = Zs[r + i * 33], zkj = Zs[r + j * 33];
        Zs[r + i * 33] = c * zki - s * zkj;
        Zs[r + j * 33] = s * zki + c * zkj;
      }
      if (r == i) wr = wi;
      if (r == j) wr = wj;
      __syncwarp();
      stable = 0;
    }
    if (stable) {
      converged = 1;
      break;
    }
  }
  const int ierr = converged ? 0 : n + 1;
  int inv = r;
  if (p.sort) {
    int cnt = 0;
    bool bad = own && (wr != wr);
    for (int q = 0; q < n; q++) {
      const T dq = __shfl_sync(0xffffffffu, wr, q);
      cnt += (dq < wr) ? 1 : 0;
      bad |= own && (q != r) && (dq == wr);
    }
    inv = cnt;
    if (__any_sync(0xffffffffu, bad)) {
      if (own) sl.sdd[r] = wr;
      __syncwarp();
      if (r == 0) {
        select_sort_serial(n, sl.sdd, sl.pos);
        for (int q = 0; q < n; q++) sl.inv[sl.pos[q]] = q;
      }
      __syncwarp();
      inv = own ? sl.inv[r] : r;
    }
  }
  for (int c = 0; c < n; c++) {
    const int dst = __shfl_sync(0xffffffffu, inv, c);
    if (own) A[r + (size_t)dst * nm] = Zs[r + c * 33];
  }
  if (own) val_ptr(p, k)[inv] = wr;
  if (r == 0) put_info(p, k, ierr);
}

// ---------------------------------------------------------------- layouts
// Transpose of a rows x cols row-major matrix (in[r*cols + c] ->
// out[c*rows + r]) through 32 x 33 shared-memory tiles, coalesced on both
// sides.  Converts between the interleaved layout (element e of all
// matrices contiguous: x[e*L + k]) and the matrix-by-matrix one
// (x[k*E + e]), in either direction.
template <class T>
__global__ void __launch_bounds__(256) k_transpose(const long rows, const long cols, const T *__restrict__ in,
                                                   T *__restrict__ out)
{
  __shared__ T tile[32][33];
  const long r0 = (long)blockIdx.y * 32, c0 = (long)blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  for (int y = ty; y < 32; y += 8) {
    const long r = r0 + y, c = c0 + tx;
    if (r < rows && c < cols) tile[y][tx] = in[r * cols + c];
  }
  __syncthreads();
  for (int y = ty; y < 32; y += 8) {
    const long c = c0 + y, r = r0 + tx;
    if (r < rows && c < cols) out[c * rows + r] = tile[tx][y];
  }
}

// ---------------------------------------------------------------- check
// Residual ||A Z - Z D||_F and orthogonality ||Z^T Z - I||_F (off-diagonal
// terms twice) in FP64 per matrix, over the first m eigenpairs, and the
// reference's flags (eigen_GPU_check.cu:34-74): bit 0 when the residual
// exceeds max(|w_1|, |w_n|) TOL, bit 1 when the orthogonality exceeds
// n TOL.  Three forms by size: k_check_w (n <= 32), k_check_cta (n <= 64),
// k_check_tc (above).
//
// D = A B + D for one 8 x 8 tile, k = 4: this lane's A(g, q), B(q, g) and
// D(g, 2q), D(g, 2q + 1), g = lane / 4, q = lane % 4
__device__ __forceinline__ void ck_dmma(double &d0, double &d1, const double a, const double b)
{
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// k_check_cta, for 32 < n <= 64, one CTA of 4 warps per matrix: A (full
// symmetric, from the upper triangle or the packed one) and Z staged in
// shared memory as FP64 (64 x 68 each, zero padded to 64 x 64), then A Z
// (8 x 8 mma tiles, warp w the mma rows 2w and 2w + 1) and the upper
// triangle of Z^T Z (36 mma tiles, warp w the mma rows w and 7 - w from the
// diagonal rightwards, 9 tiles) on the FP64 tensor cores (mma.sync
// m8n8k4); the fragments of Z serve as the B operand of both products.
// The pitch of 68 doubles (4 mod 16) keeps the fragment loads free of bank
// conflicts.  Dynamic shared memory: check_cta_smem().
constexpr int CKC_LD = 68;
__host__ __device__ constexpr size_t check_cta_smem() { return sizeof(double) * 2 * 64 * CKC_LD; }

template <class T, bool PACKED = false>
__global__ void __launch_bounds__(128) k_check_cta(const long L, const int nm, const int n, const int m,
                                                   const T *a0, const T *w, const T *z, double *err1,
                                                   double *err2, int *flags, float *ref_flags)
{
  extern __shared__ __align__(16) unsigned char ckc_smem[];
  constexpr int LD = CKC_LD;
  __shared__ double red[8];
  const int t = threadIdx.x, wp = t >> 5, lane = t & 31;
  const int g = lane >> 2, q = lane & 3;
  double *As = reinterpret_cast<double *>(ckc_smem);  // As[i * LD + k] = A(i, k)
  double *Zs = As + 64 * LD;                          // Zs[j * LD + k] = Z(k, j)
  const int R0 = wp, R1 = 7 - wp;                     // the warp's mma rows of Z^T Z
  for (long id = blockIdx.x; id < L; id += gridDim.x) {
    const T *a = PACKED ? a0 + (size_t)id * ((size_t)n * (n + 1) / 2) : a0 + (size_t)id * nm * n;
    const T *zz = z + (size_t)id * nm * n;
    const T *d = w + (size_t)id * n;
    __syncthreads();  // the previous matrix's reads are done
    for (int idx = t; idx < 64 * 64; idx += 128) {  // zero padding past n (A) and past n, m (Z)
      const int r = idx & 63, c = idx >> 6;
      if (r >= n || c >= n) As[c * LD + r] = 0.0;
      if (r >= n || c >= m) Zs[c * LD + r] = 0.0;
    }
    // eight loads in flight per thread before their stores
    for (int i0 = 0; i0 < n * n; i0 += 8 * 128) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = i0 + u * 128 + t, r = idx % n, c = idx / n;
        v[u] = (idx < n * n && r <= c) ? (double)(PACKED ? a[r + (size_t)c * (c + 1) / 2] : a[r + (size_t)c * nm])
                                       : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = i0 + u * 128 + t, r = idx % n, c = idx / n;
        if (idx < n * n && r <= c) {
          As[c * LD + r] = v[u];
          As[r * LD + c] = v[u];
        }
      }
    }
    for (int i0 = 0; i0 < n * m; i0 += 8 * 128) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = i0 + u * 128 + t;
        v[u] = idx < n * m ? (double)zz[idx % n + (size_t)(idx / n) * nm] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = i0 + u * 128 + t;
        if (idx < n * m) Zs[(idx / n) * LD + idx % n] = v[u];
      }
    }
    __syncthreads();
    // acc[8 h + C]: A Z mma tile (2 wp + h, C); acz[C]: Z^T Z mma tile
    // (R0, C), C >= R0; acz[8 + C - 4]: (R1, C), C >= R1 (R1 >= 4)
    double acc[16][2], acz[12][2];
#pragma unroll
    for (int x = 0; x < 16; x++) acc[x][0] = acc[x][1] = 0.0;
#pragma unroll
    for (int x = 0; x < 12; x++) acz[x][0] = acz[x][1] = 0.0;
#pragma unroll 4
    for (int k0 = 0; k0 < 64; k0 += 4) {
      double af[2], zf[8];
#pragma unroll
      for (int h = 0; h < 2; h++) af[h] = As[(16 * wp + 8 * h + g) * LD + k0 + q];  // A(16 wp + 8h + g, k0 + q)
#pragma unroll
      for (int C = 0; C < 8; C++) zf[C] = Zs[(8 * C + g) * LD + k0 + q];        // Z(k0 + q, 8C + g)
      const double z0 = Zs[(8 * R0 + g) * LD + k0 + q], z1 = Zs[(8 * R1 + g) * LD + k0 + q];
#pragma unroll
      for (int h = 0; h < 2; h++)
#pragma unroll
        for (int C = 0; C < 8; C++) ck_dmma(acc[8 * h + C][0], acc[8 * h + C][1], af[h], zf[C]);
#pragma unroll
      for (int C = 0; C < 8; C++)
        if (C >= R0) ck_dmma(acz[C][0], acz[C][1], z0, zf[C]);
#pragma unroll
      for (int C = 4; C < 8; C++)
        if (C >= R1) ck_dmma(acz[4 + C][0], acz[4 + C][1], z1, zf[C]);
    }
    double e1 = 0.0, e2 = 0.0;
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int C = 0; C < 8; C++)
#pragma unroll
        for (int u = 0; u < 2; u++) {
          const int i = 16 * wp + 8 * h + g, j = 8 * C + 2 * q + u;
          if (i < n && j < m) {
            const double rr = acc[8 * h + C][u] - (double)d[j] * Zs[j * LD + i];
            e1 = fma(rr, rr, e1);
          }
        }
#pragma unroll
    for (int C = 0; C < 8; C++)
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const int j = 8 * C + 2 * q + u;
        if (C >= R0) {
          const int i = 8 * R0 + g;
          if (i < m && j < m && i <= j) {
            const double rr = acz[C][u] - (i == j ? 1.0 : 0.0);
            e2 += (i == j ? 1.0 : 2.0) * rr * rr;
          }
        }
        if (C >= 4 && C >= R1) {
          const int i = 8 * R1 + g;
          if (i < m && j < m && i <= j) {
            const double rr = acz[C >= 4 ? 4 + C : 0][u] - (i == j ? 1.0 : 0.0);
            e2 += (i == j ? 1.0 : 2.0) * rr * rr;
          }
        }
      }
    e1 = warp_sum(e1);
    e2 = warp_sum(e2);
    if (lane == 0) {
      red[wp] = e1;
      red[4 + wp] = e2;
    }
    __syncthreads();
    if (t == 0) {
      double s1 = 0.0, s2 = 0.0;
      for (int k = 0; k < 4; k++) {
        s1 += red[k];
        s2 += red[4 + k];
      }
      s1 = sqrt(s1);
      s2 = sqrt(s2);
      const double dmax = fmax(fabs((double)d[0]), fabs((double)d[n - 1]));
      const double EPS = 2.220446049250313080847e-16, eps = 1.1920928955078125e-07;
      const double TOL = (sizeof(T) == 8 ? EPS * (2 * 512 - 1) : eps * (2 * 16 - 1)) * sqrt((double)(n + 16));
      const bool f1 = s1 > dmax * TOL, f2 = s2 > n * TOL;
      if (err1) err1[id] = s1;
      if (err2) err2[id] = s2;
      if (flags) flags[id] = (f1 ? 1 : 0) | (f2 ? 2 : 0);
      if (ref_flags) {  // the reference stores the verdict into the input copy, eigen_GPU_check.cu:76-80
        float *ans = ref_flags + (size_t)id * nm * n * (sizeof(T) / sizeof(float));
        ans[0] = (float)(f1 ? s1 / dmax : 0.0);
        ans[1] = (float)(f2 ? s2 : 0.0);
        ans[2] = (float)TOL;
        ans[3] = (float)(sizeof(T) == 8 ? EPS : eps);
      }
    }
  }
}

// k_check_w, for n <= 32, one warp per matrix (4 per CTA): A (full
// symmetric, from the upper triangle or the packed one) and Z staged in
// shared memory as FP64 (per warp 2 x 32 x 36, zero padded to 32 x 32), then
// A Z (4 x 4 mma tiles) and the upper triangle of Z^T Z (10 mma tiles) on
// the FP64 tensor cores (mma.sync m8n8k4), 8 fragment loads per 26 products
// per k-step of 4: the fragments of Z serve as the B operand of A Z and as
// the A operand of Z^T Z.  The pitch of 36 doubles (4 mod 16) keeps the
// fragment loads free of bank conflicts.  Dynamic shared memory:
// check_w_smem().
constexpr int CKW_WARPS = 4;
constexpr int CKW_LD = 36;
__host__ __device__ constexpr size_t check_w_smem() { return sizeof(double) * 2 * 32 * CKW_LD * CKW_WARPS; }


template <class T, bool PACKED>
__global__ void __launch_bounds__(32 * CKW_WARPS) k_check_w(const long L, const int nm, const int n, const int m,
                                                            const T *a0, const T *w, const T *z, double *err1,
                                                            double *err2, int *flags, float *ref_flags)
{
  extern __shared__ __align__(16) unsigned char ckw_smem[];
  constexpr int LD = CKW_LD;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, q = lane & 3;
  double *As = reinterpret_cast<double *>(ckw_smem) + (size_t)wid * 2 * 32 * LD;  // As[i * LD + k] = A(i, k)
  double *Zs = As + 32 * LD;                                                       // Zs[j * LD + k] = Z(k, j)
  const long nw = (long)gridDim.x * CKW_WARPS;
  for (long id = (long)blockIdx.x * CKW_WARPS + wid; id < L; id += nw) {
    const T *a = PACKED ? a0 + (size_t)id * ((size_t)n * (n + 1) / 2) : a0 + (size_t)id * nm * n;
    const T *zz = z + (size_t)id * nm * n;
    const T *d = w + (size_t)id * n;
    __syncwarp();  // the previous matrix's reads are done
    // zero padding past n (A) and past n, m (Z)
    if (n < 32 || m < 32) {
      for (int idx = lane; idx < 32 * 32; idx += 32) {
        const int r = idx & 31, c = idx >> 5;
        if (r >= n || c >= n) As[c * LD + r] = 0.0;
        if (r >= n || c >= m) Zs[c * LD + r] = 0.0;
      }
    }
    // eight loads in flight per lane before their stores (a store to shared
    // memory would otherwise wait for each load in turn)
    for (int i0 = 0; i0 < n * n; i0 += 8 * 32) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = i0 + u * 32 + lane, r = idx % n, c = idx / n;
        v[u] = (idx < n * n && r <= c) ? (double)(PACKED ? a[r + (size_t)c * (c + 1) / 2] : a[r + (size_t)c * nm])
                                       : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = i0 + u * 32 + lane, r = idx % n, c = idx / n;
        if (idx < n * n && r <= c) {
          As[c * LD + r] = v[u];
          As[r * LD + c] = v[u];
        }
      }
    }
    for (int i0 = 0; i0 < n * m; i0 += 8 * 32) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = i0 + u * 32 + lane;
        v[u] = idx < n * m ? (double)zz[idx % n + (size_t)(idx / n) * nm] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int idx = i0 + u * 32 + lane;
        if (idx < n * m) Zs[(idx / n) * LD + idx % n] = v[u];
      }
    }
    __syncwarp();
    // acc[4 R + C]: A Z mma tile (R, C); acz[x]: Z^T Z mma tile x of the
    // upper triangle, (R, C) = (0,0) (0,1) (0,2) (0,3) (1,1) (1,2) (1,3)
    // (2,2) (2,3) (3,3)
    double acc[16][2], acz[10][2];
#pragma unroll
    for (int x = 0; x < 16; x++) acc[x][0] = acc[x][1] = 0.0;
#pragma unroll
    for (int x = 0; x < 10; x++) acz[x][0] = acz[x][1] = 0.0;
#pragma unroll
    for (int k0 = 0; k0 < 32; k0 += 4) {
      double af[4], zf[4];
#pragma unroll
      for (int R = 0; R < 4; R++) af[R] = As[(8 * R + g) * LD + k0 + q];  // A(8R + g, k0 + q)
#pragma unroll
      for (int C = 0; C < 4; C++) zf[C] = Zs[(8 * C + g) * LD + k0 + q];  // Z(k0 + q, 8C + g)
#pragma unroll
      for (int R = 0; R < 4; R++)
#pragma unroll
        for (int C = 0; C < 4; C++) ck_dmma(acc[4 * R + C][0], acc[4 * R + C][1], af[R], zf[C]);
      int x = 0;
#pragma unroll
      for (int R = 0; R < 4; R++)
#pragma unroll
        for (int C = R; C < 4; C++, x++) ck_dmma(acz[x][0], acz[x][1], zf[R], zf[C]);
    }
    double e1 = 0.0, e2 = 0.0;
#pragma unroll
    for (int R = 0; R < 4; R++)
#pragma unroll
      for (int C = 0; C < 4; C++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int i = 8 * R + g, j = 8 * C + 2 * q + h;
          if (i < n && j < m) {
            const double rr = acc[4 * R + C][h] - (double)d[j] * Zs[j * LD + i];
            e1 = fma(rr, rr, e1);
          }
        }
    {
      int x = 0;
#pragma unroll
      for (int R = 0; R < 4; R++)
#pragma unroll
        for (int C = R; C < 4; C++, x++)
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int i = 8 * R + g, j = 8 * C + 2 * q + h;
            if (i < m && j < m && i <= j) {
              const double rr = acz[x][h] - (i == j ? 1.0 : 0.0);
              e2 += (i == j ? 1.0 : 2.0) * rr * rr;
            }
          }
    }
    e1 = sqrt(warp_sum(e1));
    e2 = sqrt(warp_sum(e2));
    if (lane == 0) {
      const double dmax = fmax(fabs((double)d[0]), fabs((double)d[n - 1]));
      const double EPS = 2.220446049250313080847e-16, eps = 1.1920928955078125e-07;
      const double TOL = (sizeof(T) == 8 ? EPS * (2 * 512 - 1) : eps * (2 * 16 - 1)) * sqrt((double)(n + 16));
      const bool f1 = e1 > dmax * TOL, f2 = e2 > n * TOL;
      if (err1) err1[id] = e1;
      if (err2) err2[id] = e2;
      if (flags) flags[id] = (f1 ? 1 : 0) | (f2 ? 2 : 0);
      if (ref_flags) {  // the reference stores the verdict into the input copy, eigen_GPU_check.cu:76-80
        float *ans = ref_flags + (size_t)id * nm * n * (sizeof(T) / sizeof(float));
        ans[0] = (float)(f1 ? e1 / dmax : 0.0);
        ans[1] = (float)(f2 ? e2 : 0.0);
        ans[2] = (float)TOL;
        ans[3] = (float)(sizeof(T) == 8 ? EPS : eps);
      }
    }
  }
}

// The gate for n > 64 on the FP64 tensor cores (mma.sync m8n8k4, FP64
// operands and accumulators): one CTA of 16 warps (four per scheduler, to
// hide the latencies of the fragment loads and of the products) per matrix
// walks the 128 x 128 output tiles of A Z (all) and of Z^T Z (those on and
// above the diagonal), with 16-deep panels of A (or of Z for Z^T Z) and of
// Z staged in shared memory by cp.async, two buffers, so that the next
// panels load while the current ones are multiplied.  On an A Z tile or an
// off-diagonal Z^T Z tile warp w owns the 64 x 16 block at rows 64 (w & 1),
// columns 16 (w >> 1): 8 x 2 mma tiles, 10 fragment loads per 16 products.
// On a diagonal Z^T Z tile only the 136 mma tiles on and above the
// diagonal are needed: warps 2p and 2p + 1 share mma rows p and 15 - p (17
// tiles from the diagonal rightwards), warp 2p + h taking the columns of
// parity h, 8 or 9 tiles per warp.  KC (16 or 32) is the panel depth.
// The grid is persistent (one CTA per SM, each taking every gridDim.x-th
// matrix) so that the panel pipeline runs on across tiles and matrices.  The panels keep
// the input type (FP32 inputs widen at use).  PACKED reads A from the packed upper triangle
// (ap + id n(n+1)/2, element (r, c), r <= c, at r + c(c+1)/2) instead of
// the full layout; Z has leading dimension ldz.  Dynamic shared memory:
// checkm_smem<T, KC>().
// panel pitch, 8 mod 16 doubles: a fragment load (rows g = 0..7 at k = q =
// 0..3) and a cp.async store (rows r..r+7 at k = kq = 0..3, 4 k of a row per
// 32-byte sector of the source) both hit every bank pair twice, the least
// that 32 lanes of 8 bytes can
constexpr int CKM_LDP = 136;
template <class T, int KC> __host__ __device__ constexpr size_t checkm_smem()
{
  return sizeof(T) * 2 * 2 * KC * (size_t)CKM_LDP;
}

template <int BYTES> __device__ __forceinline__ void ck_cp_async(void *dst, const void *src, bool valid)
{
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(src), "n"(BYTES),
               "r"(valid ? BYTES : 0)
               : "memory");
}
__device__ __forceinline__ void ck_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void ck_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }


template <class T, bool PACKED, int KC>
__global__ void __launch_bounds__(512, 1) k_check_tc(const long L, const int lda, const int ldz, const int n, const int m,
                                                     const T *a0, const T *w, const T *z, double *err1, double *err2,
                                                     int *flags, float *ref_flags)
{
  constexpr int TILE = 128, LDP = CKM_LDP, PANEL = KC * LDP;
  extern __shared__ __align__(16) unsigned char ck_smem[];
  T *Pb = reinterpret_cast<T *>(ck_smem);  // [2][KC][LDP]: P(k, tile row)
  T *Qb = Pb + 2 * PANEL;                   // [2][KC][LDP]: Q(k, tile column)
  __shared__ double red[64];
  const int t = threadIdx.x, wp = t >> 5, lane = t & 31;
  const int g = lane >> 2, q = lane & 3;
  const int ntn = (n + TILE - 1) / TILE, ntm = (m + TILE - 1) / TILE;
  const int nchunks = (n + KC - 1) / KC;
  const int nres = ntn * ntm, nort = ntm * (ntm + 1) / 2, ntiles = nres + nort;
  auto tile_of = [&](const int tile, int &ti, int &tj) {
    if (tile < nres) {
      ti = tile % ntn;
      tj = tile / ntn;
    } else {
      symf_tile(tile - nres, ntm, ti, tj);
    }
  };
  // the panels of chunk c of tile `tile` of matrix `id` into buffer b;
  // out-of-range entries are zero-filled (a source of 0 bytes)
  auto load = [&](const long id, const int tile, const int c, const int b) {
    const T *a = PACKED ? a0 + (size_t)id * ((size_t)n * (n + 1) / 2) : a0 + (size_t)id * lda * n;
    const T *zz = z + (size_t)id * ldz * n;
    const bool res = tile < nres;
    int ti, tj;
    tile_of(tile, ti, tj);
    const int i0 = ti * TILE, j0 = tj * TILE, ilim = res ? n : m;
    const bool same = !res && ti == tj;  // a diagonal tile of Z^T Z: P would equal Q, only Q is loaded
    T *P = Pb + b * PANEL, *Q = Qb + b * PANEL;
    const int kc = c * KC;
#pragma unroll
    for (int u = 0; u < (KC * TILE) / 512; u++) {
      const int e = t + 512 * u;
      // 4 consecutive k of one row / column per 4 lanes, 8 rows per warp
      const int cc = 4 * (e / (4 * TILE)) + (e & 3), rr = (e >> 2) % TILE;
      const int kk = kc + cc;
      const int i = i0 + rr, j = j0 + rr;
      const bool pin = kk < n && i < ilim, qin = kk < n && j < m;
      const T *ps = zz, *qs = zz;
      if (pin) {
        if (!res) {
          ps = zz + kk + (size_t)i * ldz;  // Z(k, i)
        } else {
          const int lo = i < kk ? i : kk, hi = i < kk ? kk : i;  // A(i, k) from the upper triangle
          ps = PACKED ? a + lo + (size_t)hi * (hi + 1) / 2 : a + lo + (size_t)hi * lda;
        }
      }
      if (qin) qs = zz + kk + (size_t)j * ldz;  // Z(k, j)
      if (!same) ck_cp_async<sizeof(T)>(&P[cc * LDP + rr], ps, pin);
      ck_cp_async<sizeof(T)>(&Q[cc * LDP + rr], qs, qin);
    }
    ck_commit();
  };
  const int r0 = 64 * (wp & 1), c0 = 16 * (wp >> 1);
  const int h = wp & 1, R0 = wp >> 1, R1 = 15 - (wp >> 1);
  // The CTA takes matrices blockIdx.x, + gridDim.x, ...; the chunks of all
  // its tiles form one pipeline, so the first panels of the next tile (or
  // of the next matrix) are in flight while a tile ends and its norms are
  // taken.
  int b = 0;
  if ((long)blockIdx.x < L) load(blockIdx.x, 0, 0, 0);
  for (long id = blockIdx.x; id < L; id += gridDim.x) {
    const T *zz = z + (size_t)id * ldz * n;
    const T *d = w + (size_t)id * n;
    double s1 = 0.0, s2 = 0.0;
    for (int tile = 0; tile < ntiles; tile++) {
      const bool res = tile < nres;
      int ti, tj;
      tile_of(tile, ti, tj);
      const int i0 = ti * TILE, j0 = tj * TILE;
      const bool diag = !res && ti == tj;
      // block form: acc[2 mi + ni] for mma tile (mi, ni) of the warp's 64 x 16
      // block; diagonal form: acc[x] and acc[8 + x] for mma tiles (R0, h + 2x)
      // and (R1, h + 2x) of the tile
      double acc[16][2];
#pragma unroll
      for (int x = 0; x < 16; x++) acc[x][0] = acc[x][1] = 0.0;
      for (int c = 0; c < nchunks; c++) {
        // the next chunk of the pipeline: of this tile, of the next tile, or
        // the first of the CTA's next matrix
        bool more = true;
        if (c + 1 < nchunks) load(id, tile, c + 1, b ^ 1);
        else if (tile + 1 < ntiles) load(id, tile + 1, 0, b ^ 1);
        else if (id + gridDim.x < L) load(id + gridDim.x, 0, 0, b ^ 1);
        else more = false;
        if (more) ck_wait<1>();  // this chunk has landed (this thread's copies)
        else ck_wait<0>();
        __syncthreads();  // ... and every thread's
        const T *P = Pb + b * PANEL + q * LDP + g, *Q = Qb + b * PANEL + q * LDP + g;
        if (!diag) {
#pragma unroll
          for (int ks = 0; ks < KC; ks += 4) {
            double af[8], bf[2];
#pragma unroll
            for (int mi = 0; mi < 8; mi++) af[mi] = (double)P[ks * LDP + r0 + 8 * mi];
#pragma unroll
            for (int ni = 0; ni < 2; ni++) bf[ni] = (double)Q[ks * LDP + c0 + 8 * ni];
#pragma unroll
            for (int mi = 0; mi < 8; mi++)
#pragma unroll
              for (int ni = 0; ni < 2; ni++) ck_dmma(acc[2 * mi + ni][0], acc[2 * mi + ni][1], af[mi], bf[ni]);
          }
        } else {
#pragma unroll
          for (int ks = 0; ks < KC; ks += 4) {  // the A operand Z^T from the Q panel (P was not loaded)
            const double a0f = (double)Q[ks * LDP + 8 * R0], a1f = (double)Q[ks * LDP + 8 * R1];
            double bf[8];
#pragma unroll
            for (int x = 0; x < 8; x++) bf[x] = h + 2 * x >= R0 ? (double)Q[ks * LDP + 8 * (h + 2 * x)] : 0.0;
#pragma unroll
            for (int x = 0; x < 8; x++)
              if (h + 2 * x >= R0) ck_dmma(acc[x][0], acc[x][1], a0f, bf[x]);
#pragma unroll
            for (int x = 4; x < 8; x++)
              if (h + 2 * x >= R1) ck_dmma(acc[8 + x][0], acc[8 + x][1], a1f, bf[x]);
          }
        }
        __syncthreads();  // buffer b is free for the chunk after next
        b ^= 1;
      }
      // this lane's outputs: rows i, columns j and j + 1 of each mma tile
      auto take = [&](const int i, const int j, const double v) {
        if (res) {
          if (i < n && j < m) {
            const double rr = v - (double)d[j] * (double)zz[i + (size_t)j * ldz];
            s1 = fma(rr, rr, s1);
          }
        } else if (i < m && j < m && i <= j) {
          const double rr = v - (i == j ? 1.0 : 0.0);
          s2 += (i == j ? 1.0 : 2.0) * rr * rr;
        }
      };
      if (!diag) {
#pragma unroll
        for (int mi = 0; mi < 8; mi++)
#pragma unroll
          for (int ni = 0; ni < 2; ni++) {
            const int i = i0 + r0 + 8 * mi + g, j = j0 + c0 + 8 * ni + 2 * q;
            take(i, j, acc[2 * mi + ni][0]);
            take(i, j + 1, acc[2 * mi + ni][1]);
          }
      } else {
#pragma unroll
        for (int x = 0; x < 8; x++) {
          const int C = h + 2 * x, j = j0 + 8 * C + 2 * q;
          if (C >= R0) {
            take(i0 + 8 * R0 + g, j, acc[x][0]);
            take(i0 + 8 * R0 + g, j + 1, acc[x][1]);
          }
          if (C >= R1) {
            take(i0 + 8 * R1 + g, j, acc[8 + x][0]);
            take(i0 + 8 * R1 + g, j + 1, acc[8 + x][1]);
          }
        }
      }
    }
    s1 = warp_sum(s1);
    s2 = warp_sum(s2);
    if ((t & 31) == 0) {
      red[t >> 5] = s1;
      red[32 + (t >> 5)] = s2;
    }
    __syncthreads();
    if (t == 0) {
      double e1 = 0.0, e2 = 0.0;
      for (int k = 0; k < 16; k++) {
        e1 += red[k];
        e2 += red[32 + k];
      }
      e1 = sqrt(e1);
      e2 = sqrt(e2);
      const double dmax = fmax(fabs((double)d[0]), fabs((double)d[n - 1]));
      const double EPS = 2.220446049250313080847e-16, eps = 1.1920928955078125e-07;
      const double TOL = (sizeof(T) == 8 ? EPS * (2 * 512 - 1) : eps * (2 * 16 - 1)) * sqrt((double)(n + 16));
      const bool f1 = e1 > dmax * TOL, f2 = e2 > n * TOL;
      if (err1) err1[id] = e1;
      if (err2) err2[id] = e2;
      if (flags) flags[id] = (f1 ? 1 : 0) | (f2 ? 2 : 0);
      if (ref_flags) {
        float *ans = ref_flags + (size_t)id * lda * n * (sizeof(T) / sizeof(float));
        ans[0] = (float)(f1 ? e1 / dmax : 0.0);
        ans[1] = (float)(f2 ? e2 : 0.0);
        ans[2] = (float)TOL;
        ans[3] = (float)(sizeof(T) == 8 ? EPS : eps);
      }
    }
  }
}

template <class T>
__global__ void k_check_print(const long L, const int nm, const int n, const T *a_)
{
  for (long id = 0; id < L; id++) {
    const float *ans = reinterpret_cast<const float *>(a_ + (size_t)id * nm * n);
    if (ans[0] != 0.0f)
      printf("[%06ld] Accuracy error in the relative resisdual (||Ax-dx||_F=%le/%le/%le)\n", id, (double)ans[0],
             (double)ans[2], (double)ans[3]);
    if (ans[1] != 0.0f)
      printf("[%06ld] Orthonormality error (||ZZ-I||_F=%le/%le/%le)\n", id, (double)ans[1], (double)ans[2],
             (double)ans[3]);
  }
}

}  // namespace eigb
