// Phase 1, register-resident form for 32 < n <= 32*NB (NB <= 4).
//
// Same method as eigb_tridiag.cuh (bottom-up Householder reduction of the
// reference, tred1_tiled.hpp:42-205, then M = Q^T = H_1 ... H_{n-1}), but
// the matrix never lives in shared memory: a CTA of NB*NB warps tiles the
// padded NR x NR matrix (NR = 32*NB) into 32 x 32 blocks, warp (rb, cb)
// holding rows 32*rb.. and columns 32*cb.. with one row slice of 32 values
// per lane in registers.  Shared memory only carries what every block
// needs: the reflectors (kept, zero padded, for the Q formation), the
// vector p, the per-block partial sums and the team reductions.  A step
// touches only the blocks that intersect the active leading i x i part.
#pragma once
#include <stdint.h>
#include <stdlib.h>

#include "eigb_common.cuh"

namespace eigb {

// v[i] (0 <= i < 32) for a warp-uniform (or per-lane) dynamic index, by
// selects, so that the array stays in registers: four interleaved chains
// (c = 4j + k picked by i >> 2) and a select by i & 3, nine deep with four
// values live (one chain would be 31 deep on the critical path of every
// reduction step; a full tree keeps 16 live and spills)
template <class T>
__host__ __device__ __forceinline__ T get32(const T (&v)[32], const int i)
{
  const int j = i >> 2;
  T a0 = v[0], a1 = v[1], a2 = v[2], a3 = v[3];
#pragma unroll
  for (int c = 1; c < 8; c++) {
    a0 = (j == c) ? v[4 * c] : a0;
    a1 = (j == c) ? v[4 * c + 1] : a1;
    a2 = (j == c) ? v[4 * c + 2] : a2;
    a3 = (j == c) ? v[4 * c + 3] : a3;
  }
  const T b0 = (i & 1) ? a1 : a0, b1 = (i & 1) ? a3 : a2;
  return (i & 2) ? b1 : b0;
}

// Two consecutive values from 2-element-aligned shared memory in one load.
template <class T> struct Pair;
template <> struct Pair<double> {
  using V = double2;
};
template <> struct Pair<float> {
  using V = float2;
};
template <class T>
__host__ __device__ __forceinline__ void ld2(const T *p, T &a, T &b)
{
#ifndef __CUDA_ARCH__
  // host builds (unit tests) check the alignment that the device load needs
  if (reinterpret_cast<uintptr_t>(p) % sizeof(typename Pair<T>::V) != 0) abort();
#endif
  const typename Pair<T>::V v = *reinterpret_cast<const typename Pair<T>::V *>(p);
  a = v.x;
  b = v.y;
}

// Reflectors applied per barrier in the formation of M.
constexpr int QB = 4;

// Row slice times reflector, sum_c S[c] v_c over the 32 columns of a
// block (Vc = the reflector at the block's first column).  With PIV the
// block holds the reflector pivot at column cp, whose value ul is not in
// shared memory yet: the selects substitute it (only the warps of that one
// column block take this path).
template <class T, bool PIV>
__host__ __device__ __forceinline__ T reg_symv(const T (&S)[32], const T *Vc, const int cp, const T ul)
{
  T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
#pragma unroll
  for (int c = 0; c < 32; c += 4) {
    T v0, v1, v2, v3;
    ld2(Vc + c, v0, v1);
    ld2(Vc + c + 2, v2, v3);
    if (PIV) {
      v0 = (c + 0 == cp) ? ul : v0;
      v1 = (c + 1 == cp) ? ul : v1;
      v2 = (c + 2 == cp) ? ul : v2;
      v3 = (c + 3 == cp) ? ul : v3;
    }
    a0 = fma(S[c + 0], v0, a0);
    a1 = fma(S[c + 1], v1, a1);
    a2 = fma(S[c + 2], v2, a2);
    a3 = fma(S[c + 3], v3, a3);
  }
  return (a0 + a1) + (a2 + a3);
}

// S[c] += u_c w2r + p_c ur over the block's 32 columns
template <class T>
__host__ __device__ __forceinline__ void reg_rank2(T (&S)[32], const T *Vc, const T *pc, const T ur, const T w2r)
{
#pragma unroll
  for (int c = 0; c < 32; c += 2) {
    T u0, u1, p0, p1;
    ld2(Vc + c, u0, u1);
    ld2(pc + c, p0, p1);
    S[c] = fma(p0, ur, fma(u0, w2r, S[c]));
    S[c + 1] = fma(p1, ur, fma(u1, w2r, S[c + 1]));
  }
}

template <int NB> struct RegLayout {
  static constexpr int NR = 32 * NB;
  static constexpr int NT = NR * NB;
};

// Shared-memory elements of tridiag_qt_reg: V (max(n*NR, n*(n|1)), also the
// staging area of the input and of the output), part[2*QB*NB*NR], pv[NR],
// beta[NR], red[72], gram[3*NR].
// Offset of the arrays after V, rounded to 4 elements so that the paired
// loads of V and pv stay aligned for every n.
template <int NB> __host__ __device__ inline size_t reg_voff(int n)
{
  constexpr int NR = RegLayout<NB>::NR;
  const size_t v = (size_t)n * NR > (size_t)n * (n | 1) ? (size_t)n * NR : (size_t)n * (n | 1);
  return (v + 3) & ~(size_t)3;
}
template <int NB> __host__ __device__ inline size_t reg_smem_elems(int n)
{
  constexpr int NR = RegLayout<NB>::NR;
  return reg_voff<NB>(n) + 2 * (size_t)QB * NB * NR + 2 * (size_t)NR + 72 + 3 * (size_t)NR;
}

// A: the input matrix (upper triangle used), overwritten with Q (A = Q T Q^T).
// Ap: when given, the input is read from this packed upper triangle instead
// (element (r, c), r <= c, at Ap[r + c(c+1)/2]); Q still goes to A.
template <class T, int NB, class Team>
__host__ __device__ void tridiag_qt_reg(Team &tm, T *A, const int nm, const int n, T *d_out, T *e_out, T *sm,
                                        const T *Ap = nullptr)
{
  constexpr int NR = RegLayout<NB>::NR;
  const int t = tm.rank;
  const int lane = t & 31, w = t >> 5;
  const int rb = w % NB, cb = w / NB;
  const int r = 32 * rb + lane;
  const int c0 = 32 * cb;
  const int lds = n | 1;
  T *V = sm;
  T *part = sm + reg_voff<NB>(n);
  T *pv = part + 2 * QB * NB * NR;
  T *beta_s = pv + NR;
  T *red = beta_s + NR;
  T *gram = red + 72;  // gram[3k + d - 1] = u_k . u_{k+d}

  // ---- stage the upper triangle, then build the register slices ----
  for (int idx = t; idx < n * n; idx += tm.size()) {
    const int rr = idx % n, cc = idx / n;
    if (rr <= cc) V[rr + cc * lds] = Ap ? Ap[rr + cc * (cc + 1) / 2] : A[rr + (size_t)cc * nm];
  }
  tm.sync();
  T S[32];
#pragma unroll
  for (int c = 0; c < 32; c++) {
    const int kc = c0 + c;
    S[c] = (r < n && kc < n) ? (r <= kc ? V[r + kc * lds] : V[kc + r * lds]) : T(0);
  }
  tm.sync();  // the staging area becomes the reflector store

  // ---- reduction, i = n-1 .. 1, two barriers per step ----
  // Step i applies H_i: u = rows < i of column i with the pivot u_{i-1}
  // replaced by ul, p = beta A u, alpha = beta/2 u.p, and
  // A += u w^T + w u^T with w = p + alpha u, i.e.
  //   a_rk += u_k (p_r + 2 alpha u_r) + p_k u_r = u_k w2_r + p_k u_r.
  // Schedule of step i:
  //   top      the warps of column i bring that column up to date (the
  //            rank-2 update of step i+1 restricted to it: its row i is
  //            then final, the diagonal d_i) and publish its rows < i with
  //            their partial sums of u.u;
  //   barrier  1
  //   middle   every warp applies step i+1's rank-2 update to its block
  //            (column i gets a wrong but finite value there: the
  //            reflector slot holds the raw pivot; nothing reads column i
  //            or row i of the registers after step i, since every later
  //            u and p is zero there), forms ul and beta, and its partials
  //            of A u and of u.(A u);
  //   barrier  2
  //   tail     p_r and alpha in every thread; p published for the next
  //            middle.
  // The pivot ul of step i is kept aside (gram[i], free until the
  // formation of M) and copied into the reflector after the loop, so the
  // reflector slot never changes while other warps read it; the warps of
  // its column block substitute it in registers.
  T *sg = red, *al = red + 32;  // posted partial sums: u.u and u.(A u)
  T ur = T(0), w2r = T(0);  // step i+1's u_r and w2_r (its pivot and beta are in gram, beta_s)
  T pr = T(0);              // step i+1's p_r
  for (int i = n - 1; i >= 32; --i) {
    const int cbi = i >> 5;
    // Warps past the active part (row or column block beyond cbi) stay
    // there: they keep the barriers and post the zeros their sums would be,
    // without the step's arithmetic (NB = 2 has none before step 31).
    if (NB > 2 && (rb > cbi || cb > cbi)) {
      if (cb == cbi) tm.post_zero(sg, 0);
      tm.sync();
      tm.post_zero(al, 1);
      tm.sync();
      continue;
    }
    if (cb == cbi) {
      T pi = T(0), ulp = T(0);  // p_i and the pivot of step i+1
      if (i < n - 1) {
        const int nactp = (i + 32) >> 5;
#pragma unroll
        for (int q = 0; q < NB; q++)
          if (q < nactp) pi += part[q * NR + i];
        pi *= beta_s[i + 1];
        ulp = gram[i + 1];
      }
      const T col = get32(S, i & 31) + fma(ulp, w2r, pi * ur);
      if (r == i) d_out[i] = col;
      if (i >= 1) {
        const T u0 = (r < i) ? col : T(0);
        V[(size_t)i * NR + r] = u0;
        if (r == i - 1) red[64] = u0;
        tm.post(u0 * u0, sg, 0);
      }
    }
    tm.sync();
    T *Vi = V + (size_t)i * NR;
    const bool act = (c0 < i) && (32 * rb < i);
    if (act && i < n - 1) reg_rank2<T>(S, Vi + NR + c0, pv + c0, ur, w2r);  // step i+1's update
    const T sig = tm.total(sg, 0, cbi * NB, NB);
    const T ulast = red[64];
    const T anorm = -copysign_t(sqr_t(sig), ulast);
    const T ul = ulast - anorm;
    const T beta = T(1) / flip0to1(ul * anorm);
    if (cb == cbi && r == i - 1) gram[i] = ul;
    if (t == 0) {
      e_out[i - 1] = anorm;
      beta_s[i] = beta;
    }
    const int cp = (i - 1) - c0;  // pivot column within this block, if 0 <= cp < 32
    const bool piv = (cb == ((i - 1) >> 5));
    ur = (r == i - 1) ? ul : Vi[r];  // u_r with the pivot, 0 for r >= i
    T x = T(0);
    if (act) {  // partial (A u)_r over this block's columns
      T a = piv ? reg_symv<T, true>(S, Vi + c0, cp, ul) : reg_symv<T, false>(S, Vi + c0, cp, ul);
      a = (r < i) ? a : T(0);
      part[cb * NR + r] = a;
      x = ur * a;
    }
    tm.post(x, al, 1);
    tm.sync();
    const int nact = (i + 31) >> 5;
    pr = T(0);
    if (r < i) {
#pragma unroll
      for (int q = 0; q < NB; q++)
        if (q < nact) pr += part[q * NR + r];
      pr *= beta;
    }
    if (cb == 0) pv[r] = pr;  // 0 for r >= i
    const T alpha = tm.total(al, 1, 0, NB * NB) * (beta * beta * T(0.5));
    w2r = fma(alpha + alpha, ur, pr);
  }
  // ---- steps 31 .. 0 in warp 0 ----
  // From step 31 on only the leading 32 x 32 block changes, and warp 0
  // holds all of it: the remaining steps run there with warp shuffles and
  // warp barriers, the other warps wait at the next CTA barrier.  Every
  // operation is the CTA schedule's for these steps: the partial sums of the
  // other warps are zeros (their rows and columns are past the active part),
  // so a total over them is 0 + this warp's sum, and p_i (the top's sum of
  // the posted products times beta_{i+1}) is the previous step's p_r of
  // lane i.
  if (w == 0) {
    T ulp = gram[32];  // step i+1's pivot
    T *pvb = pv;
    for (int i = 31;; --i) {
      const T pi = tm.shfl(pr, i);
      const T col = get32(S, i) + fma(ulp, w2r, pi * ur);
      if (r == i) d_out[i] = col;
      if (i == 0) break;
      const T u0 = (r < i) ? col : T(0);
      V[(size_t)i * NR + r] = u0;
      const T ulast = tm.shfl(u0, i - 1);
      const T sig = T(0) + tm.wsum(u0 * u0);
      tm.sync_warp();  // u_i stored
      reg_rank2<T>(S, V + (size_t)(i + 1) * NR, pvb, ur, w2r);  // step i+1's update
      const T anorm = -copysign_t(sqr_t(sig), ulast);
      const T ul = ulast - anorm;
      const T beta = T(1) / flip0to1(ul * anorm);
      if (r == i - 1) gram[i] = ul;
      if (r == 0) {
        e_out[i - 1] = anorm;
        beta_s[i] = beta;
      }
      ur = (r == i - 1) ? ul : u0;
      T a = reg_symv<T, true>(S, V + (size_t)i * NR, i - 1, ul);
      a = (r < i) ? a : T(0);
      const T alpha = (T(0) + tm.wsum(ur * a)) * (beta * beta * T(0.5));
      pr = (r < i) ? (T(0) + a) * beta : T(0);
      tm.sync_warp();  // every lane's reads of p_{i+1} done
      pvb[r] = pr;
      w2r = fma(alpha + alpha, ur, pr);
      ulp = ul;
    }
  }
  tm.sync();
  for (int k = 1 + t; k < n; k += tm.size()) V[(size_t)k * NR + k - 1] = gram[k];
  if (t == 0) e_out[n - 1] = T(0);
  tm.sync();

  // ---- M = H_1 ... H_{n-1}: M <- M + beta_k (M u_k) u_k^T from M = I ----
  // QB reflectors per barrier.  With a_j = M u_j for the M before the
  // block (all QB products in one exchange of partial sums), applying
  // u_0 .. u_3 in order is M += sum_j q_j u_j^T with
  //   q_j = beta_j (a_j + sum_{i<j} q_i (u_i . u_j)),
  // a recurrence per row on the Gram entries of the block, computed here
  // once for all k (each thread one pair; its walk over c starts at its
  // lane so that the threads of a warp read different banks).
  for (int idx = t; idx < 3 * n; idx += tm.size()) {
    const int k = idx / 3, d = idx % 3 + 1;
    T g = T(0);
    if (k >= 1 && k + d < n) {
      const T *u = V + (size_t)k * NR, *v = V + (size_t)(k + d) * NR;
      int c = lane % k;
      for (int j = 0; j < k; j++) {
        g = fma(u[c], v[c], g);
        c = (c + 1 == k) ? 0 : c + 1;
      }
    }
    gram[idx] = g;
  }
  T *Mr = S;
#pragma unroll
  for (int c = 0; c < 32; c++) Mr[c] = (c0 + c == r) ? T(1) : T(0);
  tm.sync();
  for (int k0 = 1, blk = 0; k0 < n; k0 += QB, blk++) {
    const int kl = min(k0 + QB - 1, n - 1);  // last reflector of the block
    T *pb = part + (blk & 1) * QB * NB * NR;  // double buffer: one barrier per block
    const bool act = (c0 < kl) && (32 * rb < kl);
    if (act) {
#pragma unroll
      for (int j = 0; j < QB; j++) {
        T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
        if (k0 + j <= kl) {
          const T *Vk = V + (size_t)(k0 + j) * NR;
#pragma unroll
          for (int c = 0; c < 32; c += 4) {
            T v0, v1, v2, v3;
            ld2(Vk + c0 + c, v0, v1);
            ld2(Vk + c0 + c + 2, v2, v3);
            a0 = fma(Mr[c + 0], v0, a0);
            a1 = fma(Mr[c + 1], v1, a1);
            a2 = fma(Mr[c + 2], v2, a2);
            a3 = fma(Mr[c + 3], v3, a3);
          }
        }
        pb[(j * NB + cb) * NR + r] = (a0 + a1) + (a2 + a3);
      }
    }
    tm.sync();
    if (act) {
      const int nact = (kl + 31) >> 5;
      T q[QB];
#pragma unroll
      for (int j = 0; j < QB; j++) {
        T a = T(0);
#pragma unroll
        for (int s = 0; s < NB; s++)
          if (s < nact) a += pb[(j * NB + s) * NR + r];
        if (k0 + j <= kl) {
#pragma unroll
          for (int i2 = 0; i2 < j; i2++) a = fma(q[i2], gram[3 * (k0 + i2) + (j - i2) - 1], a);
          q[j] = beta_s[k0 + j] * a;
        } else {
          q[j] = T(0);
        }
      }
#pragma unroll
      for (int j = 0; j < QB; j++) {
        if (k0 + j > kl) break;
        const T *Vk = V + (size_t)(k0 + j) * NR;
#pragma unroll
        for (int c = 0; c < 32; c += 2) {
          T v0, v1;
          ld2(Vk + c0 + c, v0, v1);
          Mr[c] = fma(q[j], v0, Mr[c]);
          Mr[c + 1] = fma(q[j], v1, Mr[c + 1]);
        }
      }
    }
  }
  // Q = M^T, written through the (now free) reflector store so that both
  // the shared-memory and the global accesses stay unit-stride:
  // W[x + y*lds] = M(x, y), then A(i, j) = M(j, i) = W[j + i*lds]
  tm.sync();
  if (r < n) {
#pragma unroll
    for (int c = 0; c < 32; c++)
      if (c0 + c < n) V[r + (c0 + c) * lds] = Mr[c];
  }
  tm.sync();
  for (int idx = t; idx < n * n; idx += tm.size()) {
    const int i = idx % n, j = idx / n;
    A[i + (size_t)j * nm] = V[j + i * lds];
  }
}

}  // namespace eigb
