// Mixed-precision solve with iterative refinement to FP64 accuracy.
//
// For each FP64 matrix A of the batch (no counterpart in the reference's
// code; its README:165,169 lists "TensorCore acceleration" and "half
// precision + iterative refinement" as future work):
//   1. shift: sigma = trace(A)/n, Af = A - sigma I (FP64, full symmetric),
//      A32 = fl32(Af)                                    (k_ref_prep)
//   2. solve A32 with the FP32 path of this library: X (FP32 eigenvectors)
//   3. refine X, per iteration (Ogita & Aishima, "Iterative refinement for
//      symmetric eigenvalue decomposition", Japan J. Indust. Appl. Math.
//      35 (2018), Algorithm 1, with the cluster treatment of their 2019
//      sequel done as a Rayleigh-Ritz step on each cluster block):
//        P = Af X, S = X^T P, G = X^T X   FP64-accurate int8 tensor-core
//                                        products (eigb_oz.cuh, 8 slices)
//        R = I - G;  lambda_i = s_ii / g_ii;  both S and R symmetrized
//        delta = max(2 (||S - diag S||_F + max|lambda| ||R||_F), 1e-7 max|lambda|)
//        clusters: runs of eigenvalues (in sorted order) with gaps <= delta
//        E_ij = (s_ij + lambda_j r_ij) / (lambda_j - lambda_i) between
//               clusters, r_ij / 2 inside a cluster      (k_oa_update)
//        X' = X + X E                    int8 tensor-core product, 5 x 4
//                                        slices (E is small)
//        per cluster c: M = S_cc + (Lambda_c R_cc + R_cc Lambda_c)/2, the
//        Rayleigh quotient of the corrected basis to first order;
//        M = W diag(mu) W^T by FP64 Jacobi (one warp); X'_c <- X'_c W,
//        lambda_c <- mu                          (k_cluster_apply)
//      A matrix has converged when n max|E_ij|^2 (all entries of E, the
//      orthonormalising r_ij/2 included) is at most tol (default 1e-14):
//      the update then leaves a loss of orthogonality of about ten times
//      that (X'^T X' - I = E^T E - ... to second order, as E + E^T = R
//      exactly; the factor ten is measured) and a residual below it.  It then leaves the later iterations.  From
//      this library's FP32 eigenvectors (max|E| about 1e-3 on the first
//      iteration for matrices with close eigenvalues, eps_32 ||A|| / gap)
//      that takes two or three iterations.
//   4. eigenvalues lambda + sigma, sorted ascending (ties in index order),
//      eigenvectors to the caller's a; matrices that did not converge in
//      max_iter iterations, or whose clusters exceed 32 eigenvalues, or
//      whose FP32 solve failed, are solved again by the plain FP64 path.
// FP64 arithmetic is used for the shift, the norms and delta, the E
// entries (the division by eigenvalue gaps), the cluster Rayleigh-Ritz and
// the accumulation of the tensor-core products.
#pragma once
#include <stdint.h>

#include "eigb_oz.cuh"

namespace eigb {

constexpr int REF_CL_MAX = 32;  // largest cluster resolved in place
constexpr double REF_DELTA_FLOOR = 1e-7;

// ----------------------------------------------------------------- shift
// One CTA (32 x 8 threads) per matrix: sigma, Af = A - sigma I and its FP32
// rounding, both full symmetric (leading dimension n), from the upper
// triangle of the caller's column-major a (leading dimension nm).
__global__ void __launch_bounds__(256) k_ref_prep(const double *__restrict__ a, const int nm, const int n,
                                                  double *__restrict__ af, float *__restrict__ a32,
                                                  double *__restrict__ sigma, const int shift)
{
  __shared__ double tile[32][33];
  __shared__ double red[8];
  const long b = blockIdx.x;
  const double *A = a + (size_t)b * nm * n;
  double *F = af + (size_t)b * n * n;
  float *F32 = a32 ? a32 + (size_t)b * n * n : nullptr;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  double tr = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) tr += A[(size_t)i * nm + i];
  for (int o = 16; o > 0; o >>= 1) tr += __shfl_xor_sync(0xffffffffu, tr, o);
  if (tx == 0) red[ty] = tr;
  __syncthreads();
  double sg = 0.0;
  for (int i = 0; i < 8; i++) sg += red[i];
  sg = shift ? sg / n : 0.0;
  if (threadIdx.x == 0 && sigma) sigma[b] = sg;
  const int T = (n + 31) / 32;
  for (int tj = 0; tj < T; tj++) {
    for (int ti = 0; ti <= tj; ti++) {
      __syncthreads();
      // tile (ti, tj) of the upper triangle: tile[c][r] = a(ti*32 + r, tj*32 + c)
      for (int cc = ty; cc < 32; cc += 8) {
        const int r = ti * 32 + tx, c = tj * 32 + cc;
        tile[cc][tx] = (r < n && c < n) ? A[(size_t)c * nm + r] : 0.0;
      }
      __syncthreads();
      // write tile (ti, tj): element (r, c); on the diagonal tile the lower
      // half comes from the mirror
      for (int cc = ty; cc < 32; cc += 8) {
        const int r = ti * 32 + tx, c = tj * 32 + cc;
        if (r < n && c < n) {
          double v = (ti < tj || tx <= cc) ? tile[cc][tx] : tile[tx][cc];
          if (r == c) v -= sg;
          F[(size_t)c * n + r] = v;
          if (F32) F32[(size_t)c * n + r] = (float)v;
        }
      }
      if (ti < tj) {  // the mirror tile (tj, ti): element (c, r) = a(r, c)
        for (int rr = ty; rr < 32; rr += 8) {
          const int row = tj * 32 + tx, col = ti * 32 + rr;  // row = original column index
          if (row < n && col < n) {
            const double v = tile[tx][rr];
            F[(size_t)col * n + row] = v;
            if (F32) F32[(size_t)col * n + row] = (float)v;
          }
        }
      }
    }
  }
}

// ----------------------------------------------------------------- update
struct RefP {
  int n;
  const double *S, *G;  // n x n per matrix, column-major
  double *E;            // n x n per matrix, column-major (may alias nothing read here)
  double *lam;          // n per matrix: eigenvalue estimates (shifted)
  int *order;           // n per matrix: indices by ascending estimate
  int *cl;              // n per matrix: at the sorted position where a cluster of size >= 2 starts, its size
  double *W;            // n * REF_CL_MAX per matrix: cluster rotations
  const int *act_in;    // active in this iteration
  int *act_out;         // active in the next iteration
  int *conv_it;         // iteration at which the matrix converged (0: not yet)
  int *fail;            // 1: to be solved by the fallback
  double *emax;         // max |E_ij|, per matrix (diagnostic)
  double tol;
  int it;               // this iteration (1-based)
  int last;             // 1 on the last iteration
};

__device__ __forceinline__ double blk_sum(double v, double *red)
{
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += red[i];
  return s;
}
__device__ __forceinline__ double blk_max(double v, double *red)
{
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < (int)(blockDim.x >> 5); i++) s = fmax(s, red[i]);
  return s;
}

// Jacobi on the k x k symmetric matrix M (row-major in M[p*33 + q], k <=
// 32) by one warp, in the round-robin parallel ordering: each round turns
// k/2 disjoint pairs at once, lanes < k/2 forming one rotation each, and
// the warp applies them to M from both sides in one pass over the 2 x 2
// blocks of the pairs (rows, then columns, each entry read and written
// once) and to V's columns.  A pair whose off-diagonal entry is at rounding
// level (|m_pq| <= 1.1e-16 (|m_pp| + |m_qq|) / 2) is left alone; a sweep
// without a rotation ends it, at most 30 sweeps.  V (same layout)
// receives the eigenvectors (columns), M's diagonal the eigenvalues.  PQ
// (32 ints) and CS (32 doubles) hold the round's pairs and rotations.
__device__ void warp_jacobi(double *M, double *V, const int k, int *PQ, double *CS)
{
  const int l = threadIdx.x & 31;
  for (int q = 0; q < k; q++)
    if (l < k) V[l * 33 + q] = (l == q) ? 1.0 : 0.0;
  const int np = (k + 1) & ~1, m = np - 1, half = np / 2;
  __syncwarp();
  for (int sweep = 0; sweep < 30; sweep++) {
    int rotated = 0;
    for (int r = 0; r < m; r++) {
      int rot = 0;
      if (l < half) {
        int p = l == 0 ? r : (r + l) % m, q = l == 0 ? m : (r - l + m) % m;
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        double c = 1.0, sn = 0.0;
        if (q < k) {
          const double app = M[p * 33 + p], aqq = M[q * 33 + q], apq = M[p * 33 + q];
          if (fabs(apq) > 1.1e-16 * 0.5 * (fabs(app) + fabs(aqq))) {
            rot = 1;
            const double th = (aqq - app) / (2.0 * apq);
            const double t = (fabs(th) > 1e150) ? 0.5 / th : copysign(1.0, th) / (fabs(th) + sqrt(fma(th, th, 1.0)));
            c = 1.0 / sqrt(fma(t, t, 1.0));
            sn = t * c;
          }
        }
        PQ[2 * l] = p;
        PQ[2 * l + 1] = q;
        CS[2 * l] = c;
        CS[2 * l + 1] = sn;
      }
      rotated |= __any_sync(0xffffffffu, rot);
      __syncwarp();
      for (int idx = l; idx < half * half; idx += 32) {
        const int ka = idx / half, kb = idx % half;
        const int p = PQ[2 * ka], q = PQ[2 * ka + 1], p2 = PQ[2 * kb], q2 = PQ[2 * kb + 1];
        const double ca = CS[2 * ka], sa = CS[2 * ka + 1], cb = CS[2 * kb], sb = CS[2 * kb + 1];
        if (q < k && q2 < k) {
          const double b00 = M[p * 33 + p2], b01 = M[p * 33 + q2], b10 = M[q * 33 + p2], b11 = M[q * 33 + q2];
          const double r00 = ca * b00 - sa * b10, r10 = sa * b00 + ca * b10;  // rows p, q
          const double r01 = ca * b01 - sa * b11, r11 = sa * b01 + ca * b11;
          M[p * 33 + p2] = cb * r00 - sb * r01;  // columns p2, q2
          M[p * 33 + q2] = sb * r00 + cb * r01;
          M[q * 33 + p2] = cb * r10 - sb * r11;
          M[q * 33 + q2] = sb * r10 + cb * r11;
        } else if (q2 < k) {  // pair ka is the dummy of odd k: only the columns turn
          const double b0 = M[p * 33 + p2], b1 = M[p * 33 + q2];
          M[p * 33 + p2] = cb * b0 - sb * b1;
          M[p * 33 + q2] = sb * b0 + cb * b1;
        } else if (q < k) {  // pair kb is the dummy: only the rows turn
          const double b0 = M[p * 33 + p2], b1 = M[q * 33 + p2];
          M[p * 33 + p2] = ca * b0 - sa * b1;
          M[q * 33 + p2] = sa * b0 + ca * b1;
        }
      }
      for (int idx = l; idx < k * half; idx += 32) {  // columns of V
        const int row = idx / half, kb = idx % half;
        const int p2 = PQ[2 * kb], q2 = PQ[2 * kb + 1];
        if (q2 < k) {
          const double cb = CS[2 * kb], sb = CS[2 * kb + 1];
          const double v0 = V[row * 33 + p2], v1 = V[row * 33 + q2];
          V[row * 33 + p2] = cb * v0 - sb * v1;
          V[row * 33 + q2] = sb * v0 + cb * v1;
        }
      }
      __syncwarp();
      if (rot) {  // the pair's off-diagonal entries, annihilated up to rounding, set exactly
        const int p = PQ[2 * l], q = PQ[2 * l + 1];
        M[p * 33 + q] = M[q * 33 + p] = 0.0;
      }
      __syncwarp();
    }
    if (!rotated) break;
  }
}

// One CTA (256 threads) per matrix.  Dynamic shared memory: ref_update_smem(n).
constexpr int REF_JW = 2;  // warps that run the cluster Jacobi (their scratch bounds the CTAs per SM)
__host__ __device__ inline size_t ref_update_smem(int n)
{
  return sizeof(double) * ((size_t)n + REF_JW * (2 * 32 * 33 + 64)) + sizeof(int) * 4 * (size_t)n + 64;
}

__global__ void __launch_bounds__(256) k_oa_update(const RefP p)
{
  extern __shared__ __align__(16) unsigned char ru_smem[];
  const long b = blockIdx.x;
  if (!p.act_in[b]) {  // inactive stays inactive (the flags alternate between two arrays)
    if (threadIdx.x == 0) p.act_out[b] = 0;
    return;
  }
  const int n = p.n;
  double *lam = reinterpret_cast<double *>(ru_smem);
  double *jw = lam + n;  // REF_JW warps x (M, V of 32 x 33, CS of 32, PQ of 32 ints)
  int *ord = reinterpret_cast<int *>(jw + REF_JW * (2 * 32 * 33 + 64));
  int *cid = ord + n;
  int *csz = cid + n;
  int *cst = csz + n;  // sorted start positions of the clusters of 2 .. REF_CL_MAX
  __shared__ double red[8];
  __shared__ int bad, ncl;
  const double *S = p.S + (size_t)b * n * n;
  const double *G = p.G + (size_t)b * n * n;
  double *E = p.E + (size_t)b * n * n;
  const int tid = threadIdx.x;
  if (tid == 0) bad = 0;
  for (int i = tid; i < n; i += 256) {
    const double v = S[(size_t)i * n + i] / G[(size_t)i * n + i];
    if (!(fabs(v) <= 1.7976931348623157e308)) bad = 1;  // NaN or Inf: the matrix goes to the fallback
    lam[i] = v;
  }
  __syncthreads();
  double off = 0.0, rn = 0.0, am = 0.0;
  for (int i = tid; i < n; i += 256) am = fmax(am, fabs(lam[i]));
  for (long idx = tid; idx < (long)n * n; idx += 256) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    const double s = 0.5 * (S[(size_t)j * n + i] + S[(size_t)i * n + j]);
    const double r = (i == j ? 1.0 : 0.0) - 0.5 * (G[(size_t)j * n + i] + G[(size_t)i * n + j]);
    if (i != j) off += s * s;
    rn += r * r;
  }
  off = blk_sum(off, red);
  rn = blk_sum(rn, red);
  am = blk_max(am, red);
  // eigenvalues closer than 1e-7 max|lambda| always go through the cluster
  // Rayleigh-Ritz step (exact in S and R) rather than the division by
  // their gap, whatever the iteration's corrections
  double delta = 2.0 * (sqrt(off) + am * sqrt(rn));
  if (!(delta <= 1.7976931348623157e308) || !(am <= 1.7976931348623157e308)) {  // NaN or Inf
    if (tid == 0) bad = 1;
  }
  delta = delta > REF_DELTA_FLOOR * am ? delta : REF_DELTA_FLOOR * am;
  __syncthreads();
  if (bad) {  // not finite: no ordering, clusters or update; the fallback solves it
    if (tid == 0) {
      p.emax[b] = 0.0;
      p.act_out[b] = 0;
      p.fail[b] = 1;
    }
    return;
  }
  // ascending order of the estimates (ties by index)
  for (int i = tid; i < n; i += 256) {
    const double li = lam[i];
    int rk = 0;
    for (int j = 0; j < n; j++) {
      const double lj = lam[j];
      rk += (lj < li || (lj == li && j < i)) ? 1 : 0;
    }
    ord[rk] = i;
  }
  __syncthreads();
  if (tid == 0) {  // clusters: runs of gaps <= delta in sorted order
    int c = 0, start = 0;
    for (int k = 0; k < n; k++) {
      if (k > 0 && lam[ord[k]] - lam[ord[k - 1]] > delta) {
        csz[start] = k - start;
        start = k;
        c++;
      }
      cid[ord[k]] = c;
      if (k > start) csz[k] = 0;
    }
    csz[start] = n - start;
    int nc = 0;
    for (int k = 0; k < n; k++) {
      if (csz[k] > REF_CL_MAX) bad = 1;
      if (csz[k] >= 2 && csz[k] <= REF_CL_MAX) cst[nc++] = k;
    }
    ncl = nc;
  }
  __syncthreads();
  // E, and its largest entry: the update leaves errors of the order of its
  // square, from the division by gaps and from the orthonormalisation
  // (r/2) alike
  double em = 0.0;
  for (long idx = tid; idx < (long)n * n; idx += 256) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    const double s = 0.5 * (S[(size_t)j * n + i] + S[(size_t)i * n + j]);
    const double r = (i == j ? 1.0 : 0.0) - 0.5 * (G[(size_t)j * n + i] + G[(size_t)i * n + j]);
    const double e = (cid[i] == cid[j]) ? 0.5 * r : (s + lam[j] * r) / (lam[j] - lam[i]);
    em = fmax(em, fabs(e));
    E[(size_t)j * n + i] = e;
  }
  em = blk_max(em, red);
  // cluster Rayleigh-Ritz: one warp per cluster of 2 .. REF_CL_MAX, the
  // first REF_JW warps
  const int warp = tid >> 5, l = tid & 31;
  double *M = jw + (warp % REF_JW) * (2 * 32 * 33 + 64), *V = M + 32 * 33, *CS = V + 32 * 33;
  int *PQ = reinterpret_cast<int *>(CS + 32);
  for (int c = warp; warp < REF_JW && c < ncl; c += REF_JW) {
    const int k0 = cst[c], sz = csz[k0];
    for (int q = 0; q < sz; q++) {
      if (l < sz) {
        const int ip = ord[k0 + l], iq = ord[k0 + q];
        const double s = 0.5 * (S[(size_t)iq * n + ip] + S[(size_t)ip * n + iq]);
        const double r = (ip == iq ? 1.0 : 0.0) - 0.5 * (G[(size_t)iq * n + ip] + G[(size_t)ip * n + iq]);
        M[l * 33 + q] = s + 0.5 * (lam[ip] + lam[iq]) * r;
      }
    }
    __syncwarp();
    warp_jacobi(M, V, sz, PQ, CS);
    if (l == 0) {
      // ascending eigenvalues within the cluster: column q of W is the
      // eigenvector of the q-th smallest; it replaces member ord[k0 + q]
      int perm[REF_CL_MAX];
      for (int q = 0; q < sz; q++) perm[q] = q;
      for (int q = 1; q < sz; q++) {  // insertion sort, sz <= 32
        const int v = perm[q];
        int u = q;
        while (u > 0 && M[perm[u - 1] * 33 + perm[u - 1]] > M[v * 33 + v]) {
          perm[u] = perm[u - 1];
          u--;
        }
        perm[u] = v;
      }
      double *Wc = p.W + ((size_t)b * n + k0) * REF_CL_MAX;
      for (int q = 0; q < sz; q++) {
        const int pq = perm[q];
        for (int pp = 0; pp < sz; pp++) Wc[(size_t)q * REF_CL_MAX + pp] = V[pp * 33 + pq];
        lam[ord[k0 + q]] = M[pq * 33 + pq];
      }
    }
    __syncwarp();
  }
  __syncthreads();
  for (int i = tid; i < n; i += 256) {
    p.lam[(size_t)b * n + i] = lam[i];
    p.order[(size_t)b * n + i] = ord[i];
    p.cl[(size_t)b * n + i] = (csz[i] >= 2 && csz[i] <= REF_CL_MAX) ? csz[i] : 0;
  }
  if (tid == 0) {
    const bool fin = !bad && em <= 1.7976931348623157e308;
    const bool conv = fin && (double)n * em * em <= p.tol;
    p.emax[b] = em;
    if (conv) p.conv_it[b] = p.it;
    const bool more = fin && !conv && !p.last;
    p.act_out[b] = more ? 1 : 0;
    if (!fin || (!conv && p.last)) p.fail[b] = 1;
  }
}

// ----------------------------------------------------------- cluster apply
// X'_c <- X'_c W for every cluster of the matrix; one CTA per matrix, one
// row of X' per thread.
__global__ void __launch_bounds__(256) k_cluster_apply(const int n, double *__restrict__ X, const int *__restrict__ act,
                                                       const int *__restrict__ fail, const int *__restrict__ order,
                                                       const int *__restrict__ cl, const double *__restrict__ W,
                                                       int *__restrict__ err)
{
  __shared__ double ws[REF_CL_MAX * REF_CL_MAX];
  __shared__ int mem[REF_CL_MAX];
  const long b = blockIdx.x;
  if (!act[b] || fail[b]) return;
  double *Xb = X + (size_t)b * n * n;
  __shared__ int badidx;
  for (int k0 = 0; k0 < n; k0++) {
    const int sz = cl[(size_t)b * n + k0];
    if (sz < 2) continue;
    __syncthreads();
    if (threadIdx.x == 0) badidx = (sz > REF_CL_MAX || k0 + sz > n) ? 1 : 0;
    __syncthreads();
    if (badidx) {  // an inconsistent cluster table: record it, leave X as it is
      if (threadIdx.x == 0 && err) atomicExch(err, 1);
      return;
    }
    // the entries past the cluster's size in each column of W are never
    // written: zeros here, so that the products below (over all
    // REF_CL_MAX slots) never meet whatever the workspace held
    for (int u = threadIdx.x; u < sz * REF_CL_MAX; u += blockDim.x)
      ws[u] = (u % REF_CL_MAX) < sz ? W[((size_t)b * n + k0) * REF_CL_MAX + u] : 0.0;
    if (threadIdx.x < sz) {
      const int m = order[(size_t)b * n + k0 + threadIdx.x];
      mem[threadIdx.x] = m;
      if (m < 0 || m >= n) atomicExch(&badidx, 1);
    }
    __syncthreads();
    if (badidx) {
      if (threadIdx.x == 0 && err) atomicExch(err, 1);
      return;
    }
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
      double x[REF_CL_MAX];
#pragma unroll
      for (int pp = 0; pp < REF_CL_MAX; pp++) x[pp] = (pp < sz) ? Xb[(size_t)mem[pp] * n + r] : 0.0;
      for (int q = 0; q < sz; q++) {
        double y = 0.0;
#pragma unroll
        for (int pp = 0; pp < REF_CL_MAX; pp++) y = fma(x[pp], ws[q * REF_CL_MAX + pp], y);
        Xb[(size_t)mem[q] * n + r] = y;
      }
    }
  }
}

// ------------------------------------------------------------------ final
// One CTA per matrix: converged matrices get their eigenvalues (+ sigma)
// ascending, ties in index order, and the matching eigenvectors written to
// the caller's a (leading dimension nm) from the buffer of the iteration
// they converged in; the others are appended to the fallback list.
__global__ void __launch_bounds__(256) k_ref_final(const int n, const int nm, double *__restrict__ a,
                                                   double *__restrict__ w, int *__restrict__ info,
                                                   const double *__restrict__ X0, const double *__restrict__ X1,
                                                   const double *__restrict__ lamv, const double *__restrict__ sigma,
                                                   const int *__restrict__ conv_it, const int *__restrict__ fail,
                                                   int *__restrict__ iters, int *__restrict__ fb_list,
                                                   int *__restrict__ fb_count, const long gofs)
{
  extern __shared__ __align__(16) unsigned char rf_smem[];
  double *lam = reinterpret_cast<double *>(rf_smem);
  int *rank = reinterpret_cast<int *>(lam + n);
  const long b = blockIdx.x;
  const int ci = conv_it[b];
  if (fail[b] || ci == 0) {
    if (threadIdx.x == 0) {
      fb_list[atomicAdd(fb_count, 1)] = (int)(gofs + b);
      if (iters) iters[gofs + b] = 0;
    }
    return;
  }
  const double sg = sigma[b];
  for (int i = threadIdx.x; i < n; i += blockDim.x) lam[i] = lamv[(size_t)b * n + i] + sg;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double li = lam[i];
    int rk = 0;
    for (int j = 0; j < n; j++) rk += (lam[j] < li || (lam[j] == li && j < i)) ? 1 : 0;
    rank[i] = rk;
    w[(size_t)(gofs + b) * n + rk] = li;
  }
  __syncthreads();
  const double *X = ((ci - 1) & 1) ? X1 : X0;
  X += (size_t)b * n * n;
  double *A = a + (size_t)(gofs + b) * nm * n;
  for (int i = 0; i < n; i++) {
    const int rk = rank[i];
    for (int r = threadIdx.x; r < n; r += blockDim.x) A[(size_t)rk * nm + r] = X[(size_t)i * n + r];
  }
  if (threadIdx.x == 0) {
    if (info) info[gofs + b] = 0;
    if (iters) iters[gofs + b] = ci;
  }
}

// initial state of a chunk: active unless the FP32 solve failed
__global__ void k_ref_init(const long L, const int *__restrict__ info32, int *__restrict__ act, int *__restrict__ conv_it,
                           int *__restrict__ fail)
{
  for (long b = blockIdx.x * (long)blockDim.x + threadIdx.x; b < L; b += (long)gridDim.x * blockDim.x) {
    const int ok = info32[b] == 0;
    act[b] = ok;
    conv_it[b] = 0;
    fail[b] = ok ? 0 : 1;
  }
}

// matrices left unsolved when the fallback is off: info = -1
__global__ void k_ref_mark(const int cnt, const int *__restrict__ list, int *__restrict__ info)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < cnt && info) info[list[k]] = -1;
}

// offsets of the fallback's index list: matrix k at a + k nm n, w + k n
__global__ void k_ref_offsets(const long L, const int nm, const int n, long long *__restrict__ aoff,
                              long long *__restrict__ woff)
{
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < L; k += (long)gridDim.x * blockDim.x) {
    aoff[k] = (long long)k * nm * n;
    woff[k] = (long long)k * n;
  }
}

}  // namespace eigb
