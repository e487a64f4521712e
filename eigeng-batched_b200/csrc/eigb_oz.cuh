// FP64-accurate batched matrix products on the int8 tensor cores
// (tcgen05.mma kind::i8), by exact integer splitting (Ozaki's scheme).
//
// Operands.  A product C = L_op R_op^T is taken between two operands of R
// rows by K columns each (both "K-major": an operand row is the K-vector
// that one output row or column is formed from).  Each operand row r is
// scaled by a power of two 2^e_r with max_k |x(r,k)| < 2^e_r and cut into s
// integer slices,
//     x(r,k) = 2^e_r * sum_{i=1..s} q_i(r,k) * 2^-(6 + 7(i-1)),
// q_i in [-64, 64]: q_1 = rint(x 2^(6-e)), then each remainder (|t| <= 1/2)
// times 2^7 rounds to the next slice.  Every step is exact in FP64, so the
// slices hold x to 6 + 7(s-1) bits below the row's largest element.
//
// Products.  Slice products q_i^L . q_j^R are integer dot products over K
// with |q_i q_j| <= 2^12, so for K <= 256 each partial sum stays below
// 2^20 and a sum of up to eight of them below 2^23: the int32 tensor-core
// accumulation is exact.  The products of one "diagonal" d = i + j share
// the scale 2^-(12 + 7(d-2)) and accumulate into one TMEM accumulator;
// diagonals up to dmax are kept (the dropped terms lie below
// 2^-(12 + 7(dmax-1)) of the row/column maxima).  The epilogue combines the
// diagonals in FP64 from the least significant (Horner, factor 2^-7) and
// scales by 2^(e_r + e_c - 12).  With s = 8 and dmax = 9 (36 slice
// products) the result is accurate to FP64 rounding relative to
// |L row| |R row|, like an FP64 GEMM.
//
// Layout of a slice in global memory (and, per K-block, in shared memory):
// the "no swizzle" K-major canonical layout of tcgen05, in core matrices of
// 8 rows x 16 bytes.  For a slice of Rp rows (a multiple of 128) and Kp
// columns (a multiple of KB), element (r, k) is at byte
//     (k / KB) * Rp*KB + (r / 8) * 8*KB + ((k % KB) / 16) * 128 + (r % 8) * 16 + k % 16
// so the 128 rows of an M tile (or the 64 of an N tile) of one K-block are
// one contiguous run of bytes, copied to shared memory by one bulk copy
// (cp.async.bulk, no tensor map).  The shared-memory descriptor of an MMA
// step (K = 32 bytes) then has LBO = 128 bytes (the two 16-byte K chunks)
// and SBO = 8*KB bytes (consecutive 8-row groups).
//
// The kernel (k_oz_gemm): one CTA of four warps per (matrix, 128-row M
// tile, 64-column N tile).  Warp 0 lane 0 issues the bulk copies of a
// K-block's slices, warp 1 lane 0 issues the MMAs (cta_group::1, M = 128,
// N = 64, K = 32) into (dmax - 1) accumulators of 64 TMEM columns, then all
// four warps read the accumulators back (tcgen05.ld 32x32b, one TMEM lane =
// one output row per thread) and write FP64 results.  Every wait on an
// mbarrier is bounded; on timeout the kernel records an error and finishes
// without touching its outputs.
#pragma once
#include <stdint.h>

#include "eigb_tmem.cuh"

namespace eigb {

constexpr int OZ_NT = 64;          // N tile (columns of the output per CTA)
constexpr int OZ_MT = 128;         // M tile (rows of the output per CTA)
constexpr int OZ_THREADS = 128;
constexpr int OZ_TMEM_COLS = 512;
constexpr unsigned OZ_WAIT_LIMIT = 1u << 22;  // try_wait polls before giving up

// Padded sizes of the slice layout for order n.
__host__ __device__ inline int oz_rp(int n) { return ((n + OZ_MT - 1) / OZ_MT) * OZ_MT; }
__host__ __device__ inline int oz_kp(int n) { return n <= 128 ? ((n + 31) / 32) * 32 : ((n + 127) / 128) * 128; }
__host__ __device__ inline int oz_kb(int n) { return n <= 128 ? oz_kp(n) : 128; }
__host__ __device__ inline size_t oz_slice_bytes(int n) { return (size_t)oz_rp(n) * oz_kp(n); }

__host__ __device__ inline size_t oz_offset(int r, int k, int Rp, int KB)
{
  return (size_t)(k / KB) * Rp * KB + (size_t)(r >> 3) * 8 * KB + ((k % KB) >> 4) * 128 + (r & 7) * 16 + (k & 15);
}

// ------------------------------------------------------------------ slicing
//
// Operand row r of matrix b, element k, is src[b*bs + r*rs + k*ks]
// (r < R, k < K; zero outside).  Writes s slices at
// out + (b*s + i) * Rp*Kp and the exponents e[b*Rp + r].  One thread per
// (row, 16-column chunk); rows fastest across the threads of a block.
struct OzSlice {
  const void *src;
  int src_f32;        // 1: float source, 0: double
  long long bs;       // elements between matrices
  int rs, ks;         // element strides of a row and along K
  int R, K;           // valid rows / columns
  int Rp, Kp, KB;
  int s;
  int8_t *out;
  int *e;
  const int *active;  // optional: matrices with active[b] == 0 are skipped
};

template <int CHUNKS_MAX = 16>
__global__ void __launch_bounds__(256) k_oz_slice(const OzSlice p)
{
  __shared__ unsigned long long rmax[256];
  const long b = blockIdx.x;
  if (p.active && !p.active[b]) return;
  const int chunks = p.Kp / 16;
  const int rpb = blockDim.x / chunks;  // rows per block
  const int t = threadIdx.x;
  const int rl = t % rpb, c = t / rpb;
  const int r = blockIdx.y * rpb + rl;
  const bool live = c < chunks && r < p.Rp;
  double x[16];
#pragma unroll
  for (int u = 0; u < 16; u++) x[u] = 0.0;
  double m = 0.0;
  if (live && r < p.R) {
    const long long base = b * p.bs + (long long)r * p.rs;
#pragma unroll
    for (int u = 0; u < 16; u++) {
      const int k = c * 16 + u;
      if (k < p.K) {
        const long long o = base + (long long)k * p.ks;
        x[u] = p.src_f32 ? (double)static_cast<const float *>(p.src)[o] : static_cast<const double *>(p.src)[o];
        m = fmax(m, fabs(x[u]));
      }
    }
  }
  if (t < rpb) rmax[t] = 0ull;
  __syncthreads();
  // non-negative doubles order like their bit patterns (NaN above all)
  if (live) atomicMax(&rmax[rl], (unsigned long long)__double_as_longlong(m));
  __syncthreads();
  if (!live) return;
  const double mx = __longlong_as_double((long long)rmax[rl]);
  int e = 0;
  if (mx > 0.0 && mx <= 1.7976931348623157e308) frexp(mx, &e);  // mx < 2^e
  if (c == 0) p.e[b * p.Rp + r] = e;
  const double sc = scalbn(1.0, 6 - e);
  double tv[16];
#pragma unroll
  for (int u = 0; u < 16; u++) tv[u] = x[u] * sc;  // |t| < 64
  int8_t *o = p.out + (size_t)b * p.s * p.Rp * p.Kp + oz_offset(r, c * 16, p.Rp, p.KB);
  const size_t sstride = (size_t)p.Rp * p.Kp;
  for (int i = 0; i < p.s; i++) {
    uint32_t w4[4];
#pragma unroll
    for (int g = 0; g < 4; g++) {
      uint32_t wv = 0;
#pragma unroll
      for (int h = 0; h < 4; h++) {
        const int u = g * 4 + h;
        const double q = rint(tv[u]);
        tv[u] = (tv[u] - q) * 128.0;
        wv |= ((uint32_t)(uint8_t)(int8_t)(int)q) << (8 * h);
      }
      w4[g] = wv;
    }
    *reinterpret_cast<uint4 *>(o + i * sstride) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
  }
}

// ---------------------------------------------------------- tcgen05 pieces

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init()
{
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// bounded wait for the completion of the phase with the given parity
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
  const uint32_t a = smem_u32(bar);
  for (unsigned it = 0; it < OZ_WAIT_LIMIT; it++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// shared-memory matrix descriptor, no swizzle, K-major (tcgen05 format:
// start >> 4 in [0,14), LBO >> 4 in [16,30), SBO >> 4 in [32,46), version 1
// at bit 46, layout type 0)
__device__ __forceinline__ uint64_t oz_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor of kind::i8: D s32 (bits 4-5 = 2), A and B signed
// (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
__host__ __device__ constexpr uint32_t oz_idesc(int M, int N)
{
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void oz_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc)
{
#if EIGB_TCGEN05
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
#endif
}
__device__ __forceinline__ void oz_commit(uint64_t *bar)
{
#if EIGB_TCGEN05
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
#endif
}
// sixteen consecutive 32-bit columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t a, int32_t (&v)[16])
{
  uint32_t r[16] = {};
#if EIGB_TCGEN05
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(a));
#endif
#pragma unroll
  for (int u = 0; u < 16; u++) v[u] = (int32_t)r[u];
}

// thirty-two consecutive 32-bit columns of this thread's TMEM lane (the wait
// is in the same statement, so no register is read before it arrived)
__device__ __forceinline__ void tmem_ld32(uint32_t a, int32_t (&v)[32])
{
  uint32_t r[32] = {};
#if EIGB_TCGEN05
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(a));
#endif
#pragma unroll
  for (int u = 0; u < 32; u++) v[u] = (int32_t)r[u];
}

// ------------------------------------------------------------------ product
struct OzGemm {
  const int8_t *Ls, *Rs;  // slices of the left / right operand
  const int *eL, *eR;     // their row exponents
  int RpL, RpR;           // padded rows of each operand
  int Kp, KB;             // padded K and the K-block
  int sL, sR, dmax;       // slices and the last diagonal kept (d = i + j, 1-based)
  int n;                  // valid output rows and columns
  int mtiles, ntiles;     // tiles per matrix
  double *out;            // out[b*ob + c*ldo + m]
  long long ob;
  int ldo;
  const void *add;        // optional addend, same indexing (ab, lda)
  int add_f32;
  long long ab;
  int lda;
  const int *active;      // optional: matrices with active[b] == 0 are skipped
  int *err;               // set to 1 when a wait gave up
};

// Diagonal groups.  An MMA with N = 256 costs about as long to issue as one
// with N = 64 (measured on B200: ~125 cycles each), so the right operand
// of each MMA is a window of four consecutive R slices (4 x 64 rows), and
// the four 64-column blocks of its 256-column accumulator each collect one
// diagonal.  In shared memory the R slices sit in descending order, R_j in
// slot jtop - j, with zero slots where a window reaches past R_sR or below
// R_1.  Group g (base D = 2 + 4g) accumulates diagonals D+3, D+2, D+1, D in
// its blocks 0..3; for L slice i its window starts at the slot of
// j = D + 3 - i.  (1-based slice indices, d = i + j.)
struct OzGeom {
  int groups;  // diagonal groups (256 TMEM columns each)
  int jtop;    // largest j any window reaches (>= sR: slots above R_sR are zero)
  int jbot;    // smallest j any window reaches (<= 1: slots below R_1 are zero)
  __host__ __device__ int slots() const { return jtop - jbot + 1; }
  __host__ __device__ int slot(int j) const { return jtop - j; }
};

__host__ __device__ inline bool oz_pair_used(int D, int i, int sR) { return D + 3 - i >= 1 && D - i <= sR; }

__host__ __device__ inline OzGeom oz_geom(int sL, int sR, int dmax)
{
  OzGeom g{};
  g.groups = (dmax - 2) / 4 + 1;
  g.jtop = sR;
  g.jbot = 1;
  for (int gi = 0; gi < g.groups; gi++) {
    const int D = 2 + 4 * gi;
    for (int i = 1; i <= sL; i++) {
      if (!oz_pair_used(D, i, sR)) continue;
      g.jtop = max(g.jtop, D + 3 - i);
      g.jbot = min(g.jbot, D - i);
    }
  }
  return g;
}

// TMEM columns of a CTA: 256 per diagonal group (a power of two)
__host__ __device__ inline int oz_tmem_cols(int groups) { return groups <= 1 ? 256 : 512; }

// dynamic shared memory a launch of k_oz_gemm requests: its operands, and
// enough of the SM's shared memory that the CTAs sharing an SM never ask
// for more than its 512 TMEM columns together (an allocation would wait)
__host__ inline size_t oz_launch_smem(size_t need, int groups, int smem_sm, int smem_rsv)
{
  const int per_sm = 512 / oz_tmem_cols(groups);  // CTAs whose columns fit together
  const size_t floor_bytes = (size_t)smem_sm / (size_t)(per_sm + 1) + 1024;
  (void)smem_rsv;
  return need > floor_bytes ? need : floor_bytes;
}

// dynamic shared memory of k_oz_gemm: L slices of one K-block, the R slots,
// 1 KB of barriers and column scales, 1 KB alignment slack
__host__ __device__ inline size_t oz_gemm_smem(int sL, int sR, int KB, int dmax = 0)
{
  if (dmax <= 0) dmax = sL + sR - 1;
  const OzGeom g = oz_geom(sL, sR, dmax);
  return (size_t)(sL * OZ_MT + g.slots() * OZ_NT) * KB + 2048;
}

constexpr int OZ_SMAX = 8;  // slices per operand at most

// 2^e as an exact double (normal range)
__device__ __forceinline__ double pow2(int e)
{
  e = max(-1022, min(1023, e));
  return __longlong_as_double((long long)(e + 1023) << 52);
}

__global__ void __launch_bounds__(OZ_THREADS, 1) k_oz_gemm(const OzGemm p)
{
  extern __shared__ __align__(16) unsigned char oz_smem[];  // 1 KB alignment is done by hand below
  const int tile = blockIdx.x;
  const long b = tile / (p.mtiles * p.ntiles);
  const int mt = (tile / p.ntiles) % p.mtiles;
  const int nt = tile % p.ntiles;
  if (p.active && !p.active[b]) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const OzGeom geo = oz_geom(p.sL, p.sR, p.dmax);
  const uint32_t lbytes = OZ_MT * p.KB, rbytes = OZ_NT * p.KB;
  // 1 KB-aligned operand area, then barriers and the column scales
  unsigned char *base = oz_smem + ((1024 - (smem_u32(oz_smem) & 1023)) & 1023);
  unsigned char *sLb = base;
  unsigned char *sRb = sLb + (size_t)p.sL * lbytes;  // geo.slots() slots of rbytes
  uint64_t *bars = reinterpret_cast<uint64_t *>(sRb + (size_t)geo.slots() * rbytes);
  // bars[0 .. OZ_SMAX): slices L_k, R_k of the K-block landed; bars[OZ_SMAX]:
  // the K-block's MMAs completed
  uint64_t *mdone = bars + OZ_SMAX;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + OZ_SMAX + 1);
  double *cscale = reinterpret_cast<double *>(bars + OZ_SMAX + 2);  // OZ_NT column scales
  __shared__ int failed;
  const int ns = max(p.sL, p.sR);
  if (threadIdx.x == 0) {
    failed = 0;
    for (int k = 0; k <= OZ_SMAX; k++) mbar_init(&bars[k], 1);
    mbar_fence_init();
  }
  // zero slots (never written by the copies)
  for (int j = geo.jbot; j <= geo.jtop; j++) {
    if (j >= 1 && j <= p.sR) continue;
    uint4 *z = reinterpret_cast<uint4 *>(sRb + (size_t)geo.slot(j) * rbytes);
    for (uint32_t u = threadIdx.x; u < rbytes / 16; u += OZ_THREADS) z[u] = make_uint4(0, 0, 0, 0);
  }
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  if (threadIdx.x < OZ_NT) {
    const int c = nt * OZ_NT + threadIdx.x;
    cscale[threadIdx.x] = c < p.n ? pow2(p.eR[b * p.RpR + c]) : 0.0;
  }
  const int tcols = oz_tmem_cols(geo.groups);
  if (warp == 0) tmem_alloc(tslot, tcols);
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  const uint32_t tmem = *tslot;
  const int nkb = p.Kp / p.KB;
  const size_t Lsz = (size_t)p.RpL * p.Kp, Rsz = (size_t)p.RpR * p.Kp;

  if (warp == 0 && lane == 0) {  // producer: slices L_k, R_k of each K-block, in order of k
    for (int kb = 0; kb < nkb; kb++) {
      if (kb > 0 && !mbar_wait(mdone, (kb - 1) & 1)) {
        atomicExch(&failed, 1);
        break;
      }
      const int8_t *gl = p.Ls + (size_t)b * p.sL * Lsz + (size_t)kb * p.RpL * p.KB + (size_t)mt * OZ_MT * p.KB;
      const int8_t *gr = p.Rs + (size_t)b * p.sR * Rsz + (size_t)kb * p.RpR * p.KB + (size_t)nt * OZ_NT * p.KB;
      for (int k = 0; k < ns; k++) {
        const uint32_t bytes = (k < p.sL ? lbytes : 0u) + (k < p.sR ? rbytes : 0u);
        mbar_expect_tx(&bars[k], bytes);
        if (k < p.sL) bulk_g2s(sLb + (size_t)k * lbytes, gl + (size_t)k * Lsz, lbytes, &bars[k]);
        if (k < p.sR) bulk_g2s(sRb + (size_t)geo.slot(k + 1) * rbytes, gr + (size_t)k * Rsz, rbytes, &bars[k]);
      }
    }
  } else if (warp == 1 && lane == 0) {  // MMA issuer
    const uint32_t idesc = oz_idesc(OZ_MT, 4 * OZ_NT);
    const uint32_t sbo = 8 * p.KB;
    uint32_t init = 0;
    for (int kb = 0; kb < nkb && !failed; kb++) {
      // (group, i) pairs issue once slices L_i and the window's real R_j have landed
      uint32_t done = 0;  // bit g * 8 + (i - 1)
      for (int k = 0; k < ns; k++) {
        if (!mbar_wait(&bars[k], kb & 1)) {
          atomicExch(&failed, 1);
          break;
        }
        tmem_fence_after();
        for (int gi = 0; gi < geo.groups; gi++) {
          const int D = 2 + 4 * gi;
          for (int i = 1; i <= p.sL; i++) {
            const uint32_t bit = 1u << (gi * 8 + i - 1);
            if ((done & bit) || !oz_pair_used(D, i, p.sR)) continue;
            const int jneed = min(p.sR, D + 3 - i);  // largest real slice of the window
            if (i > k + 1 || jneed > k + 1) continue;
            done |= bit;
            const uint32_t sa = smem_u32(sLb + (size_t)(i - 1) * lbytes);
            const uint32_t sb = smem_u32(sRb + (size_t)geo.slot(D + 3 - i) * rbytes);
            for (int t = 0; t < p.KB / 32; t++) {
              oz_mma(tmem + (uint32_t)(gi * 4 * OZ_NT), oz_desc(sa + t * 256, 128, sbo),
                     oz_desc(sb + t * 256, 128, sbo), idesc, (init >> gi) & 1u);
              init |= 1u << gi;
            }
          }
        }
      }
      oz_commit(mdone);
    }
    // the last K-block's MMAs: one thread waits, the barrier below releases the rest
    if (!failed && !mbar_wait(mdone, (nkb - 1) & 1)) atomicExch(&failed, 1);
  }
  __syncwarp();
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  if (failed) {
    if (threadIdx.x == 0 && p.err) atomicExch(p.err, 1);
  } else {
    const int m = mt * OZ_MT + warp * 32 + lane;  // this thread's output row
    const bool mrow = m < p.n;
    const double rsc = pow2(p.eL[b * p.RpL + m] - 12);
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    // every diagonal the groups hold, from the least significant (Horner),
    // 32 columns at a time
    const int dtop = 4 * geo.groups + 1;
    for (int h = 0; h < OZ_NT; h += 32) {
      double acc[32];
#pragma unroll
      for (int u = 0; u < 32; u++) acc[u] = 0.0;
      for (int d = dtop; d >= 2; d--) {
        const int gi = (d - 2) / 4, blk = 3 - (d - 2) % 4;
        int32_t v[32];
        tmem_ld32(lane_addr + (uint32_t)(gi * 4 * OZ_NT + blk * OZ_NT + h), v);
#pragma unroll
        for (int u = 0; u < 32; u++) acc[u] = fma(acc[u], 0.0078125, (double)v[u]);
      }
      if (mrow) {
#pragma unroll
        for (int u = 0; u < 32; u++) {
          const int c = nt * OZ_NT + h + u;
          if (c < p.n) {
            double r = acc[u] * rsc * cscale[h + u];
            if (p.add) {
              const long long ai = b * p.ab + (long long)c * p.lda + m;
              r += p.add_f32 ? (double)static_cast<const float *>(p.add)[ai] : static_cast<const double *>(p.add)[ai];
            }
            p.out[b * p.ob + (long long)c * p.ldo + m] = r;
          }
        }
      }
    }
  }
  tmem_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, tcols);
}

}  // namespace eigb
