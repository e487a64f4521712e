// The learned warm start's network: a small MLP trained and run by this
// library's own kernels.
//
//   k_mm_bf16      C = alpha A B^T (+ bias) (tanh) on the tensor cores
//                  (tcgen05.mma kind::f16, BF16 operands, FP32 accumulation
//                  in TMEM); A (M x K) and B (N x K) row-major BF16,
//                  K a multiple of 8.  One CTA of four warps per 128 x 128
//                  output tile; K-blocks of 64 staged in three shared-memory
//                  buffers by cp.async (16 bytes per thread and copy) in the
//                  no-swizzle K-major canonical layout (core matrices of
//                  8 rows x 16 bytes, LBO 128 bytes, SBO 1024 bytes); thread
//                  0 issues the MMAs, each buffer is refilled after the
//                  tcgen05.commit of the MMAs that read it.  The epilogue
//                  reads one TMEM lane (output row) per thread and writes
//                  FP32 and/or BF16.
//   k_t_bf16       BF16 transpose (32 x 32 tiles)
//   k_tanh_bwd     dZ = dH (1 - H^2) (BF16 out)
//   k_colsum       bias gradients: column sums of a BF16 matrix
//   k_mse_grad     dY = 2 (Y - T) / (rows * cols) (BF16) and the squared error
//   k_adam         Adam on the FP32 master weights; writes their BF16 copy
//                  and its transpose
//
// Parameter buffer (one allocation by the caller, eigen_GPU_mlp_size): for
// each of the three layers l (widths d0 -> d1 -> d2 -> d3), FP32 W_l (d_l+1
// x d_l, row-major), b_l, their Adam moments m and v, and the BF16 copies of
// W_l and W_l^T.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "eigb_oz.cuh"

namespace eigb {

typedef __nv_bfloat16 bf16;

constexpr int MM_T = 128;       // output tile (rows and columns)
constexpr int MM_KB = 64;       // K elements per stage (128 bytes)
constexpr int MM_STAGES = 3;
constexpr int MM_THREADS = 128;
constexpr int MM_TMEM_COLS = 128;

__host__ __device__ inline size_t mm_smem() { return (size_t)MM_STAGES * 2 * MM_T * MM_KB * 2 + 1024 + 256; }

struct MmP {
  const bf16 *A;
  long long sa;
  int lda;          // A[z][m][k] at A + z*sa + m*lda + k
  const bf16 *B;
  long long sb;
  int ldb;          // B[z][n][k]
  int M, N, K;
  float *C;
  long long sc;
  int ldc;          // optional FP32 output C[z][m][n]
  bf16 *Cb;
  long long scb;
  int ldcb;         // optional BF16 output
  const float *bias;  // optional, per column n
  float alpha;
  int act;          // 0: none, 1: tanh
  int *err;         // set when a bounded wait gave up
};

// instruction descriptor of kind::f16: D f32 (bits 4-5 = 1), A and B bf16
// (bits 7-9, 10-12 = 1), K-major, N >> 3 at bit 17, M >> 4 at bit 24
__host__ __device__ constexpr uint32_t mm_idesc(int M, int N)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mm_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc)
{
#if EIGB_TCGEN05
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
#endif
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t src_bytes)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// stage the K-block kb of the A and B tiles (rows m0.., n0..) into buffer s
__device__ __forceinline__ void mm_load(const MmP &p, const bf16 *A, const bf16 *B, int m0, int n0, int kb,
                                        unsigned char *sA, unsigned char *sB)
{
  const int k0 = kb * MM_KB;
  for (int i = threadIdx.x; i < 2 * MM_T * 8; i += MM_THREADS) {
    const int side = i >= MM_T * 8;
    const int j = side ? i - MM_T * 8 : i;
    const int row = j >> 3, c = j & 7;
    const int k = k0 + c * 8;
    const uint32_t off = (uint32_t)((row >> 3) * 1024 + c * 128 + (row & 7) * 16);
    if (!side) {
      const bool ok = (m0 + row) < p.M && k < p.K;
      const bf16 *src = ok ? A + (size_t)(m0 + row) * p.lda + k : A;
      cp_async16(smem_u32(sA) + off, src, ok ? 16u : 0u);
    } else {
      const bool ok = (n0 + row) < p.N && k < p.K;
      const bf16 *src = ok ? B + (size_t)(n0 + row) * p.ldb + k : B;
      cp_async16(smem_u32(sB) + off, src, ok ? 16u : 0u);
    }
  }
}

__global__ void __launch_bounds__(MM_THREADS) k_mm_bf16(const MmP p)
{
  extern __shared__ __align__(16) unsigned char mm_smem_raw[];  // 1 KB alignment is done by hand below
  unsigned char *base = mm_smem_raw + ((1024 - (smem_u32(mm_smem_raw) & 1023)) & 1023);
  unsigned char *sbuf = base;  // MM_STAGES x (A tile, B tile), 16 KB each
  uint64_t *bars = reinterpret_cast<uint64_t *>(base + (size_t)MM_STAGES * 2 * MM_T * MM_KB * 2);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + MM_STAGES);
  const int z = blockIdx.z;
  const int m0 = blockIdx.y * MM_T, n0 = blockIdx.x * MM_T;
  const bf16 *A = p.A + (size_t)z * p.sa;
  const bf16 *B = p.B + (size_t)z * p.sb;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < MM_STAGES; s++) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  if (warp == 0) tmem_alloc(tslot, MM_TMEM_COLS);
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  const uint32_t tmem = *tslot;
  const int nkb = (p.K + MM_KB - 1) / MM_KB;
  const uint32_t tile_bytes = MM_T * MM_KB * 2;
  auto bufA = [&](int s) { return sbuf + (size_t)s * 2 * tile_bytes; };
  auto bufB = [&](int s) { return sbuf + (size_t)s * 2 * tile_bytes + tile_bytes; };
  for (int s = 0; s < MM_STAGES - 1; s++) {
    if (s < nkb) mm_load(p, A, B, m0, n0, s, bufA(s), bufB(s));
    cp_async_commit();
  }
  const uint32_t idesc = mm_idesc(MM_T, MM_T);
  __shared__ int failed;
  if (threadIdx.x == 0) failed = 0;
  __syncthreads();
  bool ok = true;
  for (int kb = 0; kb < nkb; kb++) {
    const int s = kb % MM_STAGES;
    cp_async_wait<MM_STAGES - 2>();
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      tmem_fence_after();
      for (int t = 0; t < MM_KB / 16; t++) {
        const uint64_t da = oz_desc(smem_u32(bufA(s)) + t * 256, 128, 1024);
        const uint64_t db = oz_desc(smem_u32(bufB(s)) + t * 256, 128, 1024);
        mm_mma(tmem, da, db, idesc, (kb > 0 || t > 0) ? 1u : 0u);
      }
      oz_commit(&bars[s]);
    }
    // refill the buffer of K-block kb-1 (its MMAs must have finished)
    const int nk = kb + MM_STAGES - 1;
    if (nk < nkb) {
      const int ps = nk % MM_STAGES;
      if (kb >= 1 && !mbar_wait(&bars[ps], (uint32_t)(((kb - 1) / MM_STAGES) & 1))) ok = false;
      if (ok) mm_load(p, A, B, m0, n0, nk, bufA(ps), bufB(ps));
    }
    cp_async_commit();
  }
  cp_async_wait<0>();
  if (!mbar_wait(&bars[(nkb - 1) % MM_STAGES], (uint32_t)(((nkb - 1) / MM_STAGES) & 1))) ok = false;
  if (!ok) atomicExch(&failed, 1);
  tmem_fence_after();
  __syncthreads();
  if (failed) {  // uniform over the CTA: the read-back below is .sync.aligned
    if (p.err) atomicExch(p.err, 1);
  } else {
    const int m = m0 + warp * 32 + lane;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < MM_T; c0 += 16) {
      int32_t v[16];
      tmem_ld16(lane_addr + (uint32_t)c0, v);
      if (m < p.M) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
          const int nn = n0 + c0 + u;
          if (nn < p.N) {
            float r = p.alpha * __int_as_float(v[u]);
            if (p.bias) r += p.bias[nn];
            if (p.act == 1) r = tanhf(r);
            if (p.C) p.C[(size_t)z * p.sc + (size_t)m * p.ldc + nn] = r;
            if (p.Cb) p.Cb[(size_t)z * p.scb + (size_t)m * p.ldcb + nn] = __float2bfloat16_rn(r);
          }
        }
      }
    }
  }
  tmem_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, MM_TMEM_COLS);
}

// out[c][r] = in[r][c] (rows x cols BF16, both row-major with their widths)
__global__ void __launch_bounds__(256) k_t_bf16(const int rows, const int cols, const bf16 *__restrict__ in,
                                                 const int ldi, bf16 *__restrict__ out, const int ldo)
{
  __shared__ bf16 t[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int i = ty; i < 32; i += 8)
    if (r0 + i < rows && c0 + tx < cols) t[i][tx] = in[(size_t)(r0 + i) * ldi + c0 + tx];
  __syncthreads();
  for (int i = ty; i < 32; i += 8)
    if (c0 + i < cols && r0 + tx < rows) out[(size_t)(c0 + i) * ldo + r0 + tx] = t[tx][i];
}

// dZ = dH (1 - H^2), H = tanh(Z) (FP32), dH FP32; dZ BF16
__global__ void k_tanh_bwd(const long count, const float *__restrict__ dh, const float *__restrict__ h,
                           bf16 *__restrict__ dz, float *__restrict__ dz32)
{
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
    const float v = dh[i] * (1.0f - h[i] * h[i]);
    dz[i] = __float2bfloat16_rn(v);
    if (dz32) dz32[i] = v;
  }
}

// sums[c] = sum_r x[r][c] (FP32 rows x cols); one thread per column
__global__ void k_colsum(const int rows, const int cols, const float *__restrict__ x, float *__restrict__ sums)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.0f;
  for (int r = 0; r < rows; r++) s += x[(size_t)r * cols + c];
  sums[c] = s;
}

// dY = 2 (Y - T) / count (BF16 and FP32), sse += sum (Y - T)^2
__global__ void k_mse_grad(const long count, const float *__restrict__ y, const float *__restrict__ t,
                           bf16 *__restrict__ dy, float *__restrict__ dy32, double *__restrict__ sse)
{
  __shared__ double red[8];
  double acc = 0.0;
  const float sc = 2.0f / (float)count;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
    const float d = y[i] - t[i];
    acc += (double)d * d;
    dy[i] = __float2bfloat16_rn(sc * d);
    if (dy32) dy32[i] = sc * d;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += red[i];
    atomicAdd(sse, s);
  }
}

// Adam step on FP32 weights w (rows x cols, row-major) and bias b (rows):
// g gradient, m and v moments; writes the BF16 copy wb and its transpose
// wt (cols x rows).  lr already holds the bias-correction factors.
__global__ void k_adam(const int rows, const int cols, float *__restrict__ w, const float *__restrict__ g,
                       float *__restrict__ m, float *__restrict__ v, bf16 *__restrict__ wb, bf16 *__restrict__ wt,
                       const float lr, const float b1, const float b2, const float eps, const float c1,
                       const float c2)
{
  const long count = (long)rows * cols;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    w[i] = wi;
    if (wb) {
      const int r = (int)(i / cols), c = (int)(i % cols);
      const bf16 x = __float2bfloat16_rn(wi);
      wb[i] = x;
      if (wt) wt[(size_t)c * rows + r] = x;
    }
  }
}

// FP32 -> BF16 with a row stride change (row-major rows x cols)
__global__ void k_to_bf16(const int rows, const int cols, const float *__restrict__ x, const int ldx,
                          bf16 *__restrict__ y, const int ldy)
{
  const long count = (long)rows * ldy;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
    const int r = (int)(i / ldy), c = (int)(i % ldy);
    y[i] = __float2bfloat16_rn(c < cols ? x[(size_t)r * ldx + c] : 0.0f);
  }
}

// deterministic uniform init in [-s, s] (splitmix64 of the index and seed)
__global__ void k_init_uniform(const long count, float *__restrict__ w, const float s, const unsigned long long seed)
{
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
    unsigned long long x = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1);
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x ^= x >> 31;
    const float u = (float)((double)(x >> 11) * (1.0 / 9007199254740992.0));  // [0, 1)
    w[i] = (2.0f * u - 1.0f) * s;
  }
}

}  // namespace eigb
