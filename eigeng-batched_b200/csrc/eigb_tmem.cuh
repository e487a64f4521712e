// Tensor memory (TMEM) as the store of Z in phase 3.
//
// TMEM is 128 lanes x 512 columns of 32 bits per SM; a warp reaches the 32
// lanes of its sub-partition, lanes 32*(warp % 4) .. +31, and with the
// 32x32b shape each thread of the warp moves data of its own lane.  That
// is the access of the rotation apply (one row of Z per thread, walked
// along its columns), so a CTA of up to four warps keeps up to 128 rows of
// Z in TMEM, row r in lane r, element c in the 32-bit columns
// [c*W, c*W + W), W = sizeof(T)/4.  The rows then never touch shared
// memory, whose bandwidth the records keep to themselves.
//
// Every tcgen05 instruction here is .sync.aligned: all 32 threads of a
// warp execute it together with the same address (the lane field is the
// warp's first lane).  Loads are followed by tcgen05.wait::ld inside the
// same asm statement, so no register is read before its data arrived;
// tcgen05.wait::st orders a thread's stores before its later loads of the
// same columns (the start of every segment, and the final read-out).  The
// loads and stores touch only tensor memory and registers: their asm
// statements are volatile (kept in program order among themselves) but do
// not clobber memory, so the compiler may schedule shared-memory loads
// (the rotation records) across them.
#pragma once
#include <stdint.h>

#include "eigb_apply.cuh"
#include "eigb_common.cuh"

namespace eigb {

// TMEM columns of a CTA that holds rows of n elements: a power of two, at
// least 32 (the allocation granule), or 0 if a row does not fit.
template <class T> __host__ __device__ inline int tmem_cols(int n)
{
  const int need = n * (int)(sizeof(T) / 4);
  if (need > 512) return 0;
  int c = 32;
  while (c < need) c <<= 1;
  return c;
}

// The tcgen05 instructions exist on sm_100a; other device compilations of
// this header (host-side unit tests) get empty bodies, never called.
#if defined(__CUDA_ARCH_FEAT_SM100_ALL)
#define EIGB_TCGEN05 1
#else
#define EIGB_TCGEN05 0
#endif

// Allocation by one full warp; the address goes to shared memory.
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, const int ncols)
{
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
#if EIGB_TCGEN05
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(d), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
#endif
}
__device__ __forceinline__ void tmem_dealloc(const uint32_t taddr, const int ncols)
{
#if EIGB_TCGEN05
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
#endif
}
__device__ __forceinline__ void tmem_fence_before()
{
#if EIGB_TCGEN05
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
#endif
}
__device__ __forceinline__ void tmem_fence_after()
{
#if EIGB_TCGEN05
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#endif
}
__device__ __forceinline__ void tmem_wait_st()
{
#if EIGB_TCGEN05
  asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
#endif
}

// one element
__device__ __forceinline__ double tmem_ld1(const double *, const uint32_t a)
{
  uint32_t lo = 0, hi = 0;
#if EIGB_TCGEN05
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(lo), "=r"(hi)
      : "r"(a));
#endif
  return __hiloint2double((int)hi, (int)lo);
}
__device__ __forceinline__ float tmem_ld1(const float *, const uint32_t a)
{
  uint32_t v = 0;
#if EIGB_TCGEN05
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(v)
      : "r"(a));
#endif
  return __uint_as_float(v);
}
__device__ __forceinline__ void tmem_st1(const uint32_t a, const double v)
{
  const uint32_t lo = (uint32_t)__double2loint(v), hi = (uint32_t)__double2hiint(v);
#if EIGB_TCGEN05
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};\n" ::"r"(a), "r"(lo), "r"(hi));
#endif
}
__device__ __forceinline__ void tmem_st1(const uint32_t a, const float v)
{
#if EIGB_TCGEN05
  asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};\n" ::"r"(a), "r"(__float_as_uint(v)));
#endif
}

// eight elements, v[u] = column c - u, from the address a of column c;
// one wait for all
__device__ __forceinline__ void tmem_ld8(const uint32_t a, double (&v)[8])
{
  constexpr uint32_t s = 2;
  uint32_t r[16] = {};
#if EIGB_TCGEN05
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%16];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%2, %3}, [%17];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%4, %5}, [%18];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%6, %7}, [%19];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%8, %9}, [%20];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%10, %11}, [%21];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%12, %13}, [%22];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%14, %15}, [%23];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(a), "r"(a - s), "r"(a - 2 * s), "r"(a - 3 * s), "r"(a - 4 * s), "r"(a - 5 * s), "r"(a - 6 * s),
        "r"(a - 7 * s));
#endif
#pragma unroll
  for (int u = 0; u < 8; u++) v[u] = __hiloint2double((int)r[2 * u + 1], (int)r[2 * u]);
}
__device__ __forceinline__ void tmem_ld8(const uint32_t a, float (&v)[8])
{
  constexpr uint32_t s = 1;
  uint32_t r[8] = {};
#if EIGB_TCGEN05
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%8];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%1}, [%9];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%2}, [%10];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%3}, [%11];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%4}, [%12];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%5}, [%13];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%6}, [%14];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%7}, [%15];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(a), "r"(a - s), "r"(a - 2 * s), "r"(a - 3 * s), "r"(a - 4 * s), "r"(a - 5 * s), "r"(a - 6 * s),
        "r"(a - 7 * s));
#endif
#pragma unroll
  for (int u = 0; u < 8; u++) v[u] = __uint_as_float(r[u]);
}

// Named barrier of the nthr threads (a multiple of 32) of one part of a
// CTA; id 1..15 (0 is __syncthreads).  The aligned form: every warp
// reaches it as a whole.
__device__ __forceinline__ void part_sync(const int id, const int nthr)
{
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(nthr) : "memory");
}
// the same barrier, returning whether x held in any of the threads
__device__ __forceinline__ bool part_sync_or(const int id, const int nthr, const bool x)
{
  int r;
  asm volatile(
      "{\n\t.reg .pred px, pr;\n\t"
      "setp.ne.s32 px, %1, 0;\n\t"
      "bar.red.or.pred pr, %2, %3, px;\n\t"
      "selp.s32 %0, 1, 0, pr;\n\t}\n"
      : "=r"(r)
      : "r"((int)x), "r"(id), "r"(nthr)
      : "memory");
  return r != 0;
}

// Address of element c of this thread's row (z0: address of element 0)
template <class T> __device__ __forceinline__ uint32_t tmem_at(const uint32_t z0, const int c)
{
  return z0 + (uint32_t)(c * (int)(sizeof(T) / 4));
}

// seg_apply on a row in TMEM: the same operations in the same order, so
// the results are bit-identical to the shared-memory form.
// (seg_apply_tm_h takes z_{i0+1} as the carried value h: a sweep that
// continues another one's pass, whose stores are this thread's own)
template <class T>
__device__ __forceinline__ void seg_apply_tm_h(const uint32_t z0, const Rec<T> *__restrict__ rp, const int i0,
                                               const int len, T h)
{
  int c = i0;  // column of the next rotation's z_i
  int j = 0;
  for (; j + 8 <= len; j += 8, c -= 8) {
    T z[8];
    tmem_ld8(tmem_at<T>(z0, c), z);
    T cz[8], sz[8];
    Rec<T> r[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      r[u] = rp[j + u];
      cz[u] = r[u].c * z[u];
      sz[u] = r[u].s * z[u];
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const T y = fma(r[u].c, h, sz[u]);
      h = fma(-r[u].s, h, cz[u]);
      tmem_st1(tmem_at<T>(z0, c + 1 - u), y);
    }
  }
  for (; j < len; j++, c--) {
    const T z = tmem_ld1((const T *)nullptr, tmem_at<T>(z0, c));
    const Rec<T> r = rp[j];
    const T y = fma(r.c, h, r.s * z);
    h = fma(-r.s, h, r.c * z);
    tmem_st1(tmem_at<T>(z0, c + 1), y);
  }
  tmem_st1(tmem_at<T>(z0, c + 1), h);
}
template <class T>
__device__ __forceinline__ void seg_apply_tm(const uint32_t z0, const Rec<T> *__restrict__ rp, const int i0,
                                             const int len)
{
  tmem_wait_st();  // the previous segment's stores land before these loads
  seg_apply_tm_h<T>(z0, rp, i0, len, tmem_ld1((const T *)nullptr, tmem_at<T>(z0, i0 + 1)));
}

// Row accessor for seg_apply_group: this thread's row in TMEM
template <class T> struct RowTM {
  uint32_t z0;
  __device__ __forceinline__ T ld(const int c) const { return tmem_ld1((const T *)nullptr, tmem_at<T>(z0, c)); }
  __device__ __forceinline__ void st(const int c, const T v) const { tmem_st1(tmem_at<T>(z0, c), v); }
  __device__ __forceinline__ void ld8(const int c, T (&v)[8]) const { tmem_ld8(tmem_at<T>(z0, c), v); }
  __device__ __forceinline__ void begin() const { tmem_wait_st(); }  // earlier stores land before these loads
};

// seg_apply_pair on a row in TMEM (bit-identical to the shared-memory form)
template <class T>
__device__ __forceinline__ void seg_apply_pair_tm(const uint32_t z0, const Rec<T> *__restrict__ ra, const int la,
                                                  const Rec<T> *__restrict__ rb, const int i0, const int len)
{
  tmem_wait_st();
  int c = i0;
  T ha = tmem_ld1((const T *)nullptr, tmem_at<T>(z0, c + 1));
  T hb;
  {
    const T x = tmem_ld1((const T *)nullptr, tmem_at<T>(z0, c));
    const Rec<T> r = ra[0];
    hb = fma(r.c, ha, r.s * x);
    ha = fma(-r.s, ha, r.c * x);
  }
  c -= 1;  // column i0 - j at step j: first sweep rotation i0-j, second i0-j+1
  int j = 1;
  for (; j + 8 <= len; j += 8, c -= 8) {
    T x[8];
    tmem_ld8(tmem_at<T>(z0, c), x);
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const Rec<T> a = ra[j + u], b = rb[j - 1 + u];
      const T ya = fma(a.c, ha, a.s * x[u]);
      ha = fma(-a.s, ha, a.c * x[u]);
      const T yb = fma(b.c, hb, b.s * ya);
      hb = fma(-b.s, hb, b.c * ya);
      tmem_st1(tmem_at<T>(z0, c + 2 - u), yb);
    }
  }
  for (; j < len; j++, c--) {
    const T x = tmem_ld1((const T *)nullptr, tmem_at<T>(z0, c));
    const Rec<T> a = ra[j], b = rb[j - 1];
    const T ya = fma(a.c, ha, a.s * x);
    ha = fma(-a.s, ha, a.c * x);
    const T yb = fma(b.c, hb, b.s * ya);
    hb = fma(-b.s, hb, b.c * ya);
    tmem_st1(tmem_at<T>(z0, c + 2), yb);
  }
  if (la == len) {  // second sweep, last rotation, on the first's last value
    const Rec<T> r = rb[len - 1];
    tmem_st1(tmem_at<T>(z0, c + 2), fma(r.c, hb, r.s * ha));
    tmem_st1(tmem_at<T>(z0, c + 1), fma(-r.s, hb, r.c * ha));
  } else {  // the first sweep's rotation c, the second's last, then the first alone
    const T x = tmem_ld1((const T *)nullptr, tmem_at<T>(z0, c));
    const Rec<T> a = ra[len], b = rb[len - 1];
    const T ya = fma(a.c, ha, a.s * x);
    ha = fma(-a.s, ha, a.c * x);
    tmem_st1(tmem_at<T>(z0, c + 2), fma(b.c, hb, b.s * ya));
    tmem_st1(tmem_at<T>(z0, c + 1), fma(-b.s, hb, b.c * ya));
    seg_apply_tm_h<T>(z0, ra + len + 1, c - 1, la - len - 1, ha);
  }
}

// A single sweep on a row in TMEM (functor for apply_grouped)
template <class T> struct SingleTM {
  uint32_t z0;
  __device__ __forceinline__ void operator()(const Rec<T> *rp, const int i0, const int len) const
  {
    seg_apply_tm<T>(z0, rp, i0, len);
  }
};

// apply_segments for a row in TMEM (bit-identical to the shared-memory
// form).  KG > 1: groups of up to KG consecutive sweeps go through
// seg_apply_group; KG = 1: two consecutive sweeps from the same top, the
// second no longer than the first, go through seg_apply_pair_tm (measured on B200: groups pay off for rows
// of 128 or more, the pairs below that).
template <class T, int KG>
__device__ __forceinline__ void apply_segments_tm(const Rec<T> *rbuf, const int used, const uint32_t z0)
{
  if (KG > 1) {
    apply_grouped<T, KG>(rbuf, used, RowTM<T>{z0}, SingleTM<T>{z0});
    return;
  }
  int q = 0;
  while (q < used) {
    const Rec<T> hd = rbuf[q];
    const int L = hdr_cnt(hd), i0 = hdr_i0(hd);
    const int q2 = q + 1 + L;
    if (L >= 1 && q2 < used) {
      const Rec<T> h2 = rbuf[q2];
      const int L2 = hdr_cnt(h2);
      if (hdr_i0(h2) == i0 && L2 >= 1 && L2 <= L) {
        seg_apply_pair_tm<T>(z0, rbuf + q + 1, L, rbuf + q2 + 1, i0, L2);
        q = q2 + 1 + L2;
        continue;
      }
    }
    seg_apply_tm<T>(z0, rbuf + q + 1, i0, L);
    q = q2;
  }
}

}  // namespace eigb
