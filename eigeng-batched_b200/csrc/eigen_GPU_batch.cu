// Host launcher and C ABI of the B200 batched symmetric eigensolver.
//
// Drop-in for the reference's eigen_GPU_batch_DP / eigen_GPU_batch_FP
// (eigen_GPU_batch.h:26-30, eigen_GPU_batch.cu:327-367) with the same
// workspace-query convention, plus an extended entry point with options and
// per-matrix status, and the accuracy gate eigen_GPU_check_{DP,FP}.
//
// Per call, for each chunk of matrices (all on the caller's stream, no host
// synchronisation, no allocation):
//   phase 1  tridiagonalize, form Q^T in place of A, write d/e to workspace
//   phase 2  QL on (d, e), one matrix per thread, rotation records out
//   phase 3  apply the records to Q, sort, write eigenvectors and values
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <functional>
#include <map>
#include <mutex>
#include <vector>

#include "eigb_kernels.cuh"
#include "eigb_symfunc.cuh"
#include "eigb_refine.cuh"
#include "eigb_learned.cuh"
#include "eigb_queue.cuh"
#include "../../include/eigen_GPU_learned.h"
#include "../../include/eigen_GPU_batch.h"

namespace eigb {
namespace {

constexpr int kMaxDev = 64;
constexpr size_t kWsBudget = (size_t)8 << 30;  // workspace target per call
// the refined solve's target: its workspace holds six FP64 n x n matrices
// and the slices per matrix (about 5.5 MB at n = 256), and each chunk pays
// its FP32 solve's QL latency again (C4, 2048 matrices of n = 256: 119 ms
// in two chunks of 8 GB, 106 ms in one)
constexpr size_t kRefBudget = (size_t)16 << 30;
constexpr long kMinChunk = 512;

struct DevProps {
  int sms = 0;
  int smem_optin = 0;
  int smem_sm = 0;   // shared memory per SM
  int smem_rsv = 0;  // shared memory the system reserves per block
  int l2 = 0;
  bool ok = false;
};
DevProps g_props[kMaxDev];
std::mutex g_mu;

// Device properties, read once per device (the reference queries
// cudaGetDeviceProperties on every call, eigen_GPU_batch.hpp:33-43).
cudaError_t dev_props(DevProps &out)
{
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_mu);
  DevProps &p = g_props[dev];
  if (!p.ok) {
    if ((err = cudaDeviceGetAttribute(&p.sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return err;
    if ((err = cudaDeviceGetAttribute(&p.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess)
      return err;
    if ((err = cudaDeviceGetAttribute(&p.smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess)
      return err;
    if ((err = cudaDeviceGetAttribute(&p.smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev)) != cudaSuccess)
      return err;
    if ((err = cudaDeviceGetAttribute(&p.l2, cudaDevAttrL2CacheSize, dev)) != cudaSuccess) return err;
    p.ok = true;
  }
  out = p;
  return cudaSuccess;
}

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Tuned options (eigen_GPU_batch_tune_set): per device, per (element size,
// n), the options a solve uses where the caller leaves them automatic.
struct TuneKey {
  int dev, esize, n;
  bool operator<(const TuneKey &o) const
  {
    return dev != o.dev ? dev < o.dev : (esize != o.esize ? esize < o.esize : n < o.n);
  }
};
std::map<TuneKey, eigen_GPU_tune_entry> g_tune;

// the caller's options with the tuned values filled in where they are
// automatic (split <= 0, zmem == AUTO, ql_mpw <= 0); `out` receives them
inline const eigen_GPU_batch_opts *tuned(const eigen_GPU_batch_opts *opts, int esize, int n,
                                         eigen_GPU_batch_opts &out)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return opts;
  eigen_GPU_tune_entry e;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_tune.empty()) return opts;
    auto it = g_tune.find(TuneKey{dev, esize, n});
    if (it == g_tune.end()) return opts;
    e = it->second;
  }
  if (opts) {
    out = *opts;
  } else {  // the reference defaults
    out = eigen_GPU_batch_opts{};
    out.method = EIGEN_GPU_BATCH_TQL2;
    out.sort = 1;
    out.max_sweep = 100;
  }
  if (out.split <= 0 && e.split > 0) out.split = e.split;
  if (out.zmem == EIGEN_GPU_ZMEM_AUTO && e.zmem == EIGEN_GPU_ZMEM_SHARED) out.zmem = EIGEN_GPU_ZMEM_SHARED;
  if (out.ql_mpw <= 0 && e.ql_mpw > 0) out.ql_mpw = e.ql_mpw;
  return &out;
}

// the phase-1 kernel the table asks for (EIGEN_GPU_REDUCE_*)
inline int tuned_reduce(int esize, int n)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return EIGEN_GPU_REDUCE_AUTO;
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_tune.find(TuneKey{dev, esize, n});
  return it == g_tune.end() ? EIGEN_GPU_REDUCE_AUTO : it->second.reduce;
}

// phase timing events set by eigen_GPU_batch_trace
cudaEvent_t *g_trace = nullptr;
int g_ntrace = 0;

inline void trace(long chunk, int slot, cudaStream_t stream)
{
  cudaEvent_t *ev;
  int nev;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    ev = g_trace;
    nev = g_ntrace;
  }
  const long i = 4 * chunk + slot;
  if (ev && 4 * chunk + 3 < nev) cudaEventRecord(ev[i], stream);
}

template <class T> int k1c_threads(int n) { return std::min(1024, ((n + 31) / 32) * 32 * k1_split<T>(n)); }
// leading block of phase 1 (CTA form) held in shared memory: the whole
// matrix when it fits; otherwise the largest that fits next to the scratch
// arrays, for FP64 at most 128 x 128, which leaves L1 room for the outer
// band (measured on B200 at n = 200 and 256: 15-20 % faster than the
// largest block).  FP64 128 < n <= 240 keeps a 64 x 64 (n <= 176) or
// 96 x 96 block, FP32 128 < n <= 512 a 64 x 64 (n <= 224) or 128 x 128
// one: more CTAs per SM pay more than a larger block (see k1_split)
template <class T> int k1c_block(int n, size_t optin)
{
  const size_t base = sizeof(T) * k1c_smem_elems(n, k1c_threads<T>(n), 0);
  if (base >= optin) return 0;
  int B = n;
  if (sizeof(T) == 8 && base + sizeof(T) * (size_t)n * (size_t)(n | 1) > optin) B = std::min(n, 128);
  if (sizeof(T) == 8 && n > 128 && n <= 240) B = n <= 176 ? 64 : 96;
  if (sizeof(T) == 4 && n > 128 && n <= 512) B = std::min(B, n <= 224 ? 64 : 128);
  while (B > 0 && base + sizeof(T) * (size_t)B * (size_t)(B | 1) > optin) B--;
  return B;
}
template <class T> size_t k2_smem_per_thread(int n) { return sizeof(T) * 2 * (size_t)n; }

// Phase 2 matrices per warp: the largest power of two that still gives
// each SM about three warps; two for batches of 1025 .. 2048 (measured on
// B200: 8 per warp for 4096 matrices, 32 for 16384, 2 for 2048 at n = 32 ..
// 256).  Smaller batches, such as the chunks of solve_host that run beside
// another chunk's solve, keep the rule: one per warp would be faster alone
// but crowds out the concurrent solve.
inline int k2_mpw(long L, int sms)
{
  const long target = (L > 1024 && L <= 2048) ? L / 2 : 3L * sms;
  int m = 32;
  while (m > 1 && (L + m - 1) / m < target) m >>= 1;
  return m;
}

// Layout of the workspace for one chunk of Lc matrices.
template <class T> struct Plan {
  int n = 0, nm = 0;
  long L = 0, Lc = 0;
  int rcap = 0;
  int k1b = 0;        // phase 1 (CTA form): leading block held in shared memory
  int zrows = 0;      // phase 3: rows of Z per CTA in shared memory (0: Z in the workspace)
  int zsplit = 1;     // phase 3: CTAs per matrix
  int ztm = 0;        // phase 3: rows of Z in tensor memory instead of shared memory
  size_t off_d = 0, off_e = 0, off_meta = 0, off_rec = 0, off_z = 0, bytes = 0;
};

template <class T> int rec_capacity(int n)
{
  // tql2 / imtql2 take ~1.1 n^2 rotations plus one header per sweep on
  // random matrices; twice that leaves ample margin, and a matrix that still
  // overflows is finished by phase 3 itself.
  return 2 * n * n + 4 * n + 32;
}

template <class T>
cudaError_t make_plan(long L, int nm, int n, const DevProps &dp, Plan<T> &pl, const eigen_GPU_batch_opts *opts)
{
  const int rcap_opt = opts ? opts->rec_cap : 0;
  pl.n = n;
  pl.nm = nm;
  pl.L = L;
  pl.rcap = rcap_opt > 0 ? std::max(rcap_opt, 4) : rec_capacity<T>(n);
  const size_t optin = (size_t)dp.smem_optin;
  pl.k1b = n > 32 ? k1c_block<T>(n, optin) : 0;
  pl.zrows = 0;
  pl.zsplit = 1;
  if (n > 32) {
    // rows of Z that fit in shared memory next to the record buffers, at
    // most 256 (one thread per row); the fewest CTAs per matrix that hold
    // all rows, unless the caller asks for more
    const size_t fixed = k3c_smem_bytes<T>(n, 0);
    const size_t row = sizeof(T) * (size_t)(n | 1);
    const int rmax = fixed < optin ? (int)std::min<size_t>(256, (optin - fixed) / row) : 0;
    if (rmax >= 32 || rmax >= n) {
      int split = (n + rmax - 1) / rmax;
      const int want = opts ? opts->split : 0;
      if (want > split) split = std::min(want, (n + 31) / 32);
      pl.zsplit = split;
      pl.zrows = (n + split - 1) / split;
    } else if (fixed > optin) {
      return cudaErrorInvalidValue;
    }
    // tensor memory holds up to 128 rows of a matrix per part (rows of up
    // to 512 32-bit columns: FP64 n <= 256, FP32 n <= 512), unless that
    // takes more parts per matrix than shared memory does and leaves an SM
    // fewer warps: every part reads all of the matrix's records (measured
    // on B200: FP64 n = 160, two parts of 80 rows with one CTA per SM, is
    // slower than one shared-memory CTA of 160 rows; FP32 n = 200, two
    // parts of 100 rows with two CTAs per SM, is faster than one of 200)
    if (pl.zrows > 0 && tmem_cols<T>(n) > 0 && !(opts && opts->zmem == EIGEN_GPU_ZMEM_SHARED)) {
      int split = (n + 127) / 128;
      const int want = opts ? opts->split : 0;
      if (want > split) split = std::min(want, (n + 31) / 32);
      bool use = split <= pl.zsplit;
      if (!use) {
        const int zr_t = (n + split - 1) / split;
        const long warps_t = (long)(512 / tmem_cols<T>(n)) * ((zr_t + 31) / 32);
        const size_t foot_s = k3c_smem_bytes<T>(n, pl.zrows) + (size_t)dp.smem_rsv;
        const long ctas_s = std::max<long>(1, std::min<long>((long)dp.smem_sm / (long)foot_s,
                                                              2048 / (((pl.zrows + 31) / 32) * 32)));
        const long warps_s = ctas_s * ((pl.zrows + 31) / 32);
        use = warps_t >= warps_s;
      }
      if (use) {
        pl.zsplit = split;
        pl.zrows = (n + split - 1) / split;
        pl.ztm = 1;
      }
    }
  }
  const bool zglob = n > 32 && pl.zrows == 0;
  const size_t per = sizeof(T) * 2 * (size_t)n + sizeof(Meta) + sizeof(Rec<T>) * (size_t)pl.rcap +
                     (zglob ? sizeof(T) * (size_t)n * n : 0);
  long lc = (long)(kWsBudget / per);
  lc = std::max(lc, kMinChunk);
  if (lc < L) lc = (L + (L + lc - 1) / lc - 1) / ((L + lc - 1) / lc);  // equal chunks: phase 2
                                                                         // costs its latency per chunk
  if (opts && opts->chunk > 0) lc = opts->chunk;
  pl.Lc = std::min(L, lc);
  size_t off = 0;
  pl.off_d = off;
  off = align256(off + sizeof(T) * (size_t)n * pl.Lc);
  pl.off_e = off;
  off = align256(off + sizeof(T) * (size_t)n * pl.Lc);
  pl.off_meta = off;
  off = align256(off + sizeof(Meta) * (size_t)pl.Lc);
  pl.off_rec = off;
  off = align256(off + sizeof(Rec<T>) * (size_t)pl.rcap * pl.Lc);
  pl.off_z = off;
  if (zglob) off = align256(off + sizeof(T) * (size_t)n * n * pl.Lc);
  pl.bytes = off;
  return cudaSuccess;
}

bool bad_args(long L, int nm, int n, int m) { return L < 1 || nm < n || n < 1 || m < 1 || m > n || n > 1024; }

template <class T>
cudaError_t buffer_size(long L, int nm, int n, int m, size_t *lwork, const eigen_GPU_batch_opts *opts = nullptr)
{
  if (lwork) *lwork = 0;
  if (bad_args(L, nm, n, m)) return cudaErrorInvalidValue;
  if (n == 1) return cudaSuccess;
  if (opts && opts->method == EIGEN_GPU_BATCH_JACOBI) return cudaSuccess;
  DevProps dp;
  cudaError_t err = dev_props(dp);
  if (err != cudaSuccess) return err;
  eigen_GPU_batch_opts tuned_opts;
  opts = tuned(opts, (int)sizeof(T), n, tuned_opts);
  Plan<T> pl;
  if ((err = make_plan<T>(L, nm, n, dp, pl, opts)) != cudaSuccess) return err;
  if (lwork) *lwork = pl.bytes;
  return cudaSuccess;
}

template <class K> cudaError_t set_smem(K kern, size_t bytes)
{
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// phase 1 in registers for 32 < n <= 128 (NB = ceil(n/32) column blocks)
inline int reg_nb(int n) { return (n > 32 && n <= 128) ? (n + 31) / 32 : 0; }
template <class T> size_t k1r_smem_bytes(int n)
{
  switch (reg_nb(n)) {
    case 2: return sizeof(T) * reg_smem_elems<2>(n);
    case 3: return sizeof(T) * reg_smem_elems<3>(n);
    case 4: return sizeof(T) * reg_smem_elems<4>(n);
    default: return 0;
  }
}
template <class T> cudaError_t set_k1r_smem(int n, size_t bytes)
{
  switch (reg_nb(n)) {
    case 2: return set_smem(k1_reg<T, 2>, bytes);
    case 3: return set_smem(k1_reg<T, 3>, bytes);
    case 4: return set_smem(k1_reg<T, 4>, bytes);
    default: return cudaErrorInvalidValue;
  }
}
template <class T> void launch_k1r(const KP<T> &p, unsigned blocks, size_t smem, cudaStream_t st)
{
  const int nb = reg_nb(p.n);
  if (nb == 2) k1_reg<T, 2><<<blocks, 32 * 4, smem, st>>>(p);
  else if (nb == 3) k1_reg<T, 3><<<blocks, 32 * 9, smem, st>>>(p);
  else k1_reg<T, 4><<<blocks, 32 * 16, smem, st>>>(p);
}

// phase 1 on a cluster: usable when the device can hold one of its
// clusters (shared memory, cluster size; sizes above 8 need the
// non-portable opt-in)
template <class T> cudaLaunchConfig_t k1cl_config(int n, long cnt, cudaStream_t st, cudaLaunchAttribute *at)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(cnt * cl_cn(n)));
  cfg.blockDim = dim3(32 * K1CL_SPLIT);
  cfg.dynamicSmemBytes = cl_smem_bytes<T, K1CL_SPLIT>(n);
  cfg.stream = st;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)cl_cn(n);
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cfg;
}
template <class T> bool k1cl_usable(int n, const DevProps &dp)
{
  if (n <= 32 || n > 32 * CL_MAX_CN) return false;
  const size_t smem = cl_smem_bytes<T, K1CL_SPLIT>(n);
  if (smem > (size_t)dp.smem_optin) return false;
  if (set_smem(k1_cl<T>, smem) != cudaSuccess) return false;
  if (cl_cn(n) > 8 &&
      cudaFuncSetAttribute(k1_cl<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg = k1cl_config<T>(n, 1, nullptr, at);
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, k1_cl<T>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return clusters >= 1;
}
template <class T> cudaError_t launch_k1cl(const KP<T> &p, long cnt, cudaStream_t st)
{
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg = k1cl_config<T>(p.n, cnt, st, at);
  return cudaLaunchKernelEx(&cfg, k1_cl<T>, p);
}

template <class T> cudaError_t set_k1_smem(int n, size_t bytes)
{
  const int sp = k1_split<T>(n);
  if (sp == 4) return set_smem(k1_cta<T, 4>, bytes);
  if (sp == 2) return set_smem(k1_cta<T, 2>, bytes);
  return set_smem(k1_cta<T, 1>, bytes);
}

template <class T> void launch_k1(const KP<T> &p, unsigned blocks, int nt, size_t smem, cudaStream_t st)
{
  const int sp = k1_split<T>(p.n);
  if (sp == 4) k1_cta<T, 4><<<blocks, nt, smem, st>>>(p);
  else if (sp == 2) k1_cta<T, 2><<<blocks, nt, smem, st>>>(p);
  else k1_cta<T, 1><<<blocks, nt, smem, st>>>(p);
}

// Uneven batches: the L matrices of a call are matrices kid[0..L) of the
// caller's batch at a + aoff[.], w + woff[.], info[.] (see KP).
struct Indirect {
  const int *kid = nullptr;
  const long long *aoff = nullptr, *woff = nullptr;
};

// Part of a solve: the phases in `phases` (EIGEN_GPU_STAGE_* bits) for
// matrices first .. first+count-1 of the batch (count < 0: to its end).
struct Stage {
  long first = 0, count = -1;
  int phases = EIGEN_GPU_STAGE_ALL;
};

// ap: packed upper-triangle input (nullptr: the upper triangle of a); the
// eigenvectors go to a either way.  ix: see Indirect.  sg: a part of the
// solve; any part but the whole needs a workspace that holds the whole
// batch (one chunk), whose slot k belongs to matrix k.
template <class T>
cudaError_t run(long L, int nm, int n, int m, T *a, T *w, void *wk, size_t lwork, int *info,
                const eigen_GPU_batch_opts *opts, cudaStream_t stream, const T *ap = nullptr,
                const Indirect &ix = Indirect(), const Stage &sg = Stage())
{
  if (bad_args(L, nm, n, m) || a == nullptr || w == nullptr) return cudaErrorInvalidValue;
  eigen_GPU_batch_opts tuned_opts;
  opts = tuned(opts, (int)sizeof(T), n, tuned_opts);
  const long first = sg.first, count = sg.count <= 0 ? L - sg.first : sg.count;
  if (first < 0 || count < 1 || first + count > L || sg.phases < 1 || sg.phases > EIGEN_GPU_STAGE_ALL)
    return cudaErrorInvalidValue;
  const bool ranged = first != 0 || count != L || sg.phases != EIGEN_GPU_STAGE_ALL;
  int method = EIGEN_GPU_BATCH_TQL2, sort = 1, max_sweep = 100;
  if (opts) {
    method = opts->method;
    sort = opts->sort ? 1 : 0;
    if (opts->max_sweep > 0) max_sweep = opts->max_sweep;
  }
  if (method < EIGEN_GPU_BATCH_TQL2 || method > EIGEN_GPU_BATCH_JACOBI) return cudaErrorInvalidValue;
  if (method == EIGEN_GPU_BATCH_JACOBI && n > 32) return cudaErrorInvalidValue;
  cudaError_t err;
  KP<T> p{};
  p.n = n;
  p.nm = nm;
  p.kid = ix.kid;
  p.aoff = ix.aoff;
  p.woff = ix.woff;
  // n = 1 and the Jacobi method are one pass each: a part runs it for its
  // matrices with the apply bit and does nothing for the others
  if ((n == 1 || method == EIGEN_GPU_BATCH_JACOBI) && !(sg.phases & EIGEN_GPU_STAGE_APPLY)) return cudaSuccess;
  if (n == 1) {
    p.a = a + (size_t)first * nm * n;
    p.w = w + (size_t)first * n;
    p.ap = ap ? ap + (size_t)first * packed_size(n) : nullptr;
    p.info = info ? info + first : nullptr;
    p.Lc = count;
    const int blocks = (int)std::min<long>((count + 255) / 256, 4096);
    k_n1<T><<<blocks, 256, 0, stream>>>(p);
    return cudaGetLastError();
  }
  DevProps dp;
  if ((err = dev_props(dp)) != cudaSuccess) return err;

  p.method = (method == EIGEN_GPU_BATCH_IMTQL2) ? QL_IMTQL2 : QL_TQL2;
  p.max_sweep = max_sweep;
  p.sort = sort;

  if (method == EIGEN_GPU_BATCH_JACOBI) {
    const size_t smem = sizeof(JacSlot<T>) * K1W_NW;
    if ((err = set_smem(k_jacobi_warp<T>, smem)) != cudaSuccess) return err;
    p.a = a + (size_t)first * nm * n;
    p.w = w + (size_t)first * n;
    p.ap = ap ? ap + (size_t)first * packed_size(n) : nullptr;
    p.info = info ? info + first : nullptr;
    p.Lc = count;
    const long blocks = (count + K1W_NW - 1) / K1W_NW;
    k_jacobi_warp<T><<<(unsigned)blocks, 32 * K1W_NW, smem, stream>>>(p);
    return cudaGetLastError();
  }

  Plan<T> pl;
  if ((err = make_plan<T>(L, nm, n, dp, pl, opts)) != cudaSuccess) return err;
  if (wk == nullptr || (lwork != 0 && lwork < pl.bytes)) return cudaErrorInvalidValue;
  if (ranged && pl.Lc < L) return cudaErrorInvalidValue;  // a part needs the whole batch's workspace
  char *base = static_cast<char *>(wk);
  T *const ws_d = reinterpret_cast<T *>(base + pl.off_d);
  T *const ws_e = reinterpret_cast<T *>(base + pl.off_e);
  Meta *const ws_meta = reinterpret_cast<Meta *>(base + pl.off_meta);
  Rec<T> *const ws_rec = reinterpret_cast<Rec<T> *>(base + pl.off_rec);
  T *const ws_z = reinterpret_cast<T *>(base + pl.off_z);
  p.rcap = pl.rcap;

  // launch geometry
  const size_t k1w_smem = sizeof(T) * k1w_slot<T>() * K1W_NW;
  const size_t k3w_smem = sizeof(K3WSlot<T>) * K3W_NW;
  // phase 3: one row per thread up to 512 rows, two above
  bool ztm = pl.ztm != 0 && n > 32;
  int k3_nt = pl.zrows > 0 ? ((pl.zrows + 31) / 32) * 32
                        : (n > 512 ? (((n + 1) / 2 + 31) / 32) * 32 : ((n + 31) / 32) * 32);
  p.zrows = pl.zrows;
  p.zsplit = pl.zsplit;
  p.k1b = pl.k1b;
  const int k1c_nt = k1c_threads<T>(n);
  const int red_form = tuned_reduce((int)sizeof(T), n);
  const bool k1_cluster = red_form == EIGEN_GPU_REDUCE_CLUSTER && k1cl_usable<T>(n, dp);
  const bool k1_in_regs = !k1_cluster && reg_nb(n) > 0 && k1r_smem_bytes<T>(n) <= (size_t)dp.smem_optin;
  const size_t k1c_smem = k1_in_regs ? k1r_smem_bytes<T>(n) : sizeof(T) * k1c_smem_elems(n, k1c_nt, pl.k1b);
  size_t k3c_smem = k3c_smem_bytes<T>(n, ztm ? 0 : pl.zrows);
  int k3_wpp = 0, k3_parts = 0, k3_acols = 0;  // tensor-memory form: warps per part, parts per CTA, columns
  // sweeps per pass: up to eight for rows of 256 or more, four for rows of
  // 128 .. 255, pairs below 128 (measured on B200: the longer groups give
  // each thread more independent rotation chains, at 254 registers, which
  // costs the CTAs that share an SM; at FP64 n=128 eight save 0.12 ms of
  // phase 3 alone but lose 1.7 ms of a host-to-host solve, where the other
  // chunks' phase-1/2 CTAs run beside phase 3)
  void (*k3t)(const KP<T>, const int, const int) =
      n < 128 ? k3_tmem<T, 1> : (n >= 256 ? k3_tmem<T, 8> : k3_tmem<T, 4>);
  if (ztm) {
    // Tensor memory is allocated per CTA, and the CTAs on one SM must never
    // ask for more than its 512 columns together (an allocation would wait
    // for another CTA's columns).  Each CTA therefore requests shared memory
    // in proportion to its columns, acols/512 of the SM's (reserve
    // included): whatever mix of these CTAs, from any launch or stream,
    // shares an SM holds at most 512 columns.  A CTA is at most four warps
    // (one per lane quarter): two parts of two warps where a part has at
    // most 64 rows, unless the chunk is too small to fill the SMs.
    k3_acols = tmem_cols<T>(n);
    k3_wpp = (pl.zrows + 31) / 32;
    const long spread = (std::min(count, pl.Lc) * pl.zsplit + dp.sms - 1) / dp.sms;
    k3_parts = (int)std::max(1L, std::min<long>(4 / k3_wpp, spread));
    // (the kernel's own static shared memory, 16 bytes, is within the 64
    // left out; that slack cannot add up to another CTA's share)
    const size_t fixed = k3c_fixed_bytes<T>(n, K3_TM_SWEEPS) * (size_t)k3_parts;
    const size_t foot = (size_t)dp.smem_sm * (size_t)k3_acols / 512;
    const size_t other = (size_t)dp.smem_rsv + 64;
    k3c_smem = std::max(fixed, foot > other ? foot - other : 0);
    int nb = 0;
    bool ok = k3c_smem + 64 <= (size_t)dp.smem_optin;
    if (ok) {
      if ((err = set_smem(k3t, k3c_smem)) != cudaSuccess) return err;
      if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k3t, 32 * k3_wpp * k3_parts,
                                                               k3c_smem)) != cudaSuccess)
        return err;
      ok = nb >= 1 && nb * k3_acols <= 512;
    }
    if (!ok) {  // the shared-memory plan, which uses the same workspace layout
      eigen_GPU_batch_opts o = opts ? *opts : eigen_GPU_batch_opts{};
      o.zmem = EIGEN_GPU_ZMEM_SHARED;
      if ((err = make_plan<T>(L, nm, n, dp, pl, &o)) != cudaSuccess) return err;
      ztm = false;
      p.zrows = pl.zrows;
      p.zsplit = pl.zsplit;
      k3_nt = ((pl.zrows + 31) / 32) * 32;
      k3c_smem = k3c_smem_bytes<T>(n, pl.zrows);
    }
  }
  const bool zsm = pl.zrows > 0 && !ztm;
  // phase 2: matrices per warp, then warps per block within the shared
  // memory budget (2n values per matrix)
  p.k2mpw = k2_mpw(std::min(count, pl.Lc), dp.sms);
  if (opts && opts->ql_mpw > 0) {
    const int q = opts->ql_mpw;
    if (q > 32 || (q & (q - 1)) != 0) return cudaErrorInvalidValue;
    p.k2mpw = q;
  }
  int k2_mpb = 32;  // matrices per block, a multiple of k2mpw
  {
    const size_t per = k2_smem_per_thread<T>(n);
    const size_t budget = std::min<size_t>((size_t)dp.smem_optin, 96 * 1024);
    const int warps = (int)std::max<size_t>(
        1, std::min<size_t>(std::max(1, std::min(K2_MAX_WARPS, 32 / p.k2mpw)), budget / (per * p.k2mpw)));
    k2_mpb = warps * p.k2mpw;
    if ((size_t)k2_mpb * per > (size_t)dp.smem_optin) {
      p.k2mpw = 1;
      k2_mpb = 1;
      if (per > (size_t)dp.smem_optin) return cudaErrorInvalidValue;
    }
  }
  const size_t k2_smem = k2_smem_per_thread<T>(n) * k2_mpb;
  if (n <= 32) {
    if ((err = set_smem(k1_warp<T>, k1w_smem)) != cudaSuccess) return err;
    if ((err = set_smem(k3_warp<T>, k3w_smem)) != cudaSuccess) return err;
  } else {
    if (k1_cluster) {
      // attributes set by k1cl_usable
    } else if (k1_in_regs) {
      if ((err = set_k1r_smem<T>(n, k1c_smem)) != cudaSuccess) return err;
    } else if ((err = set_k1_smem<T>(n, k1c_smem)) != cudaSuccess) {
      return err;
    }
    if (ztm) {
      // attribute set with the launch geometry above
    } else if (zsm) {
      if ((err = set_smem(k3_cta<T, true, 1>, k3c_smem)) != cudaSuccess) return err;
    } else if ((err = set_smem(n > 512 ? k3_cta<T, false, 2> : k3_cta<T, false, 1>, k3c_smem)) != cudaSuccess) {
      return err;
    }
  }
  if ((err = set_smem(k2_ql<T>, k2_smem)) != cudaSuccess) return err;

  // the three phase launches of cnt matrices described by q, on st
  cudaError_t lerr = cudaSuccess;  // a launch error returned rather than left for cudaGetLastError
  auto phase1 = [&](const KP<T> &q, long cnt, cudaStream_t st) {
    if (n <= 32) {
      k1_warp<T><<<(unsigned)((cnt + K1W_NW - 1) / K1W_NW), 32 * K1W_NW, k1w_smem, st>>>(q);
    } else if (k1_cluster) {
      const cudaError_t e = launch_k1cl<T>(q, cnt, st);
      if (e != cudaSuccess && lerr == cudaSuccess) lerr = e;
    } else if (k1_in_regs) {
      launch_k1r<T>(q, (unsigned)cnt, k1c_smem, st);
    } else {
      launch_k1<T>(q, (unsigned)cnt, k1c_nt, k1c_smem, st);
    }
  };
  auto phase2 = [&](const KP<T> &q, long cnt, cudaStream_t st) {
    k2_ql<T><<<(unsigned)((cnt + k2_mpb - 1) / k2_mpb), 32 * (k2_mpb / q.k2mpw), k2_smem, st>>>(q);
  };
  auto phase3 = [&](const KP<T> &q, long cnt, cudaStream_t st) {
    if (n <= 32) {
      k3_warp<T><<<(unsigned)((cnt + K3W_NW - 1) / K3W_NW), 32 * K3W_NW, k3w_smem, st>>>(q);
    } else if (ztm) {
      const long nparts = cnt * pl.zsplit;
      k3t<<<(unsigned)((nparts + k3_parts - 1) / k3_parts), 32 * k3_wpp * k3_parts, k3c_smem, st>>>(
          q, k3_wpp, k3_acols);
    } else if (zsm) {
      k3_cta<T, true, 1><<<(unsigned)(cnt * pl.zsplit), k3_nt, k3c_smem, st>>>(q);
    } else if (n > 512) {
      k3_cta<T, false, 2><<<(unsigned)cnt, k3_nt, k3c_smem, st>>>(q);
    } else {
      k3_cta<T, false, 1><<<(unsigned)cnt, k3_nt, k3c_smem, st>>>(q);
    }
  };
  for (long c0 = first; c0 < first + count; c0 += pl.Lc) {
    const long lc = std::min(pl.Lc, first + count - c0);
    const long chunk = (c0 - first) / pl.Lc;
    // workspace slot of the chunk's first matrix: chunks reuse the
    // workspace from slot 0; a part of the solve uses the matrices' own
    const size_t wo = ranged ? (size_t)c0 : 0;
    p.d = ws_d + wo * n;
    p.e = ws_e + wo * n;
    p.meta = ws_meta + wo;
    p.rec = ws_rec + wo * (size_t)pl.rcap;
    p.zs = ws_z + wo * (size_t)n * n;
    if (ix.kid) {  // the index list advances instead of the pointers
      p.a = a;
      p.w = w;
      p.info = info;
      p.kid = ix.kid + c0;
      p.ap = nullptr;
    } else {
      p.a = a + (size_t)c0 * nm * n;
      p.w = w + (size_t)c0 * n;
      p.ap = ap ? ap + (size_t)c0 * packed_size(n) : nullptr;
      p.info = info ? info + c0 : nullptr;
    }
    p.Lc = lc;
    trace(chunk, 0, stream);
    if (sg.phases & EIGEN_GPU_STAGE_REDUCE) phase1(p, lc, stream);
    trace(chunk, 1, stream);
    if (sg.phases & EIGEN_GPU_STAGE_QL) phase2(p, lc, stream);
    trace(chunk, 2, stream);
    if (sg.phases & EIGEN_GPU_STAGE_APPLY) phase3(p, lc, stream);
    trace(chunk, 3, stream);
    if (lerr != cudaSuccess) return lerr;
    if ((err = cudaGetLastError()) != cudaSuccess) return err;
  }
  return cudaSuccess;
}

// Launch geometry of phase 1 (the matrix-parallel reduction) for the first
// chunk of a default solve, as run() launches it; the counterpart of the
// reference's eigen_GPU_batch_get_Launch_params (eigen_GPU_batch.hpp:23-102).
template <class T>
cudaError_t launch_params(long L, int n, int *grp, int *tb, int *gr, int *th, int *sh, int *l2)
{
  if (!grp || !tb || !gr || !th || !sh || !l2) return cudaErrorInvalidValue;
  *grp = *tb = *gr = *th = *sh = *l2 = 0;
  if (bad_args(L, n, n, n)) return cudaErrorInvalidValue;
  DevProps dp;
  cudaError_t err = dev_props(dp);
  if (err != cudaSuccess) return err;
  *l2 = dp.l2;
  if (n == 1) {  // k_n1: one thread per matrix
    *grp = 1;
    *gr = 256;
    *th = 256;
    *tb = (int)std::min<long>((L + 255) / 256, 4096);
    return cudaSuccess;
  }
  Plan<T> pl;
  if ((err = make_plan<T>(L, n, n, dp, pl, nullptr)) != cudaSuccess) return err;
  const long lc = std::min(L, pl.Lc);
  const int red_form = tuned_reduce((int)sizeof(T), n);
  if (n > 32 && red_form == EIGEN_GPU_REDUCE_CLUSTER && k1cl_usable<T>(n, dp)) {  // k1_cl: ceil(n/32) blocks per matrix
    *th = 32 * K1CL_SPLIT;
    *grp = cl_cn(n) * *th;
    *gr = 1;
    *tb = (int)(lc * cl_cn(n));
    *sh = (int)cl_smem_bytes<T, K1CL_SPLIT>(n);
  } else if (n <= 32) {  // k1_warp: one warp per matrix
    *grp = 32;
    *gr = K1W_NW;
    *th = 32 * K1W_NW;
    *tb = (int)((lc + K1W_NW - 1) / K1W_NW);
    *sh = (int)(sizeof(T) * k1w_slot<T>() * K1W_NW);
  } else if (reg_nb(n) > 0 && k1r_smem_bytes<T>(n) <= (size_t)dp.smem_optin) {  // k1_reg: NB x NB warps
    const int nb = reg_nb(n);
    *grp = *th = 32 * nb * nb;
    *gr = 1;
    *tb = (int)lc;
    *sh = (int)k1r_smem_bytes<T>(n);
  } else {  // k1_cta
    *grp = *th = k1c_threads<T>(n);
    *gr = 1;
    *tb = (int)lc;
    *sh = (int)(sizeof(T) * k1c_smem_elems(n, k1c_threads<T>(n), pl.k1b));
  }
  return cudaSuccess;
}

// ---- interleaved layout ----
//
// Element (i, j) of matrix k at ai[(i + j*n)*L + k], eigenvalue j of matrix
// k at wi[j*L + k].  Transposed into the workspace, solved there, and
// transposed back.
template <class T> cudaError_t transpose(long rows, long cols, const T *in, T *out, cudaStream_t st)
{
  const long gx = (cols + 31) / 32, gy = (rows + 31) / 32;
  if (gx > 0x7fffffffL || gy > 65535) return cudaErrorInvalidValue;
  k_transpose<T><<<dim3((unsigned)gx, (unsigned)gy), 256, 0, st>>>(rows, cols, in, out);
  return cudaGetLastError();
}

template <class T>
cudaError_t interleaved_plan(long L, int n, const eigen_GPU_batch_opts *opts, size_t &off_w, size_t &off_ws,
                             size_t &bytes)
{
  size_t inner = 0;
  cudaError_t err = buffer_size<T>(L, n, n, n, &inner, opts);
  if (err != cudaSuccess) return err;
  off_w = align256(sizeof(T) * (size_t)L * n * n);
  off_ws = align256(off_w + sizeof(T) * (size_t)L * n);
  bytes = off_ws + inner;
  return cudaSuccess;
}

template <class T>
cudaError_t run_interleaved(long L, int n, const T *ai, T *zi, T *wi, void *wk, size_t lwork, int *info,
                            const eigen_GPU_batch_opts *opts, cudaStream_t stream)
{
  if (bad_args(L, n, n, n) || ai == nullptr || zi == nullptr || wi == nullptr || wk == nullptr)
    return cudaErrorInvalidValue;
  size_t off_w, off_ws, bytes;
  cudaError_t err = interleaved_plan<T>(L, n, opts, off_w, off_ws, bytes);
  if (err != cudaSuccess) return err;
  if (lwork < bytes) return cudaErrorInvalidValue;
  char *base = static_cast<char *>(wk);
  T *a = reinterpret_cast<T *>(base);
  T *w = reinterpret_cast<T *>(base + off_w);
  const long E = (long)n * n;
  if ((err = transpose<T>(E, L, ai, a, stream)) != cudaSuccess) return err;  // (E x L) -> (L x E)
  if ((err = run<T>(L, n, n, n, a, w, base + off_ws, lwork - off_ws, info, opts, stream)) != cudaSuccess)
    return err;
  if ((err = transpose<T>(L, E, a, zi, stream)) != cudaSuccess) return err;  // (L x E) -> (E x L)
  return transpose<T>(L, n, w, wi, stream);
}

// ---- uneven batches ----
//
// Matrix k has order n_k (1 <= n_k <= 1024), column-major with leading
// dimension n_k at a + sum_{j<k} n_j^2; its eigenvalues at w + sum_{j<k} n_j.
// The host groups the matrices by order, largest first, and cuts the groups
// into waves whose workspaces fit the budget together.  In each wave the
// reduction of every group runs like a uniform batch (reaching its members
// through an index list) on one of a pool of streams, groups placed
// longest-first on the least loaded stream; then one persistent launch
// (k2_ql_queue) runs the QL recurrence of every matrix of the wave from a
// device work queue, longest first; then each group's apply phase runs on
// its stream again.  Orders 1 and the Jacobi method are one pass each and
// run beside the first wave's reductions.
constexpr int kUnevenStreams = 32;

struct UnevenItem {            // matrices start .. start+count-1 of the grouped index list, one order
  int n = 0, start = 0, count = 0, stream = 0;
  bool single = false;         // n == 1 or the Jacobi method: one pass, no workspace
  size_t ws_off = 0, ws_bytes = 0;  // workspace of the item within its wave's region
  eigen_GPU_batch_opts opts{};
};
struct UnevenWave {
  int first = 0, count = 0;    // items
  int job0 = 0, njobs = 0;     // jobs of the QL queue
  int nmax = 0;                // largest order with a QL phase
};
struct UnevenPlan {
  std::vector<int> kid;  // matrix indices, grouped
  std::vector<long long> aoff, woff;
  std::vector<UnevenItem> items;
  std::vector<UnevenWave> waves;
  std::vector<QJob> jobs;
  int nstreams = 0, mpw = 4, method = QL_TQL2, max_sweep = 100;
  size_t off_kid = 0, off_aoff = 0, off_woff = 0, off_groups = 0, off_jobs = 0, off_next = 0, off_region = 0;
  size_t region = 0, bytes = 0;
};

template <class T>
cudaError_t make_uneven_plan(long L, const int *n_host, const eigen_GPU_batch_opts *opts, UnevenPlan &up)
{
  if (L < 1 || n_host == nullptr) return cudaErrorInvalidValue;
  const int method = opts ? opts->method : EIGEN_GPU_BATCH_TQL2;
  if (method < EIGEN_GPU_BATCH_TQL2 || method > EIGEN_GPU_BATCH_JACOBI) return cudaErrorInvalidValue;
  if (opts && opts->ql_mpw > 0 && (opts->ql_mpw > 32 || (opts->ql_mpw & (opts->ql_mpw - 1)) != 0))
    return cudaErrorInvalidValue;
  std::map<int, std::vector<int>, std::greater<int>> by_n;  // largest order first
  up.aoff.resize(L);
  up.woff.resize(L);
  long long ao = 0, wo = 0;
  for (long k = 0; k < L; k++) {
    const int n = n_host[k];
    if (n < 1 || n > 1024) return cudaErrorInvalidValue;
    if (method == EIGEN_GPU_BATCH_JACOBI && n > 32) return cudaErrorInvalidValue;
    up.aoff[k] = ao;
    up.woff[k] = wo;
    ao += (long long)n * n;
    wo += n;
    by_n[n].push_back((int)k);
  }
  DevProps dp;
  cudaError_t err = dev_props(dp);
  if (err != cudaSuccess) return err;
  up.method = method == EIGEN_GPU_BATCH_IMTQL2 ? QL_IMTQL2 : QL_TQL2;
  if (opts && opts->max_sweep > 0) up.max_sweep = opts->max_sweep;
  if (opts && opts->ql_mpw > 0) up.mpw = opts->ql_mpw;
  // items: whole groups, or parts of a group whose workspace alone is over
  // the budget; single-pass groups go to the first wave
  std::vector<UnevenItem> multi, single;
  for (auto &g : by_n) {
    UnevenItem it;
    it.n = g.first;
    it.start = (int)up.kid.size();
    it.count = (int)g.second.size();
    up.kid.insert(up.kid.end(), g.second.begin(), g.second.end());
    it.opts = opts ? *opts : eigen_GPU_batch_opts{};
    if (!opts) {
      it.opts.method = EIGEN_GPU_BATCH_TQL2;
      it.opts.sort = 1;
      it.opts.max_sweep = 100;
    }
    if (it.n == 1 || method == EIGEN_GPU_BATCH_JACOBI) {
      it.single = true;
      single.push_back(it);
      continue;
    }
    // the plan run() makes for one matrix of this order, tuned as it tunes
    eigen_GPU_batch_opts t1;
    eigen_GPU_batch_opts o1 = *tuned(&it.opts, (int)sizeof(T), it.n, t1);
    o1.chunk = 1;
    Plan<T> one;
    if ((err = make_plan<T>(1, it.n, it.n, dp, one, &o1)) != cudaSuccess) return err;
    long fit = std::max<long>(1, (long)(kWsBudget / one.bytes));
    if (opts && opts->chunk > 0) fit = std::min<long>(fit, opts->chunk);
    for (int s0 = 0; s0 < it.count; s0 += (int)std::min<long>(fit, it.count)) {
      UnevenItem part = it;
      part.start = it.start + s0;
      part.count = (int)std::min<long>(fit, it.count - s0);
      multi.push_back(part);
    }
  }
  // waves: consecutive items (decreasing order) while their workspaces fit
  // the budget together, and at most opts->chunk matrices when it is set
  up.nstreams = 1;
  size_t used = 0;
  long in_wave = 0;
  const long wave_cap = (opts && opts->chunk > 0) ? opts->chunk : (1L << 40);
  UnevenWave wv;
  auto close_wave = [&]() {
    if (wv.count > 0) up.waves.push_back(wv);
    wv = UnevenWave();
    wv.first = (int)up.items.size();
    used = 0;
    in_wave = 0;
  };
  close_wave();
  for (UnevenItem it : multi) {
    eigen_GPU_batch_opts t1;
    eigen_GPU_batch_opts oc = *tuned(&it.opts, (int)sizeof(T), it.n, t1);
    oc.chunk = it.count;
    Plan<T> pl;
    if ((err = make_plan<T>(it.count, it.n, it.n, dp, pl, &oc)) != cudaSuccess) return err;
    const size_t b = align256(pl.bytes);
    if (wv.count > 0 && (used + b > kWsBudget || in_wave + it.count > wave_cap)) close_wave();
    it.opts.chunk = it.count;
    it.ws_off = used;
    it.ws_bytes = pl.bytes;
    used += b;
    in_wave += it.count;
    up.region = std::max(up.region, used);
    up.items.push_back(it);
    wv.count++;
  }
  close_wave();
  for (UnevenItem it : single) up.items.push_back(it);  // after the waves' items
  // streams: within a wave (and for the single-pass items, with the first
  // wave), longest first onto the least loaded stream
  const int nwaves = (int)up.waves.size();
  for (int wi = 0; wi < std::max(1, nwaves); wi++) {
    std::vector<int> idx;
    if (wi < nwaves)
      for (int i = 0; i < up.waves[wi].count; i++) idx.push_back(up.waves[wi].first + i);
    if (wi == 0)
      for (int i = (int)up.items.size() - (int)single.size(); i < (int)up.items.size(); i++) idx.push_back(i);
    auto cost = [&](int i) { return (double)up.items[i].count * up.items[i].n * up.items[i].n * up.items[i].n; };
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return cost(x) > cost(y); });
    const int ns = (int)std::min<size_t>(kUnevenStreams, idx.size());
    up.nstreams = std::max(up.nstreams, ns);
    std::vector<double> load(std::max(ns, 1), 0.0);
    for (int i : idx) {
      const int s = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      up.items[i].stream = s;
      load[s] += cost(i);
    }
  }
  // the QL queue of each wave: its items' matrices in item order (items are
  // in decreasing order of n already)
  for (UnevenWave &w : up.waves) {
    w.job0 = (int)up.jobs.size();
    for (int i = w.first; i < w.first + w.count; i++) {
      w.nmax = std::max(w.nmax, up.items[i].n);
      for (int k = 0; k < up.items[i].count; k++) up.jobs.push_back(QJob{i, k});
    }
    w.njobs = (int)up.jobs.size() - w.job0;
  }
  size_t off = 0;
  up.off_kid = off;
  off = align256(off + sizeof(int) * (size_t)L);
  up.off_aoff = off;
  off = align256(off + sizeof(long long) * (size_t)L);
  up.off_woff = off;
  off = align256(off + sizeof(long long) * (size_t)L);
  up.off_groups = off;
  off = align256(off + sizeof(QGroup<T>) * up.items.size());
  up.off_jobs = off;
  off = align256(off + sizeof(QJob) * std::max<size_t>(1, up.jobs.size()));
  up.off_next = off;
  off = align256(off + sizeof(int) * std::max<size_t>(1, up.waves.size()));
  up.off_region = off;
  up.bytes = off + up.region;
  return cudaSuccess;
}

// pool of streams for the groups of uneven batches, created once per device
cudaStream_t g_ustream[kMaxDev][kUnevenStreams];
cudaError_t uneven_streams(int count, cudaStream_t *out)
{
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_mu);
  for (int i = 0; i < count; i++) {
    if (g_ustream[dev][i] == nullptr &&
        (err = cudaStreamCreateWithFlags(&g_ustream[dev][i], cudaStreamNonBlocking)) != cudaSuccess)
      return err;
    out[i] = g_ustream[dev][i];
  }
  return cudaSuccess;
}

template <class T>
cudaError_t uneven_buffer_size(long L, const int *n_host, const eigen_GPU_batch_opts *opts, size_t *lwork)
{
  if (lwork) *lwork = 0;
  UnevenPlan up;
  cudaError_t err = make_uneven_plan<T>(L, n_host, opts, up);
  if (err == cudaSuccess && lwork) *lwork = up.bytes;
  return err;
}

// Launch of the QL queue of one wave on st: matrices per warp up.mpw,
// warps per block within 96 KB of slots, one resident wave of blocks.
template <class T>
cudaError_t launch_ql_queue(const UnevenPlan &up, const UnevenWave &wv, const QGroup<T> *groups,
                            const QJob *jobs, int *next, cudaStream_t st)
{
  if (wv.njobs < 1) return cudaSuccess;
  DevProps dp;
  cudaError_t err = dev_props(dp);
  if (err != cudaSuccess) return err;
  const size_t per = queue_slot_bytes<T>(wv.nmax);
  const size_t budget = std::min<size_t>((size_t)dp.smem_optin, 96 * 1024);
  int mpw = up.mpw;
  int warps = (int)std::min<size_t>(std::max(1, std::min(K2_MAX_WARPS, 32 / mpw)), budget / (per * mpw));
  if (warps < 1) {  // one slot per warp
    mpw = 1;
    warps = (int)std::min<size_t>(K2_MAX_WARPS, std::max<size_t>(1, budget / per));
    if (per > (size_t)dp.smem_optin) return cudaErrorInvalidValue;
  }
  const size_t smem = per * (size_t)mpw * warps;
  if ((err = set_smem(k2_ql_queue<T>, smem)) != cudaSuccess) return err;
  int nb = 0;
  if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k2_ql_queue<T>, 32 * warps, smem)) != cudaSuccess)
    return err;
  const long need = (wv.njobs + (long)mpw * warps - 1) / ((long)mpw * warps);
  const long blocks = std::max<long>(1, std::min<long>(need, (long)std::max(nb, 1) * dp.sms));
  k2_ql_queue<T><<<(unsigned)blocks, 32 * warps, smem, st>>>(groups, jobs + wv.job0, wv.njobs, next, mpw, wv.nmax,
                                                               up.method, up.max_sweep);
  return cudaGetLastError();
}

template <class T>
cudaError_t run_uneven(long L, const int *n_host, T *a, T *w, void *wk, size_t lwork, int *info,
                       const eigen_GPU_batch_opts *opts, cudaStream_t stream)
{
  if (a == nullptr || w == nullptr || wk == nullptr) return cudaErrorInvalidValue;
  UnevenPlan up;
  cudaError_t err = make_uneven_plan<T>(L, n_host, opts, up);
  if (err != cudaSuccess) return err;
  if (lwork < up.bytes) return cudaErrorInvalidValue;
  char *base = static_cast<char *>(wk);
  int *d_kid = reinterpret_cast<int *>(base + up.off_kid);
  long long *d_aoff = reinterpret_cast<long long *>(base + up.off_aoff);
  long long *d_woff = reinterpret_cast<long long *>(base + up.off_woff);
  QGroup<T> *d_groups = reinterpret_cast<QGroup<T> *>(base + up.off_groups);
  QJob *d_jobs = reinterpret_cast<QJob *>(base + up.off_jobs);
  int *d_next = reinterpret_cast<int *>(base + up.off_next);
  char *region = base + up.off_region;
  // each item's workspace slots, as run() lays them out for its plan
  std::vector<QGroup<T>> qg(up.items.size());
  {
    DevProps dp;
    if ((err = dev_props(dp)) != cudaSuccess) return err;
    for (size_t i = 0; i < up.items.size(); i++) {
      const UnevenItem &it = up.items[i];
      if (it.single) continue;
      eigen_GPU_batch_opts t1;
      const eigen_GPU_batch_opts *o = tuned(&it.opts, (int)sizeof(T), it.n, t1);
      Plan<T> pl;
      if ((err = make_plan<T>(it.count, it.n, it.n, dp, pl, o)) != cudaSuccess) return err;
      if (pl.Lc < it.count || pl.bytes != it.ws_bytes) return cudaErrorInvalidValue;  // not reached
      char *ws = region + it.ws_off;
      qg[i].d = reinterpret_cast<T *>(ws + pl.off_d);
      qg[i].e = reinterpret_cast<T *>(ws + pl.off_e);
      qg[i].meta = reinterpret_cast<Meta *>(ws + pl.off_meta);
      qg[i].rec = reinterpret_cast<Rec<T> *>(ws + pl.off_rec);
      qg[i].n = it.n;
      qg[i].rcap = pl.rcap;
    }
  }
  // from pageable host memory: the copies are staged before these calls return
  if ((err = cudaMemcpyAsync(d_kid, up.kid.data(), sizeof(int) * (size_t)L, cudaMemcpyHostToDevice, stream)) ||
      (err = cudaMemcpyAsync(d_aoff, up.aoff.data(), sizeof(long long) * (size_t)L, cudaMemcpyHostToDevice,
                             stream)) ||
      (err = cudaMemcpyAsync(d_woff, up.woff.data(), sizeof(long long) * (size_t)L, cudaMemcpyHostToDevice,
                             stream)))
    return err;
  if (!up.items.empty() &&
      (err = cudaMemcpyAsync(d_groups, qg.data(), sizeof(QGroup<T>) * qg.size(), cudaMemcpyHostToDevice, stream)))
    return err;
  if (!up.jobs.empty() &&
      (err = cudaMemcpyAsync(d_jobs, up.jobs.data(), sizeof(QJob) * up.jobs.size(), cudaMemcpyHostToDevice, stream)))
    return err;
  if ((err = cudaMemsetAsync(d_next, 0, sizeof(int) * std::max<size_t>(1, up.waves.size()), stream))) return err;
  cudaStream_t st[kUnevenStreams];
  if ((err = uneven_streams(up.nstreams, st)) != cudaSuccess) return err;
  // one event per pool stream (joins) and one on the caller's stream (forks);
  // an event may be recorded again once the waits on it are enqueued
  cudaEvent_t ev[kUnevenStreams + 1];
  int nev = 0;
  for (; nev <= up.nstreams; nev++)
    if ((err = cudaEventCreateWithFlags(&ev[nev], cudaEventDisableTiming)) != cudaSuccess) break;
  auto fork = [&]() {
    cudaEventRecord(ev[up.nstreams], stream);
    for (int i = 0; i < up.nstreams; i++) cudaStreamWaitEvent(st[i], ev[up.nstreams], 0);
  };
  auto join = [&]() {
    for (int i = 0; i < up.nstreams; i++) {
      cudaEventRecord(ev[i], st[i]);
      cudaStreamWaitEvent(stream, ev[i], 0);
    }
  };
  auto stage = [&](const UnevenItem &it, int phases) {
    Indirect ix;
    ix.kid = d_kid + it.start;
    ix.aoff = d_aoff;
    ix.woff = d_woff;
    Stage sg;
    sg.phases = phases;
    return run<T>(it.count, it.n, it.n, it.n, a, w, it.single ? nullptr : region + it.ws_off, it.ws_bytes, info,
                  &it.opts, st[it.stream], nullptr, ix, sg);
  };
  if (err == cudaSuccess) {
    fork();
    const int nwaves = (int)up.waves.size();
    for (const UnevenItem &it : up.items)  // single-pass groups beside the first wave
      if (it.single && err == cudaSuccess) err = stage(it, EIGEN_GPU_STAGE_ALL);
    for (int wi = 0; wi < nwaves && err == cudaSuccess; wi++) {
      const UnevenWave &wv = up.waves[wi];
      if (wi > 0) {  // the previous wave's apply phase is done with the region
        join();
        fork();
      }
      for (int i = wv.first; i < wv.first + wv.count && err == cudaSuccess; i++)
        err = stage(up.items[i], EIGEN_GPU_STAGE_REDUCE);
      if (err != cudaSuccess) break;
      join();
      if ((err = launch_ql_queue<T>(up, wv, d_groups, d_jobs, d_next + wi, stream)) != cudaSuccess) break;
      fork();
      for (int i = wv.first; i < wv.first + wv.count && err == cudaSuccess; i++)
        err = stage(up.items[i], EIGEN_GPU_STAGE_APPLY);
    }
    join();  // the caller's stream waits for every pool stream
  }
  for (int i = 0; i < nev; i++) cudaEventDestroy(ev[i]);
  return err;
}

template <class T>
void dropin(const int L, const int nm, const int n, const int m, T *a, T *w, T *wk, cudaStream_t stream)
{
  if (wk == nullptr) {
    // size query: the byte count is written through w, a host pointer in
    // this mode (eigen_GPU_batch.cu:332-339); 0 for n == 1
    size_t lwork = 0;
    if (n > 1) buffer_size<T>(L, nm, n, m, &lwork);
    if (w) *reinterpret_cast<size_t *>(w) = lwork;
    return;
  }
  run<T>(L, nm, n, m, a, w, wk, 0, nullptr, nullptr, stream);
}

// ---- solve without any allocation: workspace in a static device array ----
//
// Callers that may not allocate device memory (a plugin's enqueue that runs
// under a framework-owned allocator, real-time loops that forbid
// allocation) can still solve through
// eigen_GPU_batch_noalloc_DP.  Its workspace is this file-scope array: every
// GPU that loads the library holds it until the process exits.  Host code
// only sees a stand-in for it, so its device address is taken with
// cudaGetSymbolAddress, once per device, with that device current.
constexpr size_t kNoallocScratchBytes = (size_t)64 << 20;  // 64 MiB per GPU
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];
void *g_noalloc_ptr[kMaxDev];

cudaError_t noalloc_scratch(void **out)
{
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_noalloc_ptr[dev] == nullptr) {
    void *p = nullptr;
    err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err != cudaSuccess) return err;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

template <class T>
cudaError_t run_noalloc(long L, int nm, int n, int m, T *a, T *w, int *info, cudaStream_t stream)
{
  if (bad_args(L, nm, n, m) || a == nullptr || w == nullptr) return cudaErrorInvalidValue;
  if (n == 1) return run<T>(L, nm, n, m, a, w, nullptr, 0, info, nullptr, stream);
  DevProps dp;
  cudaError_t err = dev_props(dp);
  if (err != cudaSuccess) return err;
  // largest chunk of matrices whose workspace fits in the static array
  eigen_GPU_batch_opts o{};
  o.method = EIGEN_GPU_BATCH_TQL2;
  o.sort = 1;
  o.chunk = 1;
  Plan<T> pl;
  if ((err = make_plan<T>(L, nm, n, dp, pl, &o)) != cudaSuccess) return err;
  if (pl.bytes > kNoallocScratchBytes) return cudaErrorInvalidValue;  // one matrix does not fit
  long chunk = std::min<long>(L, (long)(kNoallocScratchBytes / pl.bytes));
  while (chunk > 1) {
    o.chunk = (int)chunk;
    if ((err = make_plan<T>(L, nm, n, dp, pl, &o)) != cudaSuccess) return err;
    if (pl.bytes <= kNoallocScratchBytes) break;
    chunk--;
  }
  o.chunk = (int)chunk;
  void *scratch = nullptr;
  if ((err = noalloc_scratch(&scratch)) != cudaSuccess) return err;
  return run<T>(L, nm, n, m, a, w, scratch, kNoallocScratchBytes, info, &o, stream);
}

// ---- mixed precision with refinement (eigb_refine.cuh) ----
//
// Workspace: one chunk of Lc matrices (the FP32 solve and its workspace,
// the FP64 matrices of the refinement, the slices of the tensor-core
// products and the per-matrix state), then a batch-wide tail (the
// fallback's index list and offsets, counters).  The fallback's plain FP64
// solve reuses the chunk area.
struct RefLayout {
  long Lc = 0;
  int n = 0, Rp = 0, Kp = 0, KB = 0;
  size_t a32 = 0, w32 = 0, i32 = 0, ws32 = 0, ws32_bytes = 0;
  size_t af = 0, x0 = 0, x1 = 0, pe = 0, sm = 0, gm = 0;
  size_t as = 0, xs = 0, ps = 0, xr = 0, es = 0;
  size_t ea = 0, ex = 0, ep = 0, exr = 0, ee = 0;
  size_t lam = 0, sig = 0, act0 = 0, act1 = 0, conv = 0, fail = 0, emax = 0, ord = 0, cl = 0, W = 0;
  size_t chunk_bytes = 0;
  size_t fb = 0, aoff = 0, woff = 0, cnt = 0, bytes = 0;
};

constexpr int REF_S = 8;                   // slices of the FP64-accurate products
constexpr int REF_SX = 5, REF_SE = 4;      // slices of X and E in X E
constexpr int REF_DMAX = 9, REF_DMAX_XE = 8;

struct RefOpts {
  int max_iter = 3;
  double tol = 1e-14;
  int fallback = 1;
  int chunk = 0;
};

inline RefOpts ref_opts(const eigen_GPU_refine_opts *o)
{
  RefOpts r;
  if (o) {
    if (o->max_iter > 0) r.max_iter = o->max_iter;
    if (o->tol > 0) r.tol = o->tol;
    r.fallback = o->fallback ? 1 : 0;
    r.chunk = o->chunk;
  }
  return r;
}

inline eigen_GPU_batch_opts ref_opts32(long Lc)
{
  eigen_GPU_batch_opts o{};
  o.method = EIGEN_GPU_BATCH_TQL2;
  o.sort = 1;
  o.max_sweep = 100;
  o.chunk = (int)Lc;
  return o;
}

inline size_t ref_chunk_layout(long Lc, int nm, int n, const DevProps &dp, RefLayout &ly)
{
  ly.Lc = Lc;
  ly.n = n;
  ly.Rp = oz_rp(n);
  ly.Kp = oz_kp(n);
  ly.KB = oz_kb(n);
  const size_t nn = (size_t)n * n, sl = oz_slice_bytes(n), rp = (size_t)ly.Rp;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o = align256(o + bytes);
    return at;
  };
  ly.a32 = take(sizeof(float) * nn * Lc);
  ly.w32 = take(sizeof(float) * n * Lc);
  ly.i32 = take(sizeof(int) * Lc);
  Plan<float> pf;
  eigen_GPU_batch_opts o32 = ref_opts32(Lc);
  if (make_plan<float>(Lc, n, n, dp, pf, &o32) != cudaSuccess) return 0;
  ly.ws32_bytes = pf.bytes;
  ly.ws32 = take(pf.bytes);
  ly.af = take(sizeof(double) * nn * Lc);
  ly.x0 = take(sizeof(double) * nn * Lc);
  ly.x1 = take(sizeof(double) * nn * Lc);
  ly.pe = take(sizeof(double) * nn * Lc);
  ly.sm = take(sizeof(double) * nn * Lc);
  ly.gm = take(sizeof(double) * nn * Lc);
  ly.as = take(sl * REF_S * Lc);
  ly.xs = take(sl * REF_S * Lc);
  ly.ps = take(sl * REF_S * Lc);
  ly.xr = take(sl * REF_SX * Lc);
  ly.es = take(sl * REF_SE * Lc);
  ly.ea = take(sizeof(int) * rp * Lc);
  ly.ex = take(sizeof(int) * rp * Lc);
  ly.ep = take(sizeof(int) * rp * Lc);
  ly.exr = take(sizeof(int) * rp * Lc);
  ly.ee = take(sizeof(int) * rp * Lc);
  ly.lam = take(sizeof(double) * n * Lc);
  ly.sig = take(sizeof(double) * Lc);
  ly.act0 = take(sizeof(int) * Lc);
  ly.act1 = take(sizeof(int) * Lc);
  ly.conv = take(sizeof(int) * Lc);
  ly.fail = take(sizeof(int) * Lc);
  ly.emax = take(sizeof(double) * Lc);
  ly.ord = take(sizeof(int) * n * Lc);
  ly.cl = take(sizeof(int) * n * Lc);
  ly.W = take(sizeof(double) * (size_t)n * REF_CL_MAX * Lc);
  // the fallback's plain FP64 solve of up to Lc matrices reuses the area
  Plan<double> pd;
  eigen_GPU_batch_opts o64{};
  o64.chunk = (int)Lc;
  if (make_plan<double>(Lc, nm, n, dp, pd, &o64) != cudaSuccess) return 0;
  return std::max(o, pd.bytes);
}

inline cudaError_t ref_plan(long L, int nm, int n, const DevProps &dp, const RefOpts &ro, RefLayout &ly)
{
  long Lc = ro.chunk > 0 ? std::min<long>(L, ro.chunk) : L;
  size_t cb = 0;
  for (;;) {
    cb = ref_chunk_layout(Lc, nm, n, dp, ly);
    if (cb == 0) return cudaErrorInvalidValue;
    if (ro.chunk > 0 || cb <= kRefBudget || Lc <= 64) break;
    Lc = std::max<long>(64, (long)((double)Lc * (double)kRefBudget / (double)cb * 0.98));
    const long nch = (L + Lc - 1) / Lc;  // equal chunks
    Lc = (L + nch - 1) / nch;
  }
  ly.chunk_bytes = align256(cb);
  size_t o = ly.chunk_bytes;
  ly.fb = o;
  o = align256(o + sizeof(int) * L);
  ly.aoff = o;
  o = align256(o + sizeof(long long) * L);
  ly.woff = o;
  o = align256(o + sizeof(long long) * L);
  ly.cnt = o;  // fallback count, then the products' error flag
  o = align256(o + 2 * sizeof(int));
  ly.bytes = o;
  return cudaSuccess;
}

inline bool ref_bad_args(long L, int nm, int n) { return L < 1 || nm < n || n < 1 || n > 256; }

cudaError_t ref_buffer_size(long L, int nm, int n, const eigen_GPU_refine_opts *opts, size_t *lwork)
{
  if (lwork == nullptr) return cudaErrorInvalidValue;
  *lwork = 0;
  if (ref_bad_args(L, nm, n)) return cudaErrorInvalidValue;
  if (n == 1) return cudaSuccess;
  DevProps dp;
  cudaError_t err = dev_props(dp);
  if (err != cudaSuccess) return err;
  RefLayout ly;
  if ((err = ref_plan(L, nm, n, dp, ref_opts(opts), ly)) != cudaSuccess) return err;
  *lwork = ly.bytes;
  return cudaSuccess;
}

// one product of the refinement
inline void ref_gemm(const RefLayout &ly, long lc, const int8_t *Ls, const int *eL, int sL, const int8_t *Rs,
                     const int *eR, int sR, int dmax, double *out, const void *add, int add_f32, const int *act,
                     int *errf, size_t smem, cudaStream_t st)
{
  OzGemm g{};
  g.Ls = Ls;
  g.Rs = Rs;
  g.eL = eL;
  g.eR = eR;
  g.RpL = g.RpR = ly.Rp;
  g.Kp = ly.Kp;
  g.KB = ly.KB;
  g.sL = sL;
  g.sR = sR;
  g.dmax = dmax;
  g.n = ly.n;
  g.mtiles = ly.Rp / OZ_MT;
  g.ntiles = (ly.n + OZ_NT - 1) / OZ_NT;
  g.out = out;
  g.ob = (long long)ly.n * ly.n;
  g.ldo = ly.n;
  g.add = add;
  g.add_f32 = add_f32;
  g.ab = (long long)ly.n * ly.n;
  g.lda = ly.n;
  g.active = act;
  g.err = errf;
  const long tiles = lc * g.mtiles * g.ntiles;
  k_oz_gemm<<<(unsigned)tiles, OZ_THREADS, smem, st>>>(g);
}

inline void ref_slice(const RefLayout &ly, long lc, const void *src, int f32, int rs, int ks, int s, int8_t *out,
                      int *e, const int *act, cudaStream_t st)
{
  OzSlice q{};
  q.src = src;
  q.src_f32 = f32;
  q.bs = (long long)ly.n * ly.n;
  q.rs = rs;
  q.ks = ks;
  q.R = ly.n;
  q.K = ly.n;
  q.Rp = ly.Rp;
  q.Kp = ly.Kp;
  q.KB = ly.KB;
  q.s = s;
  q.out = out;
  q.e = e;
  q.active = act;
  const int rpb = 256 / (ly.Kp / 16);
  dim3 grid((unsigned)lc, (unsigned)((ly.Rp + rpb - 1) / rpb));
  k_oz_slice<><<<grid, 256, 0, st>>>(q);
}

cudaError_t run_refine(long L, int nm, int n, double *a, double *w, void *wk, size_t lwork, int *info, int *iters,
                       const eigen_GPU_refine_opts *opts, cudaStream_t stream)
{
  if (ref_bad_args(L, nm, n) || a == nullptr || w == nullptr) return cudaErrorInvalidValue;
  if (n == 1) {
    cudaError_t e1 = run<double>(L, nm, n, n, a, w, nullptr, 0, info, nullptr, stream);
    if (e1 == cudaSuccess && iters) e1 = cudaMemsetAsync(iters, 0, sizeof(int) * L, stream);
    return e1;
  }
  DevProps dp;
  cudaError_t err = dev_props(dp);
  if (err != cudaSuccess) return err;
  const RefOpts ro = ref_opts(opts);
  RefLayout ly;
  if ((err = ref_plan(L, nm, n, dp, ro, ly)) != cudaSuccess) return err;
  if (wk == nullptr || (lwork != 0 && lwork < ly.bytes)) return cudaErrorInvalidValue;
  char *base = static_cast<char *>(wk);
  auto P = [&](size_t off) { return static_cast<void *>(base + off); };
  int *fb_list = static_cast<int *>(P(ly.fb));
  int *cnt = static_cast<int *>(P(ly.cnt));
  int *errf = cnt + 1;
  if ((err = cudaMemsetAsync(cnt, 0, 2 * sizeof(int), stream)) != cudaSuccess) return err;
  // shared memory of the products: their operands, and at least half of
  // the SM so that no two of these CTAs (512 TMEM columns each) share an SM
  const size_t need = std::max(oz_gemm_smem(REF_S, REF_S, ly.KB, REF_DMAX), oz_gemm_smem(REF_SX, REF_SE, ly.KB, REF_DMAX_XE));
  const size_t gsm = std::min<size_t>(oz_launch_smem(need, 2, dp.smem_sm, dp.smem_rsv), (size_t)dp.smem_optin);
  if (need > (size_t)dp.smem_optin) return cudaErrorInvalidValue;
  if ((err = set_smem(k_oz_gemm, gsm)) != cudaSuccess) return err;
  const size_t usm = ref_update_smem(n);
  if ((err = set_smem(k_oa_update, usm)) != cudaSuccess) return err;
  const size_t fsm = (sizeof(double) + sizeof(int)) * (size_t)n + 64;
  const eigen_GPU_batch_opts o32 = ref_opts32(ly.Lc);
  float *A32 = static_cast<float *>(P(ly.a32));
  double *Af = static_cast<double *>(P(ly.af));
  double *XB[2] = {static_cast<double *>(P(ly.x0)), static_cast<double *>(P(ly.x1))};
  double *PE = static_cast<double *>(P(ly.pe));
  double *Sm = static_cast<double *>(P(ly.sm));
  double *Gm = static_cast<double *>(P(ly.gm));
  int8_t *AS = static_cast<int8_t *>(P(ly.as)), *XS = static_cast<int8_t *>(P(ly.xs));
  int8_t *PS = static_cast<int8_t *>(P(ly.ps)), *XR = static_cast<int8_t *>(P(ly.xr));
  int8_t *ES = static_cast<int8_t *>(P(ly.es));
  int *eA = static_cast<int *>(P(ly.ea)), *eX = static_cast<int *>(P(ly.ex)), *eP = static_cast<int *>(P(ly.ep));
  int *eXR = static_cast<int *>(P(ly.exr)), *eE = static_cast<int *>(P(ly.ee));
  int *act[2] = {static_cast<int *>(P(ly.act0)), static_cast<int *>(P(ly.act1))};
  int *conv = static_cast<int *>(P(ly.conv)), *fail = static_cast<int *>(P(ly.fail));
  for (long c0 = 0; c0 < L; c0 += ly.Lc) {
    const long lc = std::min(ly.Lc, L - c0);
    k_ref_prep<<<(unsigned)lc, 256, 0, stream>>>(a + (size_t)c0 * nm * n, nm, n, Af, A32,
                                                 static_cast<double *>(P(ly.sig)), 1);
    if ((err = run<float>(lc, n, n, n, A32, static_cast<float *>(P(ly.w32)), P(ly.ws32), ly.ws32_bytes,
                          static_cast<int *>(P(ly.i32)), &o32, stream)) != cudaSuccess)
      return err;
    k_ref_init<<<(unsigned)((lc + 255) / 256), 256, 0, stream>>>(lc, static_cast<int *>(P(ly.i32)), act[0], conv,
                                                                 fail);
    ref_slice(ly, lc, Af, 0, n, 1, REF_S, AS, eA, act[0], stream);
    for (int it = 1; it <= ro.max_iter; it++) {
      const int *ain = act[(it - 1) & 1];
      int *aout = act[it & 1];
      const void *Xs = it == 1 ? static_cast<const void *>(A32) : static_cast<const void *>(XB[it & 1]);
      const int xf32 = it == 1 ? 1 : 0;
      double *Xd = XB[(it - 1) & 1];
      ref_slice(ly, lc, Xs, xf32, n, 1, REF_S, XS, eX, ain, stream);             // columns of X
      ref_gemm(ly, lc, AS, eA, REF_S, XS, eX, REF_S, REF_DMAX, PE, nullptr, 0, ain, errf, gsm, stream);  // P = Af X
      ref_slice(ly, lc, PE, 0, n, 1, REF_S, PS, eP, ain, stream);
      ref_gemm(ly, lc, XS, eX, REF_S, PS, eP, REF_S, REF_DMAX, Sm, nullptr, 0, ain, errf, gsm, stream);  // S = X^T P
      ref_gemm(ly, lc, XS, eX, REF_S, XS, eX, REF_S, REF_DMAX, Gm, nullptr, 0, ain, errf, gsm, stream);  // G = X^T X
      RefP rp{};
      rp.n = n;
      rp.S = Sm;
      rp.G = Gm;
      rp.E = PE;
      rp.lam = static_cast<double *>(P(ly.lam));
      rp.order = static_cast<int *>(P(ly.ord));
      rp.cl = static_cast<int *>(P(ly.cl));
      rp.W = static_cast<double *>(P(ly.W));
      rp.act_in = ain;
      rp.act_out = aout;
      rp.conv_it = conv;
      rp.fail = fail;
      rp.emax = static_cast<double *>(P(ly.emax));
      rp.tol = ro.tol;
      rp.it = it;
      rp.last = it == ro.max_iter;
      k_oa_update<<<(unsigned)lc, 256, usm, stream>>>(rp);
      ref_slice(ly, lc, Xs, xf32, 1, n, REF_SX, XR, eXR, ain, stream);           // rows of X
      ref_slice(ly, lc, PE, 0, n, 1, REF_SE, ES, eE, ain, stream);               // columns of E
      ref_gemm(ly, lc, XR, eXR, REF_SX, ES, eE, REF_SE, REF_DMAX_XE, Xd, Xs, xf32, ain, errf, gsm, stream);
      k_cluster_apply<<<(unsigned)lc, 256, 0, stream>>>(n, Xd, ain, fail, rp.order, rp.cl, rp.W, errf);
      if ((err = cudaGetLastError()) != cudaSuccess) return err;
    }
    k_ref_final<<<(unsigned)lc, 256, fsm, stream>>>(n, nm, a, w, info, XB[0], XB[1],
                                                     static_cast<double *>(P(ly.lam)),
                                                     static_cast<double *>(P(ly.sig)), conv, fail, iters, fb_list,
                                                     cnt, c0);
    if ((err = cudaGetLastError()) != cudaSuccess) return err;
  }
  // the fallback: its size is read back (one synchronisation of the stream)
  int hc[2] = {0, 0};
  if ((err = cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, stream)) != cudaSuccess) return err;
  if ((err = cudaStreamSynchronize(stream)) != cudaSuccess) return err;
  if (hc[1] != 0) return cudaErrorLaunchFailure;  // a product's wait gave up
  if (hc[0] > 0) {
    if (!ro.fallback) {
      k_ref_mark<<<(unsigned)((hc[0] + 255) / 256), 256, 0, stream>>>(hc[0], fb_list, info);
      return cudaGetLastError();
    }
    long long *aoff = static_cast<long long *>(P(ly.aoff)), *woff = static_cast<long long *>(P(ly.woff));
    k_ref_offsets<<<(unsigned)std::min<long>((L + 255) / 256, 4096), 256, 0, stream>>>(L, nm, n, aoff, woff);
    eigen_GPU_batch_opts o64{};  // the reference defaults: tql2, sorted, 100 sweeps
    o64.method = EIGEN_GPU_BATCH_TQL2;
    o64.sort = 1;
    o64.max_sweep = 100;
    o64.chunk = (int)ly.Lc;
    Indirect ix;
    ix.kid = fb_list;
    ix.aoff = aoff;
    ix.woff = woff;
    if ((err = run<double>(hc[0], nm, n, n, a, w, wk, ly.chunk_bytes, info, &o64, stream, nullptr, ix)) !=
        cudaSuccess)
      return err;
  }
  return cudaSuccess;
}

// ---- Rayleigh products S = X^T A X, G = X^T X on the int8 tensor cores ----
struct RayLayout {
  long Lc = 0;
  size_t af = 0, p = 0, as = 0, xs = 0, ps = 0, ea = 0, ex = 0, ep = 0, err = 0, bytes = 0;
};

inline void ray_layout(long Lc, int n, RayLayout &ly)
{
  const size_t nn = (size_t)n * n, sl = oz_slice_bytes(n), rp = (size_t)oz_rp(n);
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o = align256(o + bytes);
    return at;
  };
  ly.Lc = Lc;
  ly.af = take(sizeof(double) * nn * Lc);
  ly.p = take(sizeof(double) * nn * Lc);
  ly.as = take(sl * REF_S * Lc);
  ly.xs = take(sl * REF_S * Lc);
  ly.ps = take(sl * REF_S * Lc);
  ly.ea = take(sizeof(int) * rp * Lc);
  ly.ex = take(sizeof(int) * rp * Lc);
  ly.ep = take(sizeof(int) * rp * Lc);
  ly.err = take(sizeof(int));
  ly.bytes = o;
}

inline cudaError_t ray_plan(long L, int n, RayLayout &ly)
{
  long Lc = L;
  ray_layout(Lc, n, ly);
  if (ly.bytes > kWsBudget) {
    const size_t per = ly.bytes / (size_t)L + 1;
    Lc = std::max<long>(1, (long)(kWsBudget / per));
    ray_layout(Lc, n, ly);
  }
  return cudaSuccess;
}

cudaError_t ray_buffer_size(long L, int nm, int n, size_t *lwork)
{
  if (lwork == nullptr) return cudaErrorInvalidValue;
  *lwork = 0;
  if (ref_bad_args(L, nm, n)) return cudaErrorInvalidValue;
  RayLayout ly;
  ray_plan(L, n, ly);
  *lwork = ly.bytes;
  return cudaSuccess;
}

cudaError_t run_rayleigh(long L, int nm, int n, const double *a, const double *x, double *s, double *g, void *wk,
                         size_t lwork, cudaStream_t stream)
{
  if (ref_bad_args(L, nm, n) || a == nullptr || x == nullptr || (s == nullptr && g == nullptr))
    return cudaErrorInvalidValue;
  DevProps dp;
  cudaError_t err = dev_props(dp);
  if (err != cudaSuccess) return err;
  RayLayout ly;
  ray_plan(L, n, ly);
  if (wk == nullptr || (lwork != 0 && lwork < ly.bytes)) return cudaErrorInvalidValue;
  char *base = static_cast<char *>(wk);
  auto P = [&](size_t off) { return static_cast<void *>(base + off); };
  RefLayout rl;  // the slice geometry
  rl.n = n;
  rl.Rp = oz_rp(n);
  rl.Kp = oz_kp(n);
  rl.KB = oz_kb(n);
  const size_t need = oz_gemm_smem(REF_S, REF_S, rl.KB, REF_DMAX);
  const size_t gsm = std::min<size_t>(oz_launch_smem(need, 2, dp.smem_sm, dp.smem_rsv), (size_t)dp.smem_optin);
  if (need > (size_t)dp.smem_optin) return cudaErrorInvalidValue;
  if ((err = set_smem(k_oz_gemm, gsm)) != cudaSuccess) return err;
  double *Af = static_cast<double *>(P(ly.af)), *Pm = static_cast<double *>(P(ly.p));
  int8_t *AS = static_cast<int8_t *>(P(ly.as)), *XS = static_cast<int8_t *>(P(ly.xs)),
         *PS = static_cast<int8_t *>(P(ly.ps));
  int *eA = static_cast<int *>(P(ly.ea)), *eX = static_cast<int *>(P(ly.ex)), *eP = static_cast<int *>(P(ly.ep));
  int *errf = static_cast<int *>(P(ly.err));
  if ((err = cudaMemsetAsync(errf, 0, sizeof(int), stream)) != cudaSuccess) return err;
  for (long c0 = 0; c0 < L; c0 += ly.Lc) {
    const long lc = std::min(ly.Lc, L - c0);
    k_ref_prep<<<(unsigned)lc, 256, 0, stream>>>(a + (size_t)c0 * nm * n, nm, n, Af, nullptr, nullptr, 0);
    ref_slice(rl, lc, Af, 0, n, 1, REF_S, AS, eA, nullptr, stream);
    // columns of X (leading dimension nm)
    {
      OzSlice q{};
      q.src = x + (size_t)c0 * nm * n;
      q.src_f32 = 0;
      q.bs = (long long)nm * n;
      q.rs = nm;
      q.ks = 1;
      q.R = n;
      q.K = n;
      q.Rp = rl.Rp;
      q.Kp = rl.Kp;
      q.KB = rl.KB;
      q.s = REF_S;
      q.out = XS;
      q.e = eX;
      const int rpb = 256 / (rl.Kp / 16);
      k_oz_slice<><<<dim3((unsigned)lc, (unsigned)((rl.Rp + rpb - 1) / rpb)), 256, 0, stream>>>(q);
    }
    if (s) {
      ref_gemm(rl, lc, AS, eA, REF_S, XS, eX, REF_S, REF_DMAX, Pm, nullptr, 0, nullptr, errf, gsm, stream);
      ref_slice(rl, lc, Pm, 0, n, 1, REF_S, PS, eP, nullptr, stream);
      ref_gemm(rl, lc, XS, eX, REF_S, PS, eP, REF_S, REF_DMAX, s + (size_t)c0 * n * n, nullptr, 0, nullptr, errf,
               gsm, stream);
    }
    if (g)
      ref_gemm(rl, lc, XS, eX, REF_S, XS, eX, REF_S, REF_DMAX, g + (size_t)c0 * n * n, nullptr, 0, nullptr, errf,
               gsm, stream);
    if ((err = cudaGetLastError()) != cudaSuccess) return err;
  }
  return cudaSuccess;
}

// ---- the learned warm start's network (eigb_mlp.cuh) ----
//
// Parameters of the MLP d0 -> d1 -> d2 -> d3 (tanh, tanh, linear), d0 a
// multiple of 8: FP32 flat [W1 b1 W2 b2 W3 b3] (W_l row-major, out x in),
// its Adam moments m and v, then the BF16 copies W1, W2, W2^T, W3, W3^T.
struct MlpLayout {
  int d0, d1, d2, d3;
  size_t w1, b1, w2, b2, w3, b3, P;  // element offsets in the flat FP32 block, and its size
  size_t m, v, w1b, w2b, w2t, w3b, w3t, bytes;  // byte offsets
};

inline bool mlp_bad(int d0, int d1, int d2, int d3)
{
  return d0 < 8 || d1 < 8 || d2 < 8 || d3 < 8 || (d0 % 8) || (d1 % 8) || (d2 % 8) || (d3 % 8) || d1 > 4096 ||
         d2 > 4096 || d3 > 65536;
}

inline MlpLayout mlp_layout(int d0, int d1, int d2, int d3)
{
  MlpLayout l{};
  l.d0 = d0;
  l.d1 = d1;
  l.d2 = d2;
  l.d3 = d3;
  size_t e = 0;
  l.w1 = e;
  e += (size_t)d1 * d0;
  l.b1 = e;
  e += d1;
  l.w2 = e;
  e += (size_t)d2 * d1;
  l.b2 = e;
  e += d2;
  l.w3 = e;
  e += (size_t)d3 * d2;
  l.b3 = e;
  e += d3;
  l.P = e;
  size_t o = align256(sizeof(float) * e);
  l.m = o;
  o = align256(o + sizeof(float) * e);
  l.v = o;
  o = align256(o + sizeof(float) * e);
  l.w1b = o;
  o = align256(o + 2 * (size_t)d1 * d0);
  l.w2b = o;
  o = align256(o + 2 * (size_t)d2 * d1);
  l.w2t = o;
  o = align256(o + 2 * (size_t)d2 * d1);
  l.w3b = o;
  o = align256(o + 2 * (size_t)d3 * d2);
  l.w3t = o;
  o = align256(o + 2 * (size_t)d3 * d2);
  l.bytes = o;
  return l;
}

// workspace of a forward (train = 0) or training pass over `rows` rows
struct MlpWs {
  size_t xb, xt, h1, h1b, h1t, h2, h2b, h2t, y, yb, dyb, dy32, dyt, dh2, dz2b, dz2, dz2t, dh1, dz1b, dz1, dz1t, grad,
      sse, err, bytes;
};

inline MlpWs mlp_ws(const MlpLayout &l, int rows, bool train)
{
  MlpWs w{};
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o = align256(o + bytes);
    return at;
  };
  const size_t R = (size_t)rows;
  w.xb = take(2 * R * l.d0);
  w.h1b = take(2 * R * l.d1);
  w.h2b = take(2 * R * l.d2);
  w.yb = take(2 * R * l.d3);
  w.err = take(sizeof(int));
  if (train) {
    w.y = take(4 * R * l.d3);
    w.xt = take(2 * R * l.d0);
    w.h1 = take(4 * R * l.d1);
    w.h1t = take(2 * R * l.d1);
    w.h2 = take(4 * R * l.d2);
    w.h2t = take(2 * R * l.d2);
    w.dyb = take(2 * R * l.d3);
    w.dy32 = take(4 * R * l.d3);
    w.dyt = take(2 * R * l.d3);
    w.dh2 = take(4 * R * l.d2);
    w.dz2b = take(2 * R * l.d2);
    w.dz2 = take(4 * R * l.d2);
    w.dz2t = take(2 * R * l.d2);
    w.dh1 = take(4 * R * l.d1);
    w.dz1b = take(2 * R * l.d1);
    w.dz1 = take(4 * R * l.d1);
    w.dz1t = take(2 * R * l.d1);
    w.grad = take(sizeof(float) * l.P);
    w.sse = take(sizeof(double));
  }
  w.bytes = o;
  return w;
}

inline cudaError_t mm_launch(const bf16 *A, int lda, const bf16 *B, int ldb, int M, int N, int K, float *C, int ldc,
                             bf16 *Cb, int ldcb, const float *bias, int act, float alpha, int *err, cudaStream_t st)
{
  if (M < 1 || N < 1 || K < 8 || (K % 8) || (lda % 8) || (ldb % 8)) return cudaErrorInvalidValue;
  MmP p{};
  p.A = A;
  p.lda = lda;
  p.B = B;
  p.ldb = ldb;
  p.M = M;
  p.N = N;
  p.K = K;
  p.C = C;
  p.ldc = ldc;
  p.Cb = Cb;
  p.ldcb = ldcb;
  p.bias = bias;
  p.act = act;
  p.alpha = alpha;
  p.err = err;
  dim3 grid((unsigned)((N + MM_T - 1) / MM_T), (unsigned)((M + MM_T - 1) / MM_T), 1);
  k_mm_bf16<<<grid, MM_THREADS, mm_smem(), st>>>(p);
  return cudaGetLastError();
}

inline cudaError_t mm_setup()
{
  return cudaFuncSetAttribute(k_mm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mm_smem());
}

inline unsigned grid1(long count) { return (unsigned)std::max<long>(1, std::min<long>((count + 255) / 256, 8192)); }

inline void transpose_bf16(const bf16 *in, int rows, int cols, bf16 *out, cudaStream_t st)
{
  dim3 g((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
  k_t_bf16<<<g, 256, 0, st>>>(rows, cols, in, cols, out, rows);
}

// forward over rows (x: rows x d0 FP32, row-major); output Y (FP32) and its
// BF16 copy in the workspace; y (optional) receives the FP32 output
cudaError_t mlp_forward(const MlpLayout &l, const void *params, int rows, const float *x, float *y, char *ws,
                        const MlpWs &w, bool keep32, cudaStream_t st)
{
  const float *P = static_cast<const float *>(params);
  const char *pb = static_cast<const char *>(params);
  cudaError_t err;
  if ((err = mm_setup()) != cudaSuccess) return err;
  bf16 *xb = reinterpret_cast<bf16 *>(ws + w.xb);
  k_to_bf16<<<grid1((long)rows * l.d0), 256, 0, st>>>(rows, l.d0, x, l.d0, xb, l.d0);
  int *ef = reinterpret_cast<int *>(ws + w.err);
  bf16 *h1b = reinterpret_cast<bf16 *>(ws + w.h1b), *h2b = reinterpret_cast<bf16 *>(ws + w.h2b);
  float *h1 = keep32 ? reinterpret_cast<float *>(ws + w.h1) : nullptr;
  float *h2 = keep32 ? reinterpret_cast<float *>(ws + w.h2) : nullptr;
  if ((err = mm_launch(xb, l.d0, reinterpret_cast<const bf16 *>(pb + l.w1b), l.d0, rows, l.d1, l.d0, h1, l.d1, h1b,
                       l.d1, P + l.b1, 1, 1.0f, ef, st)) != cudaSuccess)
    return err;
  if ((err = mm_launch(h1b, l.d1, reinterpret_cast<const bf16 *>(pb + l.w2b), l.d1, rows, l.d2, l.d1, h2, l.d2, h2b,
                       l.d2, P + l.b2, 1, 1.0f, ef, st)) != cudaSuccess)
    return err;
  float *yo = y ? y : (keep32 ? reinterpret_cast<float *>(ws + w.y) : nullptr);
  return mm_launch(h2b, l.d2, reinterpret_cast<const bf16 *>(pb + l.w3b), l.d2, rows, l.d3, l.d2, yo, l.d3,
                   reinterpret_cast<bf16 *>(ws + w.yb), l.d3, P + l.b3, 0, 1.0f, ef, st);
}

// gradient of the mean squared error over rows x d3 outputs into grad (the
// flat FP32 layout); sse (device, optional) += sum of squared errors
cudaError_t mlp_backward(const MlpLayout &l, const void *params, int rows, const float *t, float *grad, double *sse,
                         char *ws, const MlpWs &w, cudaStream_t st)
{
  const char *pb = static_cast<const char *>(params);
  cudaError_t err;
  int *ef = reinterpret_cast<int *>(ws + w.err);
  auto F = [&](size_t off) { return reinterpret_cast<float *>(ws + off); };
  auto H = [&](size_t off) { return reinterpret_cast<bf16 *>(ws + off); };
  const long ny = (long)rows * l.d3;
  k_mse_grad<<<grid1(ny), 256, 0, st>>>(ny, F(w.y), t, H(w.dyb), F(w.dy32), sse ? sse : reinterpret_cast<double *>(ws + w.sse));
  // layer 3: dW3 = dY^T H2, db3 = colsum dY, dH2 = dY W3
  transpose_bf16(H(w.dyb), rows, l.d3, H(w.dyt), st);
  transpose_bf16(H(w.h2b), rows, l.d2, H(w.h2t), st);
  if ((err = mm_launch(H(w.dyt), rows, H(w.h2t), rows, l.d3, l.d2, rows, grad + l.w3, l.d2, nullptr, 0, nullptr, 0,
                       1.0f, ef, st)) != cudaSuccess)
    return err;
  k_colsum<<<(l.d3 + 255) / 256, 256, 0, st>>>(rows, l.d3, F(w.dy32), grad + l.b3);
  if ((err = mm_launch(H(w.dyb), l.d3, reinterpret_cast<const bf16 *>(pb + l.w3t), l.d3, rows, l.d2, l.d3, F(w.dh2),
                       l.d2, nullptr, 0, nullptr, 0, 1.0f, ef, st)) != cudaSuccess)
    return err;
  // layer 2
  k_tanh_bwd<<<grid1((long)rows * l.d2), 256, 0, st>>>((long)rows * l.d2, F(w.dh2), F(w.h2), H(w.dz2b), F(w.dz2));
  transpose_bf16(H(w.dz2b), rows, l.d2, H(w.dz2t), st);
  transpose_bf16(H(w.h1b), rows, l.d1, H(w.h1t), st);
  if ((err = mm_launch(H(w.dz2t), rows, H(w.h1t), rows, l.d2, l.d1, rows, grad + l.w2, l.d1, nullptr, 0, nullptr, 0,
                       1.0f, ef, st)) != cudaSuccess)
    return err;
  k_colsum<<<(l.d2 + 255) / 256, 256, 0, st>>>(rows, l.d2, F(w.dz2), grad + l.b2);
  if ((err = mm_launch(H(w.dz2b), l.d2, reinterpret_cast<const bf16 *>(pb + l.w2t), l.d2, rows, l.d1, l.d2, F(w.dh1),
                       l.d1, nullptr, 0, nullptr, 0, 1.0f, ef, st)) != cudaSuccess)
    return err;
  // layer 1
  k_tanh_bwd<<<grid1((long)rows * l.d1), 256, 0, st>>>((long)rows * l.d1, F(w.dh1), F(w.h1), H(w.dz1b), F(w.dz1));
  transpose_bf16(H(w.dz1b), rows, l.d1, H(w.dz1t), st);
  transpose_bf16(H(w.xb), rows, l.d0, H(w.xt), st);
  if ((err = mm_launch(H(w.dz1t), rows, H(w.xt), rows, l.d1, l.d0, rows, grad + l.w1, l.d0, nullptr, 0, nullptr, 0,
                       1.0f, ef, st)) != cudaSuccess)
    return err;
  k_colsum<<<(l.d1 + 255) / 256, 256, 0, st>>>(rows, l.d1, F(w.dz1), grad + l.b1);
  return cudaGetLastError();
}

// BF16 copies (and transposes) of the FP32 weights
inline void mlp_sync_bf16(const MlpLayout &l, void *params, cudaStream_t st)
{
  float *P = static_cast<float *>(params);
  char *pb = static_cast<char *>(params);
  k_to_bf16<<<grid1((long)l.d1 * l.d0), 256, 0, st>>>(l.d1, l.d0, P + l.w1, l.d0, reinterpret_cast<bf16 *>(pb + l.w1b),
                                                     l.d0);
  k_to_bf16<<<grid1((long)l.d2 * l.d1), 256, 0, st>>>(l.d2, l.d1, P + l.w2, l.d1, reinterpret_cast<bf16 *>(pb + l.w2b),
                                                     l.d1);
  transpose_bf16(reinterpret_cast<bf16 *>(pb + l.w2b), l.d2, l.d1, reinterpret_cast<bf16 *>(pb + l.w2t), st);
  k_to_bf16<<<grid1((long)l.d3 * l.d2), 256, 0, st>>>(l.d3, l.d2, P + l.w3, l.d2, reinterpret_cast<bf16 *>(pb + l.w3b),
                                                     l.d2);
  transpose_bf16(reinterpret_cast<bf16 *>(pb + l.w3b), l.d3, l.d2, reinterpret_cast<bf16 *>(pb + l.w3t), st);
}

cudaError_t mlp_init(const MlpLayout &l, void *params, unsigned long long seed, cudaStream_t st)
{
  float *P = static_cast<float *>(params);
  char *pb = static_cast<char *>(params);
  cudaError_t err;
  if ((err = cudaMemsetAsync(params, 0, l.bytes, st)) != cudaSuccess) return err;
  // uniform +-sqrt(6 / (fan_in + fan_out)) weights, zero biases
  k_init_uniform<<<grid1((long)l.d1 * l.d0), 256, 0, st>>>((long)l.d1 * l.d0, P + l.w1,
                                                           sqrtf(6.0f / (l.d0 + l.d1)), seed);
  k_init_uniform<<<grid1((long)l.d2 * l.d1), 256, 0, st>>>((long)l.d2 * l.d1, P + l.w2,
                                                           sqrtf(6.0f / (l.d1 + l.d2)), seed + 1);
  k_init_uniform<<<grid1((long)l.d3 * l.d2), 256, 0, st>>>((long)l.d3 * l.d2, P + l.w3,
                                                           sqrtf(6.0f / (l.d2 + l.d3)), seed + 2);
  (void)pb;
  mlp_sync_bf16(l, params, st);
  return cudaGetLastError();
}

cudaError_t mlp_adam(const MlpLayout &l, void *params, const float *grad, float lr, int step, cudaStream_t st)
{
  float *P = static_cast<float *>(params);
  char *pb = static_cast<char *>(params);
  float *m = reinterpret_cast<float *>(pb + l.m), *v = reinterpret_cast<float *>(pb + l.v);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.0f / (1.0f - powf(b1, (float)step)), c2 = 1.0f / (1.0f - powf(b2, (float)step));
  k_adam<<<grid1((long)l.P), 256, 0, st>>>(1, (int)l.P, P, grad, m, v, nullptr, nullptr, lr, b1, b2, eps, c1, c2);
  mlp_sync_bf16(l, params, st);
  return cudaGetLastError();
}

// ---- learned warm start solve (eigb_learned.cuh) ----
struct LwLayout {
  long Lc = 0;
  size_t af, x0, pm, sm, gm, ym, xm, axm, mu, sw, as, x0s, ps, x0r, ys, xs, ea, ex0, ep, ex0r, ey, ex, feat, ginv,
      v0r, mws, cnt, fb, aoff, woff, bytes, chunk_bytes;
  MlpWs mw;
};
constexpr int LW_S = 4, LW_DMAX = 5;  // FP32-level products: 4 slices, diagonals up to 5

inline size_t lw_chunk_layout(long Lc, int nm, int n, const MlpLayout &ml, const DevProps &dp, LwLayout &ly)
{
  const size_t nn = (size_t)n * n, sl = oz_slice_bytes(n), rp = (size_t)oz_rp(n);
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o = align256(o + bytes);
    return at;
  };
  ly.Lc = Lc;
  ly.af = take(8 * nn * Lc);
  ly.x0 = take(4 * nn * Lc);
  ly.pm = take(8 * nn * Lc);
  ly.sm = take(8 * nn * Lc);
  ly.gm = take(8 * nn * Lc);
  ly.ym = take(8 * nn * Lc);
  ly.xm = take(8 * nn * Lc);
  ly.axm = ly.pm;  // P is dead once S is formed
  ly.mu = take(8 * (size_t)n * Lc);
  ly.sw = take(4 * (size_t)Lc);
  ly.as = take(sl * LW_S * Lc);
  ly.x0s = take(sl * LW_S * Lc);
  ly.ps = take(sl * LW_S * Lc);
  ly.x0r = ly.ps;  // P's slices are dead once S is formed
  ly.ys = take(sl * LW_S * Lc);
  ly.xs = ly.x0s;  // X0's column slices are dead once G is formed
  ly.ea = take(4 * rp * Lc);
  ly.ex0 = take(4 * rp * Lc);
  ly.ep = take(4 * rp * Lc);
  ly.ex0r = ly.ep;
  ly.ey = take(4 * rp * Lc);
  ly.ex = ly.ex0;
  ly.feat = take(4 * (size_t)LW_D0 * Lc);
  ly.ginv = take(8 * 16);
  ly.v0r = take(2 * nn);
  ly.mw = mlp_ws(ml, (int)Lc, false);
  ly.mws = take(ly.mw.bytes);
  Plan<float> pf;
  eigen_GPU_batch_opts o32{};
  o32.method = EIGEN_GPU_BATCH_TQL2;
  o32.sort = 1;
  o32.max_sweep = 100;
  o32.chunk = (int)Lc;
  if (make_plan<float>(Lc, nm, n, dp, pf, &o32) != cudaSuccess) return 0;
  return std::max(o, pf.bytes);
}

inline cudaError_t lw_plan(long L, int nm, int n, const MlpLayout &ml, const DevProps &dp, int chunk, LwLayout &ly)
{
  long Lc = chunk > 0 ? std::min<long>(L, chunk) : L;
  size_t cb = 0;
  for (;;) {
    cb = lw_chunk_layout(Lc, nm, n, ml, dp, ly);
    if (cb == 0) return cudaErrorInvalidValue;
    if (chunk > 0 || cb <= kWsBudget || Lc <= 256) break;
    Lc = std::max<long>(256, (long)((double)Lc * (double)kWsBudget / (double)cb * 0.98));
    const long nch = (L + Lc - 1) / Lc;
    Lc = (L + nch - 1) / nch;
  }
  ly.chunk_bytes = align256(cb);
  size_t o = ly.chunk_bytes;
  ly.fb = o;
  o = align256(o + sizeof(int) * L);
  ly.aoff = o;
  o = align256(o + sizeof(long long) * L);
  ly.woff = o;
  o = align256(o + sizeof(long long) * L);
  ly.cnt = o;
  o = align256(o + 2 * sizeof(int));
  ly.bytes = o;
  return cudaSuccess;
}

struct LwOpts {
  int warm = EIGEN_GPU_WARM_NETWORK;
  int max_sweeps = 10;
  double tol = 1e-6;
  double jacobi_tol = 1e-7;
  int fallback = 1;
  int chunk = 0;
};

inline LwOpts lw_opts(const eigen_GPU_learned_opts *o)
{
  LwOpts r;
  if (o) {
    r.warm = o->warm;
    if (o->max_sweeps > 0) r.max_sweeps = o->max_sweeps;
    if (o->tol > 0) r.tol = o->tol;
    if (o->jacobi_tol > 0) r.jacobi_tol = o->jacobi_tol;
    r.fallback = o->fallback ? 1 : 0;
    r.chunk = o->chunk;
  }
  return r;
}

inline bool lw_bad(long L, int nm, int n, int d1, int d2)
{
  return L < 1 || n < 8 || n > LW_NMAX || (n % 8) || nm < n || mlp_bad(LW_D0, d1, d2, n * n);
}

cudaError_t lw_buffer_size(long L, int nm, int n, int d1, int d2, const eigen_GPU_learned_opts *opts, size_t *lwork)
{
  if (!lwork) return cudaErrorInvalidValue;
  *lwork = 0;
  if (lw_bad(L, nm, n, d1, d2)) return cudaErrorInvalidValue;
  DevProps dp;
  cudaError_t err = dev_props(dp);
  if (err != cudaSuccess) return err;
  LwLayout ly;
  if ((err = lw_plan(L, nm, n, mlp_layout(LW_D0, d1, d2, n * n), dp, lw_opts(opts).chunk, ly)) != cudaSuccess)
    return err;
  *lwork = ly.bytes;
  return cudaSuccess;
}

cudaError_t run_learned(long L, int nm, int n, float *a, float *w, const float *fam, const void *params, int d1, int d2,
                        void *wk, size_t lwork, int *info, int *sweeps, double *resid,
                        const eigen_GPU_learned_opts *opts, cudaStream_t stream)
{
  if (lw_bad(L, nm, n, d1, d2) || !a || !w || !fam) return cudaErrorInvalidValue;
  const LwOpts lo = lw_opts(opts);
  if (lo.warm < EIGEN_GPU_WARM_NETWORK || lo.warm > EIGEN_GPU_WARM_IDENTITY) return cudaErrorInvalidValue;
  if (lo.warm == EIGEN_GPU_WARM_NETWORK && !params) return cudaErrorInvalidValue;
  DevProps dp;
  cudaError_t err = dev_props(dp);
  if (err != cudaSuccess) return err;
  const MlpLayout ml = mlp_layout(LW_D0, d1, d2, n * n);
  LwLayout ly;
  if ((err = lw_plan(L, nm, n, ml, dp, lo.chunk, ly)) != cudaSuccess) return err;
  if (!wk || (lwork != 0 && lwork < ly.bytes)) return cudaErrorInvalidValue;
  char *base = static_cast<char *>(wk);
  auto P = [&](size_t off) { return static_cast<void *>(base + off); };
  auto D = [&](size_t off) { return static_cast<double *>(P(off)); };
  auto I8 = [&](size_t off) { return static_cast<int8_t *>(P(off)); };
  auto IN = [&](size_t off) { return static_cast<int *>(P(off)); };
  int *fb_list = IN(ly.fb), *cnt = IN(ly.cnt), *errf = cnt + 1;
  if ((err = cudaMemsetAsync(cnt, 0, 2 * sizeof(int), stream)) != cudaSuccess) return err;
  RefLayout rl;
  rl.n = n;
  rl.Rp = oz_rp(n);
  rl.Kp = oz_kp(n);
  rl.KB = oz_kb(n);
  const size_t need = oz_gemm_smem(LW_S, LW_S, rl.KB, LW_DMAX);
  const size_t gsm = std::min<size_t>(oz_launch_smem(need, oz_geom(LW_S, LW_S, LW_DMAX).groups, dp.smem_sm,
                                                     dp.smem_rsv), (size_t)dp.smem_optin);
  if ((err = set_smem(k_oz_gemm, gsm)) != cudaSuccess) return err;
  const size_t psm = lw_polish_smem(n);
  if ((err = set_smem(k_lw_polish, psm)) != cudaSuccess) return err;
  const size_t nn = (size_t)n * n;
  const float *v0 = fam + 5 * nn;
  double *ginv = D(ly.ginv);
  k_lw_gram<<<1, 256, 0, stream>>>(n, fam, ginv);
  bf16 *v0r = static_cast<bf16 *>(P(ly.v0r));
  k_lw_v0rows<<<grid1((long)nn), 256, 0, stream>>>(n, v0, v0r);
  float *X0 = static_cast<float *>(P(ly.x0));
  char *mws = static_cast<char *>(P(ly.mws));
  for (long c0 = 0; c0 < L; c0 += ly.Lc) {
    const long lc = std::min(ly.Lc, L - c0);
    k_lw_prep<<<(unsigned)lc, 256, 0, stream>>>(a + (size_t)c0 * nm * n, nm, n, D(ly.af));
    if (lo.warm == EIGEN_GPU_WARM_NETWORK) {
      float *feat = static_cast<float *>(P(ly.feat));
      k_lw_features<<<(unsigned)lc, 256, 0, stream>>>(n, D(ly.af), fam, ginv, feat);
      if ((err = mlp_forward(ml, params, (int)lc, feat, nullptr, mws, ly.mw, false, stream)) != cudaSuccess) return err;
      // X0 = V0 C: rows (matrix, column j) of the output, K index k
      if ((err = mm_launch(reinterpret_cast<const bf16 *>(mws + ly.mw.yb), n, v0r, n, (int)(lc * n), n, n, X0, n,
                           nullptr, 0, nullptr, 0, 1.0f, errf, stream)) != cudaSuccess)
        return err;
    } else {
      k_lw_fill<<<grid1(lc * (long)nn), 256, 0, stream>>>(lc, n, lo.warm, v0, X0);
    }
    // S = X0^T A X0, G = X0^T X0
    ref_slice(rl, lc, D(ly.af), 0, n, 1, LW_S, I8(ly.as), IN(ly.ea), nullptr, stream);
    ref_slice(rl, lc, X0, 1, n, 1, LW_S, I8(ly.x0s), IN(ly.ex0), nullptr, stream);
    ref_gemm(rl, lc, I8(ly.as), IN(ly.ea), LW_S, I8(ly.x0s), IN(ly.ex0), LW_S, LW_DMAX, D(ly.pm), nullptr, 0, nullptr,
             errf, gsm, stream);
    ref_slice(rl, lc, D(ly.pm), 0, n, 1, LW_S, I8(ly.ps), IN(ly.ep), nullptr, stream);
    ref_gemm(rl, lc, I8(ly.x0s), IN(ly.ex0), LW_S, I8(ly.ps), IN(ly.ep), LW_S, LW_DMAX, D(ly.sm), nullptr, 0, nullptr,
             errf, gsm, stream);
    ref_gemm(rl, lc, I8(ly.x0s), IN(ly.ex0), LW_S, I8(ly.x0s), IN(ly.ex0), LW_S, LW_DMAX, D(ly.gm), nullptr, 0,
             nullptr, errf, gsm, stream);
    k_lw_polish<<<(unsigned)lc, 256, psm, stream>>>(n, D(ly.sm), D(ly.gm), D(ly.ym), D(ly.mu), IN(ly.sw),
                                                    lo.max_sweeps, lo.jacobi_tol);
    // X = X0 Y, then A X for the gate
    ref_slice(rl, lc, X0, 1, 1, n, LW_S, I8(ly.x0r), IN(ly.ex0r), nullptr, stream);
    ref_slice(rl, lc, D(ly.ym), 0, n, 1, LW_S, I8(ly.ys), IN(ly.ey), nullptr, stream);
    ref_gemm(rl, lc, I8(ly.x0r), IN(ly.ex0r), LW_S, I8(ly.ys), IN(ly.ey), LW_S, LW_DMAX, D(ly.xm), nullptr, 0, nullptr,
             errf, gsm, stream);
    ref_slice(rl, lc, D(ly.xm), 0, n, 1, LW_S, I8(ly.xs), IN(ly.ex), nullptr, stream);
    ref_gemm(rl, lc, I8(ly.as), IN(ly.ea), LW_S, I8(ly.xs), IN(ly.ex), LW_S, LW_DMAX, D(ly.axm), nullptr, 0, nullptr,
             errf, gsm, stream);
    k_lw_gate<<<(unsigned)lc, 256, 0, stream>>>(n, nm, D(ly.axm), D(ly.xm), D(ly.mu), IN(ly.sw), lo.tol, a, w, info,
                                                sweeps, resid, fb_list, cnt, c0);
    if ((err = cudaGetLastError()) != cudaSuccess) return err;
  }
  int hc[2] = {0, 0};
  if ((err = cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, stream)) != cudaSuccess) return err;
  if ((err = cudaStreamSynchronize(stream)) != cudaSuccess) return err;
  if (hc[1] != 0) return cudaErrorLaunchFailure;
  if (hc[0] > 0) {
    if (!lo.fallback) {
      k_ref_mark<<<(unsigned)((hc[0] + 255) / 256), 256, 0, stream>>>(hc[0], fb_list, info);
      return cudaGetLastError();
    }
    long long *aoff = static_cast<long long *>(P(ly.aoff)), *woff = static_cast<long long *>(P(ly.woff));
    k_ref_offsets<<<grid1(L), 256, 0, stream>>>(L, nm, n, aoff, woff);
    eigen_GPU_batch_opts o32{};
    o32.method = EIGEN_GPU_BATCH_TQL2;
    o32.sort = 1;
    o32.max_sweep = 100;
    o32.chunk = (int)ly.Lc;
    Indirect ix;
    ix.kid = fb_list;
    ix.aoff = aoff;
    ix.woff = woff;
    if ((err = run<float>(hc[0], nm, n, n, a, w, wk, ly.chunk_bytes, info, &o32, stream, nullptr, ix)) != cudaSuccess)
      return err;
  }
  return cudaSuccess;
}

static_assert(EIGEN_GPU_FUNC_DIAG == SYMF_DIAG && EIGEN_GPU_FUNC_POW == SYMF_POW && EIGEN_GPU_FUNC_EXP == SYMF_EXP,
              "matrix-function codes of the header and the kernel agree");

template <class T>
cudaError_t symfunc_run(long L, int nm, int n, const T *v, const T *w, T *z, int func, double p, cudaStream_t stream)
{
  if (L < 1 || n < 1 || nm < n || n > 1024 || v == nullptr || w == nullptr || z == nullptr)
    return cudaErrorInvalidValue;
  if (func < SYMF_DIAG || func > SYMF_EXP) return cudaErrorInvalidValue;
  if (v == z) return cudaErrorInvalidValue;  // Z is written while V is still read
  const int nt = (n + SF_TILE - 1) / SF_TILE;
  const int ntiles = nt * (nt + 1) / 2;
  const long blocks = L * ntiles;
  if (blocks > 0x7fffffffL) return cudaErrorInvalidValue;
  k_symfunc<T><<<(unsigned)blocks, 256, 0, stream>>>(L, nm, n, v, w, z, func, (T)p, ntiles);
  return cudaGetLastError();
}

// the tensor-core gate, 32-deep panels from n = 128 on (16 below, where a
// 32-deep panel would be mostly padding); one persistent CTA per SM
template <class T, bool PACKED>
cudaError_t launch_check_tc(long L, int lda, int ldz, int n, int m, const T *a, const T *w, const T *z, double *err1,
                            double *err2, int *flags, float *ref_flags, cudaStream_t stream)
{
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const unsigned grid = (unsigned)std::min<long>(L, std::max(sms, 1));
  if (n >= 128) {
    const size_t smb = checkm_smem<T, 32>();
    if ((e = set_smem(k_check_tc<T, PACKED, 32>, smb)) != cudaSuccess) return e;
    k_check_tc<T, PACKED, 32><<<grid, 512, smb, stream>>>(L, lda, ldz, n, m, a, w, z, err1, err2, flags, ref_flags);
  } else {
    const size_t smb = checkm_smem<T, 16>();
    if ((e = set_smem(k_check_tc<T, PACKED, 16>, smb)) != cudaSuccess) return e;
    k_check_tc<T, PACKED, 16><<<grid, 512, smb, stream>>>(L, lda, ldz, n, m, a, w, z, err1, err2, flags, ref_flags);
  }
  return cudaGetLastError();
}

template <class T>
cudaError_t check_run(long L, int nm, int n, int m, const T *a0, const T *w, const T *z, double *err1, double *err2,
                      int *flags, float *ref_flags, cudaStream_t stream)
{
  if (bad_args(L, nm, n, m) || !a0 || !w || !z) return cudaErrorInvalidValue;
  if (n > 64) {  // 128 x 128 tiles on the FP64 tensor cores
    if (L > 0x7fffffffL) return cudaErrorInvalidValue;
    return launch_check_tc<T, false>(L, nm, nm, n, m, a0, w, z, err1, err2, flags, ref_flags, stream);
  }
  if (n > 32) {
    if (L > 0x7fffffffL) return cudaErrorInvalidValue;
    cudaError_t e = set_smem(k_check_cta<T, false>, check_cta_smem());
    if (e != cudaSuccess) return e;
    k_check_cta<T, false><<<(unsigned)L, 128, check_cta_smem(), stream>>>(L, nm, n, m, a0, w, z, err1, err2, flags,
                                                                         ref_flags);
    return cudaGetLastError();
  }
  const long blocks = std::min<long>((L + CKW_WARPS - 1) / CKW_WARPS, 65535);
  cudaError_t e = set_smem(k_check_w<T, false>, check_w_smem());
  if (e != cudaSuccess) return e;
  k_check_w<T, false><<<(unsigned)blocks, 32 * CKW_WARPS, check_w_smem(), stream>>>(L, nm, n, m, a0, w, z, err1, err2,
                                                                                    flags, ref_flags);
  return cudaGetLastError();
}

// The gate on a packed input (left intact by the packed solve): the same
// kernels, in the same order of operations, as check_run on the full
// layout, so the norms and flags are those of eigen_GPU_check_ex_* bit
// for bit.
template <class T>
cudaError_t check_packed_run(long L, int n, const T *ap, const T *w, const T *z, int ldz, double *err1, double *err2,
                             int *flags, cudaStream_t stream)
{
  if (L < 1 || L > 0x7fffffffL || n < 1 || n > 1024 || ldz < n || !ap || !w || !z) return cudaErrorInvalidValue;
  if (n > 64) {
    cudaError_t e = launch_check_tc<T, true>(L, 0, ldz, n, n, ap, w, z, err1, err2, flags, nullptr, stream);
    if (e != cudaSuccess) return e;
  } else if (n > 32) {
    cudaError_t e = set_smem(k_check_cta<T, true>, check_cta_smem());
    if (e != cudaSuccess) return e;
    k_check_cta<T, true><<<(unsigned)L, 128, check_cta_smem(), stream>>>(L, ldz, n, n, ap, w, z, err1, err2, flags,
                                                                        nullptr);
  } else {
    const long blocks = std::min<long>((L + CKW_WARPS - 1) / CKW_WARPS, 65535);
    cudaError_t e = set_smem(k_check_w<T, true>, check_w_smem());
    if (e != cudaSuccess) return e;
    k_check_w<T, true><<<(unsigned)blocks, 32 * CKW_WARPS, check_w_smem(), stream>>>(L, ldz, n, n, ap, w, z, err1,
                                                                                     err2, flags, nullptr);
  }
  return cudaGetLastError();
}

}  // namespace
}  // namespace eigb

extern "C" {

void eigen_GPU_batch_DP(const int L, const int nm, const int n, const int m, double *a, double *w, double *wk,
                        const cudaStream_t stream)
{
  eigb::dropin<double>(L, nm, n, m, a, w, wk, stream);
}

void eigen_GPU_batch_FP(const int L, const int nm, const int n, const int m, float *a, float *w, float *wk,
                        const cudaStream_t stream)
{
  eigb::dropin<float>(L, nm, n, m, a, w, wk, stream);
}

cudaError_t eigen_GPU_batch_BufferSize_DP(const int L, const int nm, const int n, const int m, size_t *lwork)
{
  return eigb::buffer_size<double>(L, nm, n, m, lwork);
}

cudaError_t eigen_GPU_batch_BufferSize_FP(const int L, const int nm, const int n, const int m, size_t *lwork)
{
  return eigb::buffer_size<float>(L, nm, n, m, lwork);
}

cudaError_t eigen_GPU_batch_ex_BufferSize_DP(const int L, const int nm, const int n, const int m,
                                             const eigen_GPU_batch_opts *opts, size_t *lwork)
{
  return eigb::buffer_size<double>(L, nm, n, m, lwork, opts);
}

cudaError_t eigen_GPU_batch_ex_BufferSize_FP(const int L, const int nm, const int n, const int m,
                                             const eigen_GPU_batch_opts *opts, size_t *lwork)
{
  return eigb::buffer_size<float>(L, nm, n, m, lwork, opts);
}

cudaError_t eigen_GPU_batch_ex_DP(const int L, const int nm, const int n, const int m, double *a, double *w, void *wk,
                                  const size_t lwork, int *info, const eigen_GPU_batch_opts *opts,
                                  const cudaStream_t stream)
{
  return eigb::run<double>(L, nm, n, m, a, w, wk, lwork, info, opts, stream);
}

cudaError_t eigen_GPU_batch_ex_FP(const int L, const int nm, const int n, const int m, float *a, float *w, void *wk,
                                  const size_t lwork, int *info, const eigen_GPU_batch_opts *opts,
                                  const cudaStream_t stream)
{
  return eigb::run<float>(L, nm, n, m, a, w, wk, lwork, info, opts, stream);
}

cudaError_t eigen_GPU_batch_stage_DP(const int L, const int nm, const int n, const int m, double *a, double *w,
                                     void *wk, const size_t lwork, int *info, const eigen_GPU_batch_opts *opts,
                                     const int phases, const int first, const int count, const cudaStream_t stream)
{
  eigb::Stage sg;
  sg.first = first;
  sg.count = count;
  sg.phases = phases;
  return eigb::run<double>(L, nm, n, m, a, w, wk, lwork, info, opts, stream, nullptr, eigb::Indirect(), sg);
}

cudaError_t eigen_GPU_batch_stage_FP(const int L, const int nm, const int n, const int m, float *a, float *w,
                                     void *wk, const size_t lwork, int *info, const eigen_GPU_batch_opts *opts,
                                     const int phases, const int first, const int count, const cudaStream_t stream)
{
  eigb::Stage sg;
  sg.first = first;
  sg.count = count;
  sg.phases = phases;
  return eigb::run<float>(L, nm, n, m, a, w, wk, lwork, info, opts, stream, nullptr, eigb::Indirect(), sg);
}

void eigen_GPU_check_DP(const int L, const int nm, const int n, const int m, double *a, double *w, double *z,
                        const cudaStream_t stream)
{
  if (eigb::check_run<double>(L, nm, n, m, a, w, z, nullptr, nullptr, nullptr, reinterpret_cast<float *>(a),
                              stream) == cudaSuccess)
    eigb::k_check_print<double><<<1, 1, 0, stream>>>(L, nm, n, a);
}

void eigen_GPU_check_FP(const int L, const int nm, const int n, const int m, float *a, float *w, float *z,
                        const cudaStream_t stream)
{
  if (eigb::check_run<float>(L, nm, n, m, a, w, z, nullptr, nullptr, nullptr, reinterpret_cast<float *>(a),
                             stream) == cudaSuccess)
    eigb::k_check_print<float><<<1, 1, 0, stream>>>(L, nm, n, a);
}

cudaError_t eigen_GPU_batch_packed_DP(const int L, const int n, const double *ap, double *z, const int ldz,
                                      double *w, void *wk, const size_t lwork, int *info,
                                      const eigen_GPU_batch_opts *opts, const cudaStream_t stream)
{
  if (ap == nullptr) return cudaErrorInvalidValue;
  return eigb::run<double>(L, ldz, n, n, z, w, wk, lwork, info, opts, stream, ap);
}

cudaError_t eigen_GPU_batch_packed_FP(const int L, const int n, const float *ap, float *z, const int ldz, float *w,
                                      void *wk, const size_t lwork, int *info, const eigen_GPU_batch_opts *opts,
                                      const cudaStream_t stream)
{
  if (ap == nullptr) return cudaErrorInvalidValue;
  return eigb::run<float>(L, ldz, n, n, z, w, wk, lwork, info, opts, stream, ap);
}

cudaError_t eigen_GPU_batch_packed_check_DP(const int L, const int n, const double *ap, double *z, const int ldz,
                                            double *w, void *wk, const size_t lwork, int *info,
                                            const eigen_GPU_batch_opts *opts, double *err1, double *err2, int *flags,
                                            const cudaStream_t stream)
{
  if (ap == nullptr) return cudaErrorInvalidValue;
  const cudaError_t err = eigb::run<double>(L, ldz, n, n, z, w, wk, lwork, info, opts, stream, ap);
  if (err != cudaSuccess) return err;
  return eigb::check_packed_run<double>(L, n, ap, w, z, ldz, err1, err2, flags, stream);
}

cudaError_t eigen_GPU_batch_packed_check_FP(const int L, const int n, const float *ap, float *z, const int ldz,
                                            float *w, void *wk, const size_t lwork, int *info,
                                            const eigen_GPU_batch_opts *opts, double *err1, double *err2, int *flags,
                                            const cudaStream_t stream)
{
  if (ap == nullptr) return cudaErrorInvalidValue;
  const cudaError_t err = eigb::run<float>(L, ldz, n, n, z, w, wk, lwork, info, opts, stream, ap);
  if (err != cudaSuccess) return err;
  return eigb::check_packed_run<float>(L, n, ap, w, z, ldz, err1, err2, flags, stream);
}

cudaError_t eigen_GPU_batch_interleaved_BufferSize_DP(const int L, const int n, const eigen_GPU_batch_opts *opts,
                                                      size_t *lwork)
{
  size_t a, b, bytes = 0;
  const cudaError_t err = eigb::interleaved_plan<double>(L, n, opts, a, b, bytes);
  if (lwork) *lwork = err == cudaSuccess ? bytes : 0;
  return err;
}

cudaError_t eigen_GPU_batch_interleaved_BufferSize_FP(const int L, const int n, const eigen_GPU_batch_opts *opts,
                                                      size_t *lwork)
{
  size_t a, b, bytes = 0;
  const cudaError_t err = eigb::interleaved_plan<float>(L, n, opts, a, b, bytes);
  if (lwork) *lwork = err == cudaSuccess ? bytes : 0;
  return err;
}

cudaError_t eigen_GPU_batch_interleaved_DP(const int L, const int n, const double *ai, double *zi, double *wi,
                                           void *wk, const size_t lwork, int *info,
                                           const eigen_GPU_batch_opts *opts, const cudaStream_t stream)
{
  return eigb::run_interleaved<double>(L, n, ai, zi, wi, wk, lwork, info, opts, stream);
}

cudaError_t eigen_GPU_batch_interleaved_FP(const int L, const int n, const float *ai, float *zi, float *wi,
                                           void *wk, const size_t lwork, int *info,
                                           const eigen_GPU_batch_opts *opts, const cudaStream_t stream)
{
  return eigb::run_interleaved<float>(L, n, ai, zi, wi, wk, lwork, info, opts, stream);
}

cudaError_t eigen_GPU_batch_uneven_BufferSize_DP(const int L, const int *n, const eigen_GPU_batch_opts *opts,
                                                 size_t *lwork)
{
  return eigb::uneven_buffer_size<double>(L, n, opts, lwork);
}

cudaError_t eigen_GPU_batch_uneven_BufferSize_FP(const int L, const int *n, const eigen_GPU_batch_opts *opts,
                                                 size_t *lwork)
{
  return eigb::uneven_buffer_size<float>(L, n, opts, lwork);
}

cudaError_t eigen_GPU_batch_uneven_DP(const int L, const int *n, double *a, double *w, void *wk, const size_t lwork,
                                      int *info, const eigen_GPU_batch_opts *opts, const cudaStream_t stream)
{
  return eigb::run_uneven<double>(L, n, a, w, wk, lwork, info, opts, stream);
}

cudaError_t eigen_GPU_batch_uneven_FP(const int L, const int *n, float *a, float *w, void *wk, const size_t lwork,
                                      int *info, const eigen_GPU_batch_opts *opts, const cudaStream_t stream)
{
  return eigb::run_uneven<float>(L, n, a, w, wk, lwork, info, opts, stream);
}

cudaError_t eigen_GPU_batch_noalloc_DP(const int L, const int nm, const int n, const int m, double *a, double *w,
                                       int *info, const cudaStream_t stream)
{
  return eigb::run_noalloc<double>(L, nm, n, m, a, w, info, stream);
}

cudaError_t eigen_GPU_batch_symfunc_DP(const int L, const int nm, const int n, const double *v, const double *w,
                                       double *z, const int func, const double p, const cudaStream_t stream)
{
  return eigb::symfunc_run<double>(L, nm, n, v, w, z, func, p, stream);
}

cudaError_t eigen_GPU_batch_symfunc_FP(const int L, const int nm, const int n, const float *v, const float *w,
                                       float *z, const int func, const double p, const cudaStream_t stream)
{
  return eigb::symfunc_run<float>(L, nm, n, v, w, z, func, p, stream);
}

cudaError_t eigen_GPU_batch_launch_params_DP(const int L, const int n, int *grpSZ, int *numTB, int *numGR,
                                             int *numTH, int *sizeSH, int *sizeL2)
{
  return eigb::launch_params<double>(L, n, grpSZ, numTB, numGR, numTH, sizeSH, sizeL2);
}

cudaError_t eigen_GPU_batch_launch_params_FP(const int L, const int n, int *grpSZ, int *numTB, int *numGR,
                                             int *numTH, int *sizeSH, int *sizeL2)
{
  return eigb::launch_params<float>(L, n, grpSZ, numTB, numGR, numTH, sizeSH, sizeL2);
}

cudaError_t eigen_GPU_batch_refine_BufferSize_DP(const int L, const int nm, const int n,
                                                const eigen_GPU_refine_opts *opts, size_t *lwork)
{
  return eigb::ref_buffer_size(L, nm, n, opts, lwork);
}

cudaError_t eigen_GPU_batch_refine_DP(const int L, const int nm, const int n, double *a, double *w, void *wk,
                                      const size_t lwork, int *info, int *iters, const eigen_GPU_refine_opts *opts,
                                      const cudaStream_t stream)
{
  return eigb::run_refine(L, nm, n, a, w, wk, lwork, info, iters, opts, stream);
}

cudaError_t eigen_GPU_batch_rayleigh_BufferSize_DP(const int L, const int nm, const int n, size_t *lwork)
{
  return eigb::ray_buffer_size(L, nm, n, lwork);
}

cudaError_t eigen_GPU_batch_rayleigh_DP(const int L, const int nm, const int n, const double *a, const double *x,
                                        double *s, double *g, void *wk, const size_t lwork, const cudaStream_t stream)
{
  return eigb::run_rayleigh(L, nm, n, a, x, s, g, wk, lwork, stream);
}

cudaError_t eigen_GPU_mlp_size(const int d0, const int d1, const int d2, const int d3, size_t *bytes)
{
  if (!bytes) return cudaErrorInvalidValue;
  *bytes = 0;
  if (eigb::mlp_bad(d0, d1, d2, d3)) return cudaErrorInvalidValue;
  *bytes = eigb::mlp_layout(d0, d1, d2, d3).bytes;
  return cudaSuccess;
}

cudaError_t eigen_GPU_mlp_ws_size(const int d0, const int d1, const int d2, const int d3, const int rows, size_t *bytes)
{
  if (!bytes) return cudaErrorInvalidValue;
  *bytes = 0;
  if (eigb::mlp_bad(d0, d1, d2, d3) || rows < 8 || (rows % 8)) return cudaErrorInvalidValue;
  *bytes = eigb::mlp_ws(eigb::mlp_layout(d0, d1, d2, d3), rows, true).bytes;
  return cudaSuccess;
}

cudaError_t eigen_GPU_mlp_init(const int d0, const int d1, const int d2, const int d3, void *params,
                               const unsigned long long seed, const cudaStream_t stream)
{
  if (eigb::mlp_bad(d0, d1, d2, d3) || !params) return cudaErrorInvalidValue;
  return eigb::mlp_init(eigb::mlp_layout(d0, d1, d2, d3), params, seed, stream);
}

cudaError_t eigen_GPU_mlp_forward(const int d0, const int d1, const int d2, const int d3, const void *params,
                                  const int rows, const float *x, float *y, void *ws, const size_t lws,
                                  const cudaStream_t stream)
{
  if (eigb::mlp_bad(d0, d1, d2, d3) || rows < 8 || (rows % 8) || !params || !x || !y || !ws)
    return cudaErrorInvalidValue;
  const eigb::MlpLayout l = eigb::mlp_layout(d0, d1, d2, d3);
  const eigb::MlpWs w = eigb::mlp_ws(l, rows, true);
  if (lws != 0 && lws < w.bytes) return cudaErrorInvalidValue;
  return eigb::mlp_forward(l, params, rows, x, y, static_cast<char *>(ws), w, false, stream);
}

cudaError_t eigen_GPU_mlp_gradient(const int d0, const int d1, const int d2, const int d3, const void *params,
                                   const int rows, const float *x, const float *t, float *grad, double *sse,
                                   void *ws, const size_t lws, const cudaStream_t stream)
{
  if (eigb::mlp_bad(d0, d1, d2, d3) || rows < 8 || (rows % 8) || !params || !x || !t || !grad || !ws)
    return cudaErrorInvalidValue;
  const eigb::MlpLayout l = eigb::mlp_layout(d0, d1, d2, d3);
  const eigb::MlpWs w = eigb::mlp_ws(l, rows, true);
  if (lws != 0 && lws < w.bytes) return cudaErrorInvalidValue;
  char *wsp = static_cast<char *>(ws);
  cudaError_t err = cudaMemsetAsync(wsp + w.err, 0, sizeof(int), stream);
  if (err != cudaSuccess) return err;
  if ((err = eigb::mlp_forward(l, params, rows, x, nullptr, wsp, w, true, stream)) != cudaSuccess) return err;
  return eigb::mlp_backward(l, params, rows, t, grad, sse, wsp, w, stream);
}

cudaError_t eigen_GPU_mlp_train_step(const int d0, const int d1, const int d2, const int d3, void *params,
                                     const int rows, const float *x, const float *t, const float lr, const int step,
                                     double *sse, void *ws, const size_t lws, const cudaStream_t stream)
{
  if (eigb::mlp_bad(d0, d1, d2, d3) || rows < 8 || (rows % 8) || !params || !x || !t || !ws || step < 1)
    return cudaErrorInvalidValue;
  const eigb::MlpLayout l = eigb::mlp_layout(d0, d1, d2, d3);
  const eigb::MlpWs w = eigb::mlp_ws(l, rows, true);
  if (lws != 0 && lws < w.bytes) return cudaErrorInvalidValue;
  char *wsp = static_cast<char *>(ws);
  float *grad = reinterpret_cast<float *>(wsp + w.grad);
  cudaError_t err;
  if ((err = eigb::mlp_forward(l, params, rows, x, nullptr, wsp, w, true, stream)) != cudaSuccess) return err;
  if ((err = eigb::mlp_backward(l, params, rows, t, grad, sse, wsp, w, stream)) != cudaSuccess) return err;
  return eigb::mlp_adam(l, params, grad, lr, step, stream);
}

cudaError_t eigen_GPU_learned_targets_FP(const int L, const int n, const float *v, const int ldv, const float *v0,
                                         float *c, const cudaStream_t stream)
{
  if (L < 1 || n < 1 || n > eigb::LW_NMAX || ldv < n || !v || !v0 || !c) return cudaErrorInvalidValue;
  const size_t smem = sizeof(float) * 2 * (size_t)n * n;
  cudaError_t err = eigb::set_smem(eigb::k_lw_targets, smem);
  if (err != cudaSuccess) return err;
  eigb::k_lw_targets<<<(unsigned)L, 256, smem, stream>>>(n, v, ldv, v0, c);
  return cudaGetLastError();
}

cudaError_t eigen_GPU_batch_learned_BufferSize_FP(const int L, const int nm, const int n, const int d1, const int d2,
                                                  const eigen_GPU_learned_opts *opts, size_t *lwork)
{
  return eigb::lw_buffer_size(L, nm, n, d1, d2, opts, lwork);
}

cudaError_t eigen_GPU_batch_learned_FP(const int L, const int nm, const int n, float *a, float *w, const float *family,
                                       const void *params, const int d1, const int d2, void *wk, const size_t lwork,
                                       int *info, int *sweeps, double *resid, const eigen_GPU_learned_opts *opts,
                                       const cudaStream_t stream)
{
  return eigb::run_learned(L, nm, n, a, w, family, params, d1, d2, wk, lwork, info, sweeps, resid, opts, stream);
}

cudaError_t eigen_GPU_batch_tune_set(const eigen_GPU_tune_entry *entries, const int count)
{
  if (count < 0 || (count > 0 && entries == nullptr)) return cudaErrorInvalidValue;
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  for (int i = 0; i < count; i++) {
    const eigen_GPU_tune_entry &e = entries[i];
    if ((e.esize != 4 && e.esize != 8) || e.n < 1 || e.n > 1024 || e.split < 0 || e.split > 32 ||
        (e.zmem != EIGEN_GPU_ZMEM_AUTO && e.zmem != EIGEN_GPU_ZMEM_SHARED) || e.ql_mpw < 0 || e.ql_mpw > 32 ||
        (e.ql_mpw & (e.ql_mpw - 1)) != 0 || e.reduce < EIGEN_GPU_REDUCE_AUTO || e.reduce > EIGEN_GPU_REDUCE_CLUSTER)
      return cudaErrorInvalidValue;
  }
  std::lock_guard<std::mutex> lk(eigb::g_mu);
  for (auto it = eigb::g_tune.begin(); it != eigb::g_tune.end();) {
    if (it->first.dev == dev) it = eigb::g_tune.erase(it);
    else ++it;
  }
  for (int i = 0; i < count; i++) eigb::g_tune[eigb::TuneKey{dev, entries[i].esize, entries[i].n}] = entries[i];
  return cudaSuccess;
}

cudaError_t eigen_GPU_batch_tune_get(const int esize, const int n, eigen_GPU_tune_entry *out)
{
  if (!out) return cudaErrorInvalidValue;
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  std::lock_guard<std::mutex> lk(eigb::g_mu);
  auto it = eigb::g_tune.find(eigb::TuneKey{dev, esize, n});
  if (it == eigb::g_tune.end()) return cudaErrorInvalidValue;
  *out = it->second;
  return cudaSuccess;
}

cudaError_t eigen_GPU_batch_trace(cudaEvent_t *events, const int nevents)
{
  if (events != nullptr && nevents < 4) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lk(eigb::g_mu);
  eigb::g_trace = events;
  eigb::g_ntrace = events ? nevents : 0;
  return cudaSuccess;
}

cudaError_t eigen_GPU_check_ex_DP(const int L, const int nm, const int n, const int m, const double *a,
                                  const double *w, const double *z, double *err1, double *err2, int *flags,
                                  const cudaStream_t stream)
{
  return eigb::check_run<double>(L, nm, n, m, a, w, z, err1, err2, flags, nullptr, stream);
}

cudaError_t eigen_GPU_check_ex_FP(const int L, const int nm, const int n, const int m, const float *a,
                                  const float *w, const float *z, double *err1, double *err2, int *flags,
                                  const cudaStream_t stream)
{
  return eigb::check_run<float>(L, nm, n, m, a, w, z, err1, err2, flags, nullptr, stream);
}

}  // extern "C"
