// The QL phase of a mixed-size batch in one persistent launch.
//
// The reduction and apply phases of a mixed-size batch run per order (their
// kernels are shaped by n); the QL phase is one serial recurrence per
// matrix, whatever its order, so every matrix of a wave of the batch goes
// through a single launch.  Its threads (mpw lanes per warp, each with a
// shared-memory slot for 2 nmax values) take matrices from one device work
// queue, an atomic counter over a job list sorted by decreasing order
// (longest processing time first: the longest chains start at once, the
// short ones fill in behind them).  Each job runs the same recurrence as
// k2_ql (ql_tql2_fast / ql_imtql2_fast on a shared-memory copy of d and e:
// identical rotations and eigenvalues) and leaves the records, the status
// block and the unsorted eigenvalues exactly where k2_ql leaves them, so the
// apply phase of each group runs unchanged.
#pragma once
#include "eigb_kernels.cuh"

namespace eigb {

// one group (or part of a group) of a mixed-size batch: its matrices' slots
// in the workspace of its reduction and apply launches
template <class T> struct QGroup {
  T *d, *e;      // n per matrix
  Meta *meta;    // one per matrix
  Rec<T> *rec;   // rcap per matrix
  int n, rcap;
};

struct QJob {
  int g, k;  // group, matrix within the group
};

template <class T> __host__ __device__ constexpr size_t queue_slot_bytes(int nmax) { return 2 * sizeof(T) * (size_t)nmax; }

template <class T>
__global__ void __launch_bounds__(K2_MAX_WARPS * 32)
    k2_ql_queue(const QGroup<T> *__restrict__ groups, const QJob *__restrict__ jobs, const int njobs,
                int *__restrict__ next, const int mpw, const int nmax, const int method, const int max_sweep)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  if (lane >= mpw) return;  // no barriers in this kernel
  const int st = (blockDim.x >> 5) * mpw;  // slots per block
  const int slot = (threadIdx.x >> 5) * mpw + lane;
  T *dd = reinterpret_cast<T *>(smem_raw) + slot;
  T *ee = dd + (size_t)nmax * st;
  for (;;) {
    const int j = atomicAdd(next, 1);
    if (j >= njobs) return;
    const QJob job = jobs[j];
    const QGroup<T> G = groups[job.g];
    const int n = G.n;
    if (n > nmax) {  // not reached: the host sizes the slots for the wave's largest order
      Meta bad;
      bad.nrec = 0;
      bad.pad = 0;
      bad.overflow = 1;  // the apply phase solves the matrix itself
      bad.ierr = 0;
      G.meta[job.k] = bad;
      continue;
    }
    const T *din = G.d + (size_t)job.k * n;
    T *ein = G.e + (size_t)job.k * n;
    for (int i = 0; i < n; i++) {
      dd[(size_t)i * st] = din[i];
      ee[(size_t)i * st] = ein[i];
    }
    Rec<T> *out = G.rec + (size_t)job.k * G.rcap;
    int ierr = 0;
    const int nr = (method == QL_IMTQL2) ? ql_imtql2_fast(dd, ee, st, n, out, G.rcap, max_sweep, &ierr)
                                         : ql_tql2_fast(dd, ee, st, n, out, G.rcap, max_sweep, &ierr);
    Meta mt;
    mt.nrec = nr < 0 ? 0 : nr;
    mt.pad = 0;
    if (nr < 0) {
      mt.overflow = 1;
      mt.ierr = 0;
    } else {
      mt.overflow = 0;
      mt.ierr = ierr;
      for (int i = 0; i < n; i++) ein[i] = dd[(size_t)i * st];  // unsorted eigenvalues over e, as k2_ql
    }
    G.meta[job.k] = mt;
  }
}

}  // namespace eigb
