// Host build of the phase-3 apply (csrc/eigb_kernels.cuh: seg_walk,
// apply_segments with seg_apply and seg_apply_pair; csrc/eigb_apply.cuh:
// apply_grouped with seg_apply_group) for CPU unit tests: applies a rotation
// record stream to a row-major n x n matrix, staging it in chunks of `ch`
// records exactly as k3_cta and k3_tmem do.
#include "../../eigeng-batched_b200/csrc/eigb_kernels.cuh"

// a single sweep on a row in memory (functor for apply_grouped)
template <class T> struct SingleMem {
  T *z;
  void operator()(const eigb::Rec<T> *rp, const int i0, const int len) const { eigb::seg_apply<T, 1>(z, 1, rp, i0, len); }
};

// kg = 0: apply_segments (k3_cta's walker, pairs of equal sweeps);
// kg = 2, 4, 8: apply_grouped with groups of up to kg sweeps (k3_tmem's walker)
template <class T> static int run(int n, T *Z, const T *recs, int nrec, int ch, int kg)
{
  using namespace eigb;
  const Rec<T> *src = reinterpret_cast<const Rec<T> *>(recs);
  int base = 0, segs = 0;
  while (base < nrec) {
    const int cnt = nrec - base < ch ? nrec - base : ch;
    const Rec<T> *rb = src + base;
    const int used = seg_walk(rb, cnt);
    for (int r = 0; r < n; r++) {
      T *z = Z + r * n;
      if (kg == 8) apply_grouped<T, 8>(rb, used, RowMem<T, 1>{z, 1}, SingleMem<T>{z});
      else if (kg == 4) apply_grouped<T, 4>(rb, used, RowMem<T, 1>{z, 1}, SingleMem<T>{z});
      else if (kg == 2) apply_grouped<T, 2>(rb, used, RowMem<T, 1>{z, 1}, SingleMem<T>{z});
      else apply_segments<T, 1>(rb, used, z, 1);
    }
    for (int q = 0; q < used; q += 1 + hdr_cnt(rb[q])) segs++;
    base += used > 0 ? used : cnt;
  }
  return segs;
}

extern "C" int host_apply_d(int n, double *Z, const double *recs, int nrec, int ch, int kg)
{
  return run<double>(n, Z, recs, nrec, ch, kg);
}
extern "C" int host_apply_f(int n, float *Z, const float *recs, int nrec, int ch, int kg)
{
  return run<float>(n, Z, recs, nrec, ch, kg);
}
