// Host build of the phase-3 apply (csrc/eigb_kernels.cuh: seg_walk,
// apply_segments with seg_apply and seg_apply_pair) for CPU unit tests: applies a rotation record stream to a
// row-major n x n matrix, staging it in chunks of `ch` records exactly as
// k3_cta does.
#include "../../eigeng-batched_b200/csrc/eigb_kernels.cuh"

template <class T> static int run(int n, T *Z, const T *recs, int nrec, int ch)
{
  using namespace eigb;
  const Rec<T> *src = reinterpret_cast<const Rec<T> *>(recs);
  int base = 0, segs = 0;
  while (base < nrec) {
    const int cnt = nrec - base < ch ? nrec - base : ch;
    const Rec<T> *rb = src + base;
    const int used = seg_walk(rb, cnt);
    for (int r = 0; r < n; r++) apply_segments<T, 1>(rb, used, Z + r * n, 1);
    for (int q = 0; q < used; q += 1 + hdr_cnt(rb[q])) segs++;
    base += used > 0 ? used : cnt;
  }
  return segs;
}

extern "C" int host_apply_d(int n, double *Z, const double *recs, int nrec, int ch) { return run<double>(n, Z, recs, nrec, ch); }
extern "C" int host_apply_f(int n, float *Z, const float *recs, int nrec, int ch) { return run<float>(n, Z, recs, nrec, ch); }
