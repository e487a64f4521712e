// Host build of the phase-3 wavefront (csrc/eigb_kernels.cuh: parse_group,
// wave_apply) for CPU unit tests: applies a rotation record stream to a
// row-major n x n matrix, staging it in chunks of `ch` records exactly as
// k3_cta does.
#include "../../eigeng-batched_b200/csrc/eigb_kernels.cuh"

template <class T> static int run(int n, T *Z, const T *recs, int nrec, int ch)
{
  using namespace eigb;
  const Rec<T> *src = reinterpret_cast<const Rec<T> *>(recs);
  int base = 0, groups = 0;
  while (base < nrec) {
    const int cnt = nrec - base < ch ? nrec - base : ch;
    const Rec<T> *rb = src + base;
    int q = 0;
    while (true) {
      int i0[K3_WAVE], len[K3_WAVE], off[K3_WAVE];
      const int ns = parse_group(rb, cnt, q, i0, len, off);
      if (ns == 0) break;
      groups++;
      for (int r = 0; r < n; r++) wave_apply<T, 1>(Z + r * n, 1, n, rb, i0, len, off, ns);
    }
    base += q > 0 ? q : cnt;
  }
  return groups;
}

extern "C" int host_apply_d(int n, double *Z, const double *recs, int nrec, int ch) { return run<double>(n, Z, recs, nrec, ch); }
extern "C" int host_apply_f(int n, float *Z, const float *recs, int nrec, int ch) { return run<float>(n, Z, recs, nrec, ch); }
