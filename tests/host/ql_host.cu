// Host build of the library's QL rotation generator (csrc/eigb_ql.cuh) for
// CPU unit tests: the same source that phase 2 and the phase-3 fallback run
// on the GPU, compiled as host code.
#include "../../eigeng-batched_b200/csrc/eigb_ql.cuh"

template <class T>
static int run(int n, T *d, T *e, int method, int max_sweep, int cap, int chunk, T *rec_out, int *nrec_out,
               int *ierr)
{
  using namespace eigb;
  QLGen<T> g;
  g.pc = PC_START;
  DEView<T> v{d, e, 1};
  Rec<T> *out = reinterpret_cast<Rec<T> *>(rec_out);
  int total = 0;
  // chunk > 0: resume in pieces of `chunk` records (the phase-3 fallback);
  // otherwise one call with capacity `cap` (phase 2)
  while (true) {
    const int room = chunk > 0 ? chunk : cap - total;
    if (room < 2 || total + room > cap) return -1;
    const int nr = ql_run(method, g, v, n, out + total, room, max_sweep);
    total += nr;
    if (g.pc == PC_DONE) break;
    if (chunk <= 0) {
      *nrec_out = total;
      *ierr = 0;
      return 1;  // overflow
    }
  }
  *nrec_out = total;
  *ierr = g.ierr;
  return 0;
}

extern "C" int host_ql_d(int n, double *d, double *e, int method, int max_sweep, int cap, int chunk, double *rec,
                         int *nrec, int *ierr)
{
  return run<double>(n, d, e, method, max_sweep, cap, chunk, rec, nrec, ierr);
}
extern "C" int host_ql_f(int n, float *d, float *e, int method, int max_sweep, int cap, int chunk, float *rec,
                         int *nrec, int *ierr)
{
  return run<float>(n, d, e, method, max_sweep, cap, chunk, rec, nrec, ierr);
}

template <class T>
static int run_fast(int n, T *d, T *e, int method, int max_sweep, int cap, T *rec_out, int *nrec_out, int *ierr)
{
  using namespace eigb;
  Rec<T> *out = reinterpret_cast<Rec<T> *>(rec_out);
  const int nr = method == QL_IMTQL2 ? ql_imtql2_fast(d, e, 1, n, out, cap, max_sweep, ierr)
                                    : ql_tql2_fast(d, e, 1, n, out, cap, max_sweep, ierr);
  *nrec_out = nr < 0 ? 0 : nr;
  return nr < 0 ? 1 : 0;
}
extern "C" int host_ql_fast_d(int n, double *d, double *e, int method, int max_sweep, int cap, double *rec,
                              int *nrec, int *ierr)
{
  return run_fast<double>(n, d, e, method, max_sweep, cap, rec, nrec, ierr);
}
extern "C" int host_ql_fast_f(int n, float *d, float *e, int method, int max_sweep, int cap, float *rec,
                              int *nrec, int *ierr)
{
  return run_fast<float>(n, d, e, method, max_sweep, cap, rec, nrec, ierr);
}
