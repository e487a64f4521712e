// Host build of the library's phase-1 team code (csrc/eigb_tridiag.cuh:
// tridiagonalization + explicit Q^T) for CPU unit tests.  The GPU team (a
// warp or a CTA) is emulated by one std::thread per GPU thread, with
// std::barrier standing in for __syncthreads and a shared array for the
// team reductions, so the source's barrier placement is exercised too.
#include <barrier>
#include <thread>
#include <vector>

#include "../../eigeng-batched_b200/csrc/eigb_tridiag.cuh"
#include "../../eigeng-batched_b200/csrc/eigb_tridiag_reg.cuh"

template <class T> struct HostShared {
  std::barrier<> bar;
  std::barrier<> wbar;   // the barrier of warp 0 alone
  std::vector<T> slots;  // 2 x nthr, alternating halves
  std::vector<T> posted; // 2 x nthr: the buffers of post()/total()
  std::vector<T> wsl;    // 32: the exchanges of warp 0
  explicit HostShared(int nthr)
      : bar(nthr), wbar(32), slots(2 * (size_t)nthr), posted(2 * (size_t)nthr), wsl(32)
  {
  }
};

template <class T> struct HostTeam {
  int rank, nthr, flip;
  HostShared<T> *sh;
  int size() const { return nthr; }
  void sync() const { sh->bar.arrive_and_wait(); }
  T sum(T x, T *)
  {
    T *buf = sh->slots.data() + (flip ? nthr : 0);
    flip ^= 1;
    buf[rank] = x;
    sh->bar.arrive_and_wait();
    T s = T(0);
    for (int k = 0; k < nthr; k++) s += buf[k];  // same order in every thread
    return s;
  }
  // one slot per thread; total() adds the threads of warps w0 .. w0+nw-1
  void post(T x, T *, int id) { sh->posted[(size_t)id * nthr + rank] = x; }
  void post_zero(T *, int id) { sh->posted[(size_t)id * nthr + rank] = T(0); }
  // warp 0's own operations (only its 32 threads call them)
  void sync_warp() const { sh->wbar.arrive_and_wait(); }
  T shfl(T x, int src) const
  {
    sh->wsl[rank & 31] = x;
    sh->wbar.arrive_and_wait();
    const T v = sh->wsl[src];
    sh->wbar.arrive_and_wait();
    return v;
  }
  T wsum(T x) const
  {
    sh->wsl[rank & 31] = x;
    sh->wbar.arrive_and_wait();
    T s = T(0);
    for (int k = 0; k < 32; k++) s += sh->wsl[k];
    sh->wbar.arrive_and_wait();
    return s;
  }
  T total(const T *, int id, int w0, int nw) const
  {
    const T *buf = sh->posted.data() + (size_t)id * nthr;
    T s = T(0);
    for (int k = 32 * w0; k < 32 * (w0 + nw) && k < nthr; k++) s += buf[k];
    return s;
  }
};

// The matrix (full symmetric, column-major, leading dimension ldg) is in G;
// its leading B x B block is moved to a separate "shared" array for the run
// and back afterwards, as k1_cta stages it.
template <class T, int SPLIT> static void run(int n, int nthr, T *G, int ldg, int B, T *d, T *e)
{
  HostShared<T> sh(nthr);
  const int ld = B | 1;
  std::vector<T> beta(n + 1), pv(n + 1), part(eigb::TQ_QB * nthr), red(72), S((size_t)B * ld + 1),
      ubuf(eigb::TQ_QB * (size_t)n), gram(3 * (size_t)n);
  for (int c = 0; c < B; c++)
    for (int r = 0; r < B; r++) S[r + (size_t)c * ld] = G[r + (size_t)c * ldg];
  std::vector<std::thread> th;
  for (int t = 0; t < nthr; t++)
    th.emplace_back([&, t]() {
      HostTeam<T> tm{t, nthr, 0, &sh};
      eigb::tridiag_qt<T, SPLIT>(tm, S.data(), ld, G, ldg, B, n, d, e, beta.data(), pv.data(), part.data(),
                                 red.data(), ubuf.data(), gram.data());
    });
  for (auto &x : th) x.join();
  for (int c = 0; c < B; c++)
    for (int r = 0; r < B; r++) G[r + (size_t)c * ldg] = S[r + (size_t)c * ld];
}

template <class T> static void run_split(int n, int nthr, int split, T *S, int ld, int B, T *d, T *e)
{
  if (split == 4) run<T, 4>(n, nthr, S, ld, B, d, e);
  else if (split == 2) run<T, 2>(n, nthr, S, ld, B, d, e);
  else run<T, 1>(n, nthr, S, ld, B, d, e);
}

extern "C" void host_tridiag_d(int n, int nthr, int split, double *S, int ld, int B, double *d, double *e)
{
  run_split<double>(n, nthr, split, S, ld, B, d, e);
}
extern "C" void host_tridiag_f(int n, int nthr, int split, float *S, int ld, int B, float *d, float *e)
{
  run_split<float>(n, nthr, split, S, ld, B, d, e);
}

// register-resident variant: one "thread" per GPU thread of the CTA
template <class T, int NB> static void run_reg(int n, T *A, int nm, T *d, T *e)
{
  const int nthr = 32 * NB * NB;
  HostShared<T> sh(nthr);
  std::vector<double2> smem_store((eigb::reg_smem_elems<NB>(n) * sizeof(T) + 15) / 16);
  T *smem_p = reinterpret_cast<T *>(smem_store.data());
  std::vector<std::thread> th;
  for (int t = 0; t < nthr; t++)
    th.emplace_back([&, t]() {
      HostTeam<T> tm{t, nthr, 0, &sh};
      eigb::tridiag_qt_reg<T, NB>(tm, A, nm, n, d, e, smem_p);
    });
  for (auto &x : th) x.join();
}

template <class T> static void run_reg_nb(int n, T *A, int nm, T *d, T *e)
{
  const int nb = (n + 31) / 32;
  if (nb <= 2) run_reg<T, 2>(n, A, nm, d, e);
  else if (nb == 3) run_reg<T, 3>(n, A, nm, d, e);
  else run_reg<T, 4>(n, A, nm, d, e);
}

extern "C" void host_tridiag_reg_d(int n, double *A, int nm, double *d, double *e) { run_reg_nb<double>(n, A, nm, d, e); }
extern "C" void host_tridiag_reg_f(int n, float *A, int nm, float *d, float *e) { run_reg_nb<float>(n, A, nm, d, e); }
