// Phase 2: QL iteration on the tridiagonal (d, e), emitting plane rotations.
//
// The eigenvalue recurrence of QL is a serial chain per matrix; it does not
// depend on the eigenvectors.  It therefore runs one matrix per thread
// (a warp advances 32 independent chains at once) and writes the rotations
// as a stream of records that phase 3 applies to Q with a whole team per
// matrix.  The same generator also runs inside phase 3 (one thread, small
// chunks) for the rare matrix whose stream exceeded its capacity.
//
// The generator is resumable: it returns when the output buffer is full,
// keeping every loop variable in QLGen, and continues from the same
// rotation on the next call.
//
// tql2: explicit-shift QL, tql2_tiled.hpp:3-192 / tql2.hpp:3-213.
// imtql2: implicit Wilkinson-shift QL, imtql2_tiled.hpp:3-176 / imtql2.hpp.
// Deflation tolerances, the sweep limit and the e(n) = 0 convention follow
// the reference; the rotation (c, s, r) is formed with one reciprocal
// square root (givens()) rather than hypot + two divisions.
#pragma once
#include "eigb_common.cuh"

namespace eigb {

enum { QL_TQL2 = 0, QL_IMTQL2 = 1 };
enum { PC_START = 0, PC_ROT = 1, PC_DONE = 2 };

template <class T> struct QLGen {
  int pc, l, m, i, itr, ierr;
  int seg_pos, seg_cnt, seg_i0;
  T shift, tst1, c, c2, c3, s, s2, p, el1, dl1, ei, di1, r, delta;
};

// Strided view of one chain's d and e (interleaved across the threads of a
// block so that divergent indices stay bank-conflict free).
template <class T> struct DEView {
  T *d, *e;
  int st;
  __host__ __device__ __forceinline__ T &D(int i) const { return d[i * st]; }
  __host__ __device__ __forceinline__ T &E(int i) const { return e[i * st]; }
};

// One tql2 chase step at index i (tql2_tiled.hpp:94-115): from the
// previous (c, s, p) and (e_i, d_i) to the new rotation (cn, sn), the new p
// and the values stored at i+1.  Shared by both generators.
template <class T>
__host__ __device__ __forceinline__ void tql2_step(const T c, const T s, const T p, const T ei, const T di, T &cn,
                                                   T &sn, T &pn, T &ei1, T &di1)
{
  const T gg = mul_rn(c, ei);
  const T h = mul_rn(c, p);
  T r;
  givens(p, ei, cn, sn, r);
  ei1 = mul_rn(s, r);
  pn = fma(cn, di, -mul_rn(sn, gg));
  di1 = fma(sn, fma(cn, gg, mul_rn(sn, di)), h);
}

// Explicit shift of tql2 (tql2_tiled.hpp:64-75): new d(l), d(l+1).
template <class T>
__host__ __device__ __forceinline__ void tql2_shift(const T dl_old, const T dl1_old, const T el, T &dl, T &dl1)
{
  const T p = (dl1_old - dl_old) / (el + el);
  const T r = hypot1(p);
  const T psr = p + copysign_t(r, p);
  dl = el / psr;
  dl1 = mul_rn(el, psr);
}

// End of a tql2 sweep (tql2_tiled.hpp:126-130): new e(l), d(l).
template <class T>
__host__ __device__ __forceinline__ void tql2_close(const T c, const T s, const T s2, const T c3, const T el1,
                                                    const T ei, const T dl1, T &el, T &dl)
{
  const T r = mul_rn(mul_rn(mul_rn(mul_rn(-s, s2), c3), el1), ei) / dl1;
  el = mul_rn(s, r);
  dl = mul_rn(c, r);
}

// One imtql2 chase step (imtql2_tiled.hpp:86-115) after the rotation
// (cn, sn) has been formed: returns the new d(i+1) and updates di1, delta,
// r.
template <class T>
__host__ __device__ __forceinline__ T imtql2_step(const T cn, const T sn, const T c_old, const T ei, const T di,
                                                  T &di1, T &delta, T &r)
{
  const T b = mul_rn(c_old, ei);
  const T dix = di1 - delta;
  di1 = di;
  const T q = fma(di - dix, sn, mul_rn(T(2) * cn, b));
  const T dx1 = fma(sn, q, dix);
  delta = dx1 - dix;
  r = fma(cn, q, -b);
  return dx1;
}

// Wilkinson-type shift of imtql2 (imtql2_tiled.hpp:67-75).
template <class T>
__host__ __device__ __forceinline__ T imtql2_shift(const T dl, const T dl1, const T el, const T dm)
{
  const T f = (dl1 - dl) / (el + el);
  const T g = hypot1(f);
  return (dm - dl) + el / (f + copysign_t(g, f));
}

template <class T>
__host__ __device__ __forceinline__ void ql_close_seg(QLGen<T> &g, Rec<T> *buf)
{
  if (g.seg_pos >= 0) {
    buf[g.seg_pos] = make_hdr(g.seg_i0, g.seg_cnt, T(0));
    g.seg_pos = -1;
  }
}

// Runs until done or until `cap` records are in buf; returns the number of
// records written.  g.pc == PC_DONE when the iteration has finished; then
// g.ierr is 0 or the failing index l (1-based, tql2_tiled.hpp:138).
template <class T>
__host__ __device__ int ql_tql2(QLGen<T> &g, const DEView<T> v, const int n, Rec<T> *buf, const int cap,
                       const int max_sweep)
{
  const T tol = Num<T>::eps() * Num<T>::tolmul();
  int nrec = 0;
  if (g.pc == PC_DONE) return 0;
  if (g.pc == PC_ROT) goto resume_rot;
  g.ierr = 0;
  g.shift = T(0);
  g.tst1 = T(0);
  g.seg_pos = -1;
  if (n <= 1) goto finish;
  for (g.l = 0; g.l < n; g.l++) {
    {
      const T t = (fabs_t(v.D(g.l)) + fabs_t(v.E(g.l))) * tol;
      g.tst1 = fmax_t(g.tst1, t);
      int m = g.l;
      while (m < n && !(fabs_t(v.E(m)) <= g.tst1)) m++;
      if (m >= n) {  // only with NaN data
        g.ierr = g.l + 1;
        goto finish;
      }
      g.m = m;
    }
    if (g.m != g.l) {
      for (g.itr = 0; g.itr < max_sweep; g.itr++) {
        {  // explicit shift, tql2_tiled.hpp:64-80
          const int l = g.l;
          const T dl_old = v.D(l);
          T dl;
          tql2_shift(dl_old, v.D(l + 1), v.E(l), dl, g.dl1);
          v.D(l) = dl;
          v.D(l + 1) = g.dl1;
          g.delta = dl_old - dl;
          // d(j) -= delta for j >= l+2 (tql2_tiled.hpp:77-80): the sweep below
          // reads d(l+2..m) exactly once, before overwriting them, and
          // subtracts delta on that read; only d(m+1..n-1) are updated here.
          for (int j = g.m + 1; j < n; j++) v.D(j) -= g.delta;
          g.shift += g.delta;
        }
        g.c = T(1); g.c2 = T(1); g.c3 = T(1);
        g.s = T(0); g.s2 = T(0);
        g.p = (g.m >= g.l + 2) ? v.D(g.m) - g.delta : v.D(g.m);
        g.el1 = v.E(g.l + 1);
        g.ei = T(0);
        for (g.i = g.m - 1; g.i >= g.l; g.i--) {
          if (nrec + (g.seg_pos < 0 ? 2 : 1) > cap) {
            ql_close_seg(g, buf);
            g.pc = PC_ROT;
            return nrec;
          }
        resume_rot:
          if (g.seg_pos < 0) {
            g.seg_pos = nrec++;
            g.seg_cnt = 0;
            g.seg_i0 = g.i;
          }
          {  // QL step, tql2_tiled.hpp:94-115
            const int i = g.i;
            g.c3 = g.c2;
            g.c2 = g.c;
            g.s2 = g.s;
            const T ei = v.E(i);
            const T di = (i >= g.l + 2) ? v.D(i) - g.delta : v.D(i);
            T c, s, pn, ei1, di1;
            tql2_step(g.c, g.s, g.p, ei, di, c, s, pn, ei1, di1);
            g.p = pn;
            v.E(i + 1) = ei1;
            v.D(i + 1) = di1;
            g.c = c;
            g.s = s;
            g.ei = ei;
            Rec<T> rec;
            rec.c = c;
            rec.s = s;
            buf[nrec++] = rec;
            g.seg_cnt++;
          }
        }
        ql_close_seg(g, buf);
        {  // tql2_tiled.hpp:126-135
          T el, dl;
          tql2_close(g.c, g.s, g.s2, g.c3, g.el1, g.ei, g.dl1, el, dl);
          v.E(g.l) = el;
          v.D(g.l) = dl;
        }
        if (fabs_t(v.E(g.l)) <= g.tst1) break;
      }
      if (g.itr >= max_sweep) {
        g.ierr = g.l + 1;
        goto finish;
      }
    }
    v.D(g.l) += g.shift;
  }
finish:
  ql_close_seg(g, buf);
  g.pc = PC_DONE;
  return nrec;
}

template <class T>
__host__ __device__ int ql_imtql2(QLGen<T> &g, const DEView<T> v, const int n, Rec<T> *buf, const int cap,
                         const int max_sweep)
{
  const T tol = Num<T>::eps() * Num<T>::tolmul();
  int nrec = 0;
  if (g.pc == PC_DONE) return 0;
  if (g.pc == PC_ROT) goto resume_rot;
  g.ierr = 0;
  g.seg_pos = -1;
  if (n <= 1) goto finish;
  for (g.l = 0; g.l < n; g.l++) {
    for (g.itr = 0; g.itr <= max_sweep; g.itr++) {
      {  // deflation test, imtql2_tiled.hpp:56-61
        int m = n - 1;
        for (int mm = g.l; mm < n - 1; mm++) {
          const T t1 = (fabs_t(v.D(mm)) + fabs_t(v.D(mm + 1))) * tol;
          const T t2 = fabs_t(v.E(mm));
          if (!(t2 > t1)) {
            m = mm;
            break;
          }
        }
        g.m = m;
      }
      if (g.m == g.l) break;
      // Wilkinson-type shift, imtql2_tiled.hpp:67-75
      g.di1 = v.D(g.m);
      g.r = imtql2_shift(v.D(g.l), v.D(g.l + 1), v.E(g.l), g.di1);
      g.s = T(1);
      g.c = T(1);
      g.delta = T(0);
      for (g.i = g.m - 1; g.i >= g.l; g.i--) {
        if (nrec + (g.seg_pos < 0 ? 2 : 1) > cap) {
          ql_close_seg(g, buf);
          g.pc = PC_ROT;
          return nrec;
        }
      resume_rot:
        {  // imtql2_tiled.hpp:86-115
          const int i = g.i;
          const T ei = v.E(i);
          const T f = mul_rn(g.s, ei);
          T c, s, r;
          givens(g.r, f, c, s, r);
          if (r == T(0)) {
            g.r = T(0);
            break;
          }
          if (g.seg_pos < 0) {
            g.seg_pos = nrec++;
            g.seg_cnt = 0;
            g.seg_i0 = i;
          }
          const T dx1 = imtql2_step(c, s, g.c, ei, v.D(i), g.di1, g.delta, g.r);
          v.E(i + 1) = r;
          v.D(i + 1) = dx1;
          g.c = c;
          g.s = s;
          Rec<T> rec;
          rec.c = c;
          rec.s = s;
          buf[nrec++] = rec;
          g.seg_cnt++;
        }
      }
      ql_close_seg(g, buf);
      {
        const int j = (g.i + 1 > g.l) ? g.i + 1 : g.l;
        v.D(j) -= g.delta;
        v.E(j) = g.r;
        v.E(g.m) = T(0);
      }
    }
    if (g.itr > max_sweep) {
      g.ierr = g.l + 1;
      goto finish;
    }
  }
finish:
  ql_close_seg(g, buf);
  g.pc = PC_DONE;
  return nrec;
}

// ---------------------------------------------------------------------------
// Fast single-call forms used by phase 2: the whole iteration in one call
// with a fixed record capacity, no resume points, and the capacity checked
// once per sweep.  Same arithmetic as ql_tql2 / ql_imtql2 (identical
// rotations and eigenvalues).  Returns the record count, or -1 when the
// capacity would be exceeded (phase 3 then regenerates with the resumable
// form).  *ierr receives 0 or the failing 1-based index.
template <class T>
__host__ __device__ int ql_tql2_fast(T *__restrict__ d, T *__restrict__ e, const int st, const int n,
                                     Rec<T> *__restrict__ out, const int cap, const int max_sweep, int *ierr)
{
  const T tol = Num<T>::eps() * Num<T>::tolmul();
  int nrec = 0;
  *ierr = 0;
  if (n <= 1) return 0;
  T shift = T(0), tst1 = T(0);
  for (int l = 0; l < n; l++) {
    T *dl_p = d + l * st;
    T *el_p = e + l * st;
    tst1 = fmax_t(tst1, (fabs_t(*dl_p) + fabs_t(*el_p)) * tol);
    int m = l;
    {
      const T *ep = el_p;
      while (m < n && !(fabs_t(*ep) <= tst1)) {
        m++;
        ep += st;
      }
    }
    if (m >= n) {
      *ierr = l + 1;
      return nrec;
    }
    if (m != l) {
      const int len = m - l;
      int itr;
      for (itr = 0; itr < max_sweep; itr++) {
        if (nrec + 1 + len > cap) return -1;
        const T dl_old = *dl_p;
        T dl, dl1;
        tql2_shift(dl_old, dl_p[st], *el_p, dl, dl1);
        *dl_p = dl;
        dl_p[st] = dl1;
        const T delta = dl_old - dl;
        for (int j = m + 1; j < n; j++) d[j * st] -= delta;  // d(l+2..m) are shifted on read
        shift += delta;
        T c = T(1), c2 = T(1), c3 = T(1), s = T(0), s2 = T(0);
        T *dp = d + m * st;
        T *ep = e + (m - 1) * st;
        T p = (m >= l + 2) ? *dp - delta : *dp;
        const T el1 = el_p[st];
        T ei = T(0);
        Rec<T> *o = out + nrec + 1;
        // e(i), d(i) of the next step are loaded before this step's stores
        // of e(i+1), d(i+1) (distinct addresses)
        T ei_n = *ep, dsi_n = dp[-st];
        for (int i = m - 1; i >= l; i--) {
          c3 = c2;
          c2 = c;
          s2 = s;
          ei = ei_n;
          const T dsi = dsi_n;
          if (i > l) {
            ei_n = ep[-st];
            dsi_n = dp[-2 * st];
          }
          const T di = (i >= l + 2) ? dsi - delta : dsi;
          T cn, sn, pn, ei1, di1;
          tql2_step(c, s, p, ei, di, cn, sn, pn, ei1, di1);
          ep[st] = ei1;
          p = pn;
          *dp = di1;
          c = cn;
          s = sn;
          Rec<T> rec;
          rec.c = cn;
          rec.s = sn;
          *o++ = rec;
          dp -= st;
          ep -= st;
        }
        out[nrec] = make_hdr(m - 1, len, T(0));
        nrec += 1 + len;
        T eln, dln;
        tql2_close(c, s, s2, c3, el1, ei, dl1, eln, dln);
        *el_p = eln;
        *dl_p = dln;
        if (fabs_t(*el_p) <= tst1) break;
      }
      if (itr >= max_sweep) {
        *ierr = l + 1;
        return nrec;
      }
    }
    *dl_p += shift;
  }
  return nrec;
}

template <class T>
__host__ __device__ int ql_imtql2_fast(T *__restrict__ d, T *__restrict__ e, const int st, const int n,
                                       Rec<T> *__restrict__ out, const int cap, const int max_sweep, int *ierr)
{
  const T tol = Num<T>::eps() * Num<T>::tolmul();
  int nrec = 0;
  *ierr = 0;
  if (n <= 1) return 0;
  for (int l = 0; l < n; l++) {
    int itr;
    for (itr = 0; itr <= max_sweep; itr++) {
      int m = n - 1;
      for (int mm = l; mm < n - 1; mm++) {
        const T t1 = (fabs_t(d[mm * st]) + fabs_t(d[(mm + 1) * st])) * tol;
        if (!(fabs_t(e[mm * st]) > t1)) {
          m = mm;
          break;
        }
      }
      if (m == l) break;
      if (nrec + 1 + (m - l) > cap) return -1;
      T di1 = d[m * st];
      T r = imtql2_shift(d[l * st], d[(l + 1) * st], e[l * st], di1);
      T s = T(1), c = T(1), delta = T(0);
      Rec<T> *o = out + nrec + 1;
      int i;
      int cnt = 0;
      for (i = m - 1; i >= l; i--) {
        const T ei = e[i * st];
        const T f = mul_rn(s, ei);
        T cn, sn, rn;
        givens(r, f, cn, sn, rn);
        if (rn == T(0)) {
          r = T(0);
          break;
        }
        const T dx1 = imtql2_step(cn, sn, c, ei, d[i * st], di1, delta, r);
        e[(i + 1) * st] = rn;
        d[(i + 1) * st] = dx1;
        c = cn;
        s = sn;
        Rec<T> rec;
        rec.c = cn;
        rec.s = sn;
        *o++ = rec;
        cnt++;
      }
      if (cnt > 0) {
        out[nrec] = make_hdr(m - 1, cnt, T(0));
        nrec += 1 + cnt;
      }
      const int j = (i + 1 > l) ? i + 1 : l;
      d[j * st] -= delta;
      e[j * st] = r;
      e[m * st] = T(0);
    }
    if (itr > max_sweep) {
      *ierr = l + 1;
      return nrec;
    }
  }
  return nrec;
}

template <class T>
__host__ __device__ __forceinline__ int ql_run(int method, QLGen<T> &g, const DEView<T> v, const int n,
                                      Rec<T> *buf, const int cap, const int max_sweep)
{
  return method == QL_IMTQL2 ? ql_imtql2(g, v, n, buf, cap, max_sweep)
                             : ql_tql2(g, v, n, buf, cap, max_sweep);
}

}  // namespace eigb
