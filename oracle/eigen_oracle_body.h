/*
 * Type-generic body of the CPU oracle.  Included twice by eigen_oracle.c,
 * once with T=double / SFX(x)=x##_d and once with T=float / SFX(x)=x##_f.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a scalar restatement of the
 * reference's batched symmetric eigensolver (EigenG-Batched) used as the
 * checker for the CUDA library; nothing in the product links it.
 *
 * Matrices are column-major, a(i,j) = a[(i-1) + (j-1)*nm] (1-based macros
 * below follow the reference's Fortran-style indexing so each loop can be
 * compared line by line with the file:line it cites).
 */

#define A_(i, j) a[((i) - 1) + (size_t)((j) - 1) * nm]
#define Z_(i, j) z[((i) - 1) + (size_t)((j) - 1) * nm]
#define D_(i) d[(i) - 1]
#define E_(i) e[(i) - 1]
#define W_(i) w[(i) - 1]
#define P_(i) pos[(i) - 1]

/* Square root used inside the hypot correction.  The reference seeds the
 * FP64 correction with a single-precision square root
 * (misc_gpu.hpp:402-405 FastSqrt(double) = (double)sqrtf((float)x)); its
 * FP32 seed is sqrt.approx (misc_gpu.hpp:390-400), restated here with the
 * correctly rounded sqrtf. */
static inline T SFX(o_fastsqrt)(T x) { return (T)sqrtf((float)x); }

static inline T SFX(o_flip0to1)(T x) { return (x == (T)0) ? (T)1 : x; }

/* Fortran SIGN(x, y) as copysign, misc_gpu.hpp:441-469. */
static inline T SFX(o_sign)(T x, T y) { return (T)copysign((double)x, (double)y); }

/* hypot(x, 1) with one fma correction step (Borges 2020, ACM TOMS 1014),
 * as in misc_gpu.hpp:514-530. */
static T SFX(o_pythag1)(T x)
{
  const T one = (T)1;
  const T x_sq = x * x;
  const T sigma = x_sq + one;
  const T h = SFX(o_fastsqrt)(sigma);
  const T sigma_e = (sigma - x_sq) - one;
  const T tau = (T)fma(x, x, -x_sq) - sigma_e + (T)fma(-h, h, sigma);
  return (T)fma(tau / SFX(o_flip0to1)(h), (T)0.5, h);
}

/* hypot(x, y), misc_gpu.hpp:533-548. */
static T SFX(o_pythag)(T x, T y)
{
  const T x_sq = x * x;
  const T y_sq = y * y;
  const T sigma = x_sq + y_sq;
  const T h = SFX(o_fastsqrt)(sigma);
  const T sigma_e = (sigma - x_sq) - y_sq;
  const T tau = (T)fma(y, y, -y_sq) + (T)fma(x, x, -x_sq) - sigma_e + (T)fma(-h, h, sigma);
  return (T)fma(tau / SFX(o_flip0to1)(h), (T)0.5, h);
}

static inline T SFX(o_tol)(void) { return SFX(o_eps)() * (T)(sizeof(T) == 8 ? 512 : 16); }

/* Householder reduction of the upper triangle to tridiagonal form, the
 * unblocked algorithm of tred1_tiled.hpp:3-222 (used by the reference for
 * n<=32; its blocked n>32 variant hhsy2tr.hpp:3-326 computes the same
 * reflectors up to rounding).
 *  in : upper triangle of a (the strictly lower part is never read)
 *  out: d(1:n) diagonal, e(1:n) off-diagonal (e(k) couples k,k+1; e(n)=0),
 *       reflector i (i=2..n) in a(1:i-1, i) with its pivot entry replaced
 *       by ul = u_l - anorm (tred1_tiled.hpp:55-68), and a(i,i) = e(i-1),
 *       a(1,1) = 0 (tred1_tiled.hpp:207-212). */
void SFX(oracle_tred1)(int nm, int n, T *a, T *d, T *e)
{
  if (n <= 0) return;
  if (n == 1) { D_(1) = A_(1, 1); E_(1) = 0; A_(1, 1) = 0; return; }
  T *u = (T *)calloc((size_t)n + 1, sizeof(T));
  T *v = (T *)calloc((size_t)n + 1, sizeof(T));
  T *el = (T *)calloc((size_t)n + 1, sizeof(T)); /* el(j): e produced when l == j */
  for (int i = n; i >= 2; i--) {
    const int l = i - 1;
    T anorm = 0;
    for (int k = 1; k <= l; k++) { u[k] = A_(k, i); anorm += u[k] * u[k]; }
    const T ul0 = u[l];
    anorm = -SFX(o_sign)((T)sqrt((double)anorm), ul0);
    const T ul = ul0 - anorm;
    const T beta = (T)1 / SFX(o_flip0to1)(ul * anorm);
    el[l] = anorm;
    u[l] = ul;
    /* v = A(1:l,1:l) u on the upper triangle, tred1_tiled.hpp:76-164 */
    for (int j = 1; j <= l; j++) {
      T s = 0;
      for (int k = 1; k <= l; k++) s += (j <= k ? A_(j, k) : A_(k, j)) * u[k];
      v[j] = s;
    }
    A_(l, i) = ul; /* reflector stored back, tred1_tiled.hpp:161-163 */
    /* v := beta*v + (beta/2)(u'beta v) u, tred1_tiled.hpp:174-181 */
    T alpha = 0;
    for (int j = 1; j <= l; j++) { v[j] *= beta; alpha += v[j] * u[j]; }
    alpha *= beta * (T)0.5;
    for (int j = 1; j <= l; j++) v[j] += alpha * u[j];
    /* A(j,k) += u_k v_j + v_k u_j for j <= k <= l, tred1_tiled.hpp:184-203 */
    for (int k = 1; k <= l; k++)
      for (int j = 1; j <= k; j++)
        A_(j, k) = (A_(j, k) + u[k] * v[j]) + v[k] * u[j];
  }
  /* tred1_tiled.hpp:207-212 */
  for (int my = 1; my <= n; my++) {
    const int j = (my < n) ? my + 1 : 1;
    D_(j) = A_(j, j);
    const T ev = (my < n) ? el[my] : (T)0;
    E_(my) = ev;
    A_(j, j) = ev;
  }
  free(u); free(v); free(el);
}

/* Selection sort of DO_SORT, tql2_tiled.hpp:149-176 (identical in tql2.hpp,
 * imtql2*.hpp): for each l, the FIRST strict minimum of d(l:n) is swapped
 * into place and pos() records the original index. */
void SFX(oracle_select_sort)(int n, T *d, int *pos)
{
  for (int i = 1; i <= n; i++) P_(i) = i;
  for (int i = 2; i <= n; i++) {
    const int l = i - 1;
    T dl = D_(l);
    int il = l;
    for (int j = i; j <= n; j++) {
      const T dj = D_(j);
      if (dl > dj) { dl = dj; il = j; }
    }
    if (il != l) {
      const int p = P_(l); P_(l) = P_(il); P_(il) = p;
      D_(il) = D_(l); D_(l) = dl;
    }
  }
}

/* Explicit-shift QL with eigenvector accumulation, tql2_tiled.hpp:3-192
 * (the reference default, USE_IMTQL 0, eigen_GPU_batch.cu:3).  z is set to
 * the identity first.  Returns 0, or l when the sweep limit is hit
 * (tql2_tiled.hpp:138).  *nrot receives the number of plane rotations. */
int SFX(oracle_tql2)(int nm, int n, T *d, T *e, T *z, int max_sweep, long *nrot)
{
  long rots = 0;
  int ierror = 0;
  for (int j = 1; j <= n; j++)
    for (int k = 1; k <= n; k++) Z_(k, j) = (k == j) ? (T)1 : (T)0;
  if (n <= 1) { if (nrot) *nrot = 0; return 0; }
  const T tol = SFX(o_tol)();
  T shift = 0, tst1 = 0;
  for (int l = 1; l <= n; l++) {
    /* tql2_tiled.hpp:51-55 */
    {
      const T t = (T)(fabs((double)D_(l)) + fabs((double)E_(l))) * tol;
      tst1 = (T)fmax((double)tst1, (double)t);
    }
    int m;
    for (m = l; m <= n; m++)
      if (fabs((double)E_(m)) <= tst1) break;
    if (m > n) { ierror = l; break; } /* only reachable with NaN data */
    if (m != l) {
      int itr;
      for (itr = 0; itr < max_sweep; itr++) {
        /* shift, tql2_tiled.hpp:64-80 */
        T dl1, delta;
        {
          const T dl_old = D_(l);
          const T elv = E_(l);
          const T p = (D_(l + 1) - dl_old) / (elv + elv);
          const T r = SFX(o_pythag1)(p);
          const T psr = p + SFX(o_sign)(r, p);
          const T dl = elv / psr;
          dl1 = elv * psr;
          D_(l) = dl; D_(l + 1) = dl1;
          delta = dl_old - dl;
        }
        for (int i = l + 2; i <= n; i++) D_(i) -= delta;
        shift += delta;
        /* QL sweep, tql2_tiled.hpp:84-124 */
        T c = 1, c2 = 1, c3 = 1, s = 0, s2 = 0;
        T p = D_(m);
        const T el1 = E_(l + 1);
        T ei = 0;
        for (int i = m - 1; i >= l; i--) {
          c3 = c2; c2 = c; s2 = s;
          ei = E_(i);
          const T di = D_(i);
          const T g = c * ei;
          const T h = c * p;
          const T r = SFX(o_pythag)(p, ei);
          const T ei1 = s * r;
          s = ei / r;
          c = p / r;
          p = c * di - s * g;
          const T di1 = h + s * (c * g + s * di);
          E_(i + 1) = ei1; D_(i + 1) = di1;
          for (int k = 1; k <= n; k++) {
            const T h0 = Z_(k, i), h1 = Z_(k, i + 1);
            Z_(k, i + 1) = s * h0 + c * h1;
            Z_(k, i) = c * h0 - s * h1;
          }
          rots++;
        }
        /* tql2_tiled.hpp:126-135 */
        {
          const T r = (-s * s2 * c3 * el1 * ei) / dl1;
          E_(l) = s * r;
          D_(l) = c * r;
        }
        if (fabs((double)E_(l)) <= tst1) break;
      }
      if (itr >= max_sweep) { ierror = l; break; }
    }
    D_(l) += shift;
  }
  if (nrot) *nrot = rots;
  return ierror;
}

/* Implicit-shift QL with eigenvector accumulation, imtql2_tiled.hpp:3-176
 * (USE_IMTQL 1).  Returns 0, or l when more than max_sweep+1 sweeps were
 * needed (imtql2_tiled.hpp:126). */
int SFX(oracle_imtql2)(int nm, int n, T *d, T *e, T *z, int max_sweep, long *nrot)
{
  long rots = 0;
  int ierror = 0;
  for (int j = 1; j <= n; j++)
    for (int k = 1; k <= n; k++) Z_(k, j) = (k == j) ? (T)1 : (T)0;
  if (n <= 1) { if (nrot) *nrot = 0; return 0; }
  const T tol = SFX(o_tol)();
  for (int l = 1; l <= n; l++) {
    int itr;
    for (itr = 0; itr <= max_sweep; itr++) {
      /* deflation test, imtql2_tiled.hpp:56-61 */
      int m = n;
      for (int mm = l; mm <= n - 1; mm++) {
        const T t1 = (T)(fabs((double)D_(mm)) + fabs((double)D_(mm + 1))) * tol;
        const T t2 = (T)fabs((double)E_(mm));
        if (!(t2 > t1)) { m = mm; break; }
      }
      if (m == l) break;
      /* Wilkinson-type shift, imtql2_tiled.hpp:67-75 */
      T di1, r;
      {
        const T dl = D_(l), dl1 = D_(l + 1), elv = E_(l);
        const T f = (dl1 - dl) / (elv + elv);
        const T g = SFX(o_pythag1)(f);
        di1 = D_(m);
        r = (di1 - dl) + elv / (f + SFX(o_sign)(g, f));
      }
      T s = 1, c = 1, delta = 0;
      int i;
      for (i = m - 1; i >= l; i--) {
        const T ei = E_(i);
        const T f = s * ei;
        const T g = r;
        r = SFX(o_pythag)(f, g);
        if (r == (T)0) break;
        const T b = c * ei;
        s = f / r;
        c = g / r;
        const T dix = di1 - delta;
        di1 = D_(i);
        const T q = (di1 - dix) * s + (T)2 * c * b;
        const T dx1 = (T)fma(s, q, dix);
        delta = dx1 - dix;
        E_(i + 1) = r; D_(i + 1) = dx1;
        r = c * q - b;
        for (int k = 1; k <= n; k++) {
          const T h0 = Z_(k, i), h1 = Z_(k, i + 1);
          Z_(k, i + 1) = s * h0 + c * h1;
          Z_(k, i) = c * h0 - s * h1;
        }
        rots++;
      }
      {
        const int j = (i + 1 > l) ? i + 1 : l;
        D_(j) -= delta;
        E_(j) = r;
        E_(m) = 0;
      }
    }
    if (itr > max_sweep) { ierror = l; break; }
  }
  if (nrot) *nrot = rots;
  return ierror;
}

/* Householder back-transformation Z := H(n) ... H(2) Z, the unblocked form
 * of hhtr2sy_tiled.hpp:47-69 (the blocked part :71-211 aggregates the same
 * reflectors, Joffrain et al. ACM TOMS 32(2) 2006, and equals this up to
 * rounding).  Reflector i lives in a(1:i-1,i); its scale is
 * 1/flip0to1(a(i,i)*a(i-1,i)) (hhtr2sy_tiled.hpp:58). */
void SFX(oracle_hhtr2sy)(int nm, int n, const T *a, T *z)
{
  for (int i = 2; i <= n; i++) {
    const int l = i - 1;
    const T scale = (T)1 / SFX(o_flip0to1)(A_(i, i) * A_(l, i));
    for (int j = 1; j <= n; j++) {
      T s = 0;
      for (int k = 1; k <= l; k++) s += A_(k, i) * Z_(k, j);
      const T t = s * scale;
      for (int k = 1; k <= l; k++) Z_(k, j) += t * A_(k, i);
    }
  }
}

/* Cyclic-by-column classical Jacobi, jac_tiled.hpp:3-152, on the full
 * symmetric matrix.  The reference loops until a pass makes no rotation
 * (jac_tiled.hpp:34,140) with no limit; here at most max_pass passes run
 * and the return value is 1 when that limit stopped the iteration.
 * On exit w holds the (unsorted) eigenvalues and a the eigenvectors. */
int SFX(oracle_jacobi)(int nm, int n, T *a, T *w, T *z, int max_pass, long *nrot)
{
  long rots = 0;
  for (int j = 1; j <= n; j++)
    for (int k = 1; k <= n; k++) Z_(k, j) = (k == j) ? (T)1 : (T)0;
  for (int k = 1; k <= n; k++) { W_(k) = A_(k, k); A_(k, k) = 0; }
  const T tol = (T)(sizeof(T) == 4 ? 1e-10 : 1e-20);
  int converged = 0;
  for (int pass = 0; pass < max_pass; pass++) {
    int stable = 1;
    for (int i0 = 1; i0 <= n; i0++) {
      /* two arg-max searches with lower-index tie break, jac_tiled.hpp:38-64 */
      int ii = 1; T x = (T)fabs((double)A_(1, i0));
      for (int k = 2; k <= n; k++) { T t = (T)fabs((double)A_(k, i0)); if (t > x) { x = t; ii = k; } }
      int jj = 1; T y = (T)fabs((double)A_(1, ii));
      for (int k = 2; k <= n; k++) { T t = (T)fabs((double)A_(k, ii)); if (t > y) { y = t; jj = k; } }
      int i = ii, j = jj;
      if (i > j) { int t = i; i = j; j = t; }
      if (i == j) continue;
      T aij = A_(j, i);
      const T aii = W_(i), ajj = W_(j);
      if (fabs((double)aij) < (fabs((double)aii) + fabs((double)ajj)) * tol) continue;
      /* rotation, jac_tiled.hpp:79-95 */
      const T alpha = 2 * aij;
      const T beta = ajj - aii;
      const T t = alpha / (beta + SFX(o_sign)(SFX(o_pythag)(alpha, beta), beta));
      const T c = (T)1 / SFX(o_pythag1)(t);
      const T s = c * t;
      const T cc = c * c, ss = s * s, cs = -(c * s);
      aij = ((c - s) * (c + s) * aij) + cs * beta;
      const T wi = ((cc * aii) + ss * ajj) + cs * alpha;
      const T wj = (aii + ajj) - wi;
      W_(i) = wi; W_(j) = wj;
      /* jac_tiled.hpp:97-136 */
      for (int k = 1; k <= n; k++) {
        if (k == i || k == j) continue;
        const T aki = A_(k, i), akj = A_(k, j);
        const T bki = c * aki - s * akj;
        const T bkj = s * aki + c * akj;
        A_(i, k) = bki; A_(j, k) = bkj; A_(k, i) = bki; A_(k, j) = bkj;
      }
      A_(i, j) = aij; A_(j, i) = aij;
      for (int k = 1; k <= n; k++) {
        const T zki = Z_(k, i), zkj = Z_(k, j);
        Z_(k, i) = c * zki - s * zkj;
        Z_(k, j) = s * zki + c * zkj;
      }
      rots++;
      stable = 0;
    }
    if (stable) { converged = 1; break; }
  }
  for (int k = 1; k <= n; k++)
    for (int j = 1; j <= n; j++) A_(j, k) = Z_(j, k);
  if (nrot) *nrot = rots;
  return converged ? 0 : 1;
}

/* One matrix through the whole path.  method 0 = tql2 (reference default),
 * 1 = imtql2, 2 = Jacobi.  Mirrors eigen_GPU_batch_tiled_ /
 * eigen_GPU_batch_ (eigen_GPU_batch.cu:56-245) plus the n==1 kernel
 * (eigen_GPU_batch.cu:36-54).  On QL failure the eigenvectors are still
 * back-transformed (unsorted) and the failing index is returned. */
int SFX(oracle_eigen_one)(int nm, int n, T *a, T *w, T *z, int method, int do_sort,
                          int max_sweep, long *nrot)
{
  if (nrot) *nrot = 0;
  if (n == 1) { W_(1) = A_(1, 1); A_(1, 1) = 1; return 0; }
  if (method == 2) {
    /* the Jacobi path reads the full matrix: fill it from the upper triangle */
    for (int j = 1; j <= n; j++)
      for (int k = j + 1; k <= n; k++) A_(k, j) = A_(j, k);
    int info = SFX(oracle_jacobi)(nm, n, a, w, z, max_sweep, nrot);
    if (do_sort) {
      int *pos = (int *)malloc(sizeof(int) * (size_t)n);
      T *tmp = (T *)malloc(sizeof(T) * (size_t)n * (size_t)n);
      SFX(oracle_select_sort)(n, w, pos);
      for (int j = 1; j <= n; j++)
        for (int k = 1; k <= n; k++) tmp[(k - 1) + (size_t)(j - 1) * n] = A_(k, P_(j));
      for (int j = 1; j <= n; j++)
        for (int k = 1; k <= n; k++) A_(k, j) = tmp[(k - 1) + (size_t)(j - 1) * n];
      free(pos); free(tmp);
    }
    return info;
  }
  T *d = w;
  T *e = (T *)malloc(sizeof(T) * (size_t)n);
  int *pos = (int *)malloc(sizeof(int) * (size_t)n);
  SFX(oracle_tred1)(nm, n, a, d, e);
  int ierr = (method == 1) ? SFX(oracle_imtql2)(nm, n, d, e, z, max_sweep, nrot)
                           : SFX(oracle_tql2)(nm, n, d, e, z, max_sweep, nrot);
  const int sorted = do_sort && ierr == 0;
  if (sorted) SFX(oracle_select_sort)(n, d, pos);
  SFX(oracle_hhtr2sy)(nm, n, a, z);
  /* permuted copy, hhtr2sy_tiled.hpp:214-221 */
  for (int i = 1; i <= n; i++) {
    const int col = sorted ? P_(i) : i;
    for (int k = 1; k <= n; k++) A_(k, i) = Z_(k, col);
  }
  free(e); free(pos);
  return ierr;
}

/* Batched driver with OpenMP over matrices (the EISPACK-style CPU path).
 * Matrix k at a + k*nm*n, eigenvalues at w + k*n (eigen_GPU_batch.cu:89,133).
 * info[k] = 0 or the failing QL index.  Returns the total rotation count. */
long SFX(oracle_eigen_batch)(int L, int nm, int n, int m, T *a, T *w, int method, int do_sort,
                             int max_sweep, int *info, int nthreads)
{
  (void)m;
  long total = 0;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads) reduction(+ : total)
  {
    T *z = (T *)malloc(sizeof(T) * (size_t)nm * (size_t)n);
#pragma omp for schedule(dynamic, 4)
    for (long k = 0; k < L; k++) {
      long r = 0;
      const int st = SFX(oracle_eigen_one)(nm, n, a + (size_t)k * nm * n, w + (size_t)k * n, z,
                                           method, do_sort, max_sweep, &r);
      if (info) info[k] = st;
      total += r;
    }
    free(z);
  }
  return total;
}

/* Residual and orthogonality gate of eigen_GPU_check.cu:4-88, in FP64.
 * a0 is the input matrix (upper triangle used, symmetric completion), w the
 * eigenvalues and z the eigenvectors.  err1 = ||A Z - Z D||_F,
 * err2 = ||Z'Z - I||_F with off-diagonal terms counted twice
 * (eigen_GPU_check.cu:54-59).  flags bit0: err1 > Dmax*TOL, bit1: err2 >
 * n*TOL with TOL of eigen_GPU_check.cu:71. */
void SFX(oracle_check)(int L, int nm, int n, int m, const T *a0, const T *w, const T *z,
                       double *err1, double *err2, int *flags)
{
#pragma omp parallel for schedule(dynamic, 4)
  for (long id = 0; id < L; id++) {
    const T *a = a0 + (size_t)id * nm * n;
    const T *zz = z + (size_t)id * nm * n;
    const T *d = w + (size_t)id * n;
    double e1 = 0, e2 = 0;
    for (int i = 1; i <= m; i++) {
      for (int k = 1; k <= n; k++) {
        double ek = 0;
        for (int j = 1; j <= n; j++) {
          const double akj = (k <= j) ? (double)a[(k - 1) + (size_t)(j - 1) * nm]
                                      : (double)a[(j - 1) + (size_t)(k - 1) * nm];
          ek += akj * (double)zz[(j - 1) + (size_t)(i - 1) * nm];
        }
        const double r = ek - (double)d[i - 1] * (double)zz[(k - 1) + (size_t)(i - 1) * nm];
        e1 += r * r;
      }
    }
    for (int i = 1; i <= m; i++) {
      for (int j = i; j <= m; j++) {
        double r = 0;
        for (int k = 1; k <= n; k++)
          r += (double)zz[(k - 1) + (size_t)(i - 1) * nm] * (double)zz[(k - 1) + (size_t)(j - 1) * nm];
        r -= (i == j) ? 1.0 : 0.0;
        e2 += ((i == j) ? 1.0 : 2.0) * r * r;
      }
    }
    e1 = sqrt(e1); e2 = sqrt(e2);
    const double dmax = fmax(fabs((double)d[0]), fabs((double)d[n - 1]));
    const double EPS = 1.0 / 4503599627370496.0; /* 2^-52 */
    const double eps = 1.0 / 8388608.0;          /* 2^-23 */
    const double TOL = (sizeof(T) == 8 ? EPS * (2 * 512 - 1) : eps * (2 * 16 - 1)) * sqrt((double)(n + 16));
    int f = 0;
    if (e1 > dmax * TOL) f |= 1;
    if (e2 > n * TOL) f |= 2;
    if (err1) err1[id] = e1;
    if (err2) err2[id] = e2;
    if (flags) flags[id] = f;
  }
}

/* The reference's test-matrix generators, main.cpp:63-195.  type 0 =
 * MATRIX_SYM_RAND (rand_r stream, uniform [-1,1]), 1 = MATRIX_LETKF,
 * 2 = MATRIX_FRANK (a(i,j) = min(i,j)).  Both triangles are written. */
void SFX(oracle_set_mat)(T *a, int nm, int n, int type, int seed_)
{
  unsigned int seed = (unsigned int)seed_;
  if (type == 1) {
    T *w = (T *)malloc(sizeof(T) * (size_t)n);
    const T eps = SFX(o_eps)();
    for (int i = 1; i <= n; i++) {
      const T R = 16 - 1;
      const T rr = (T)((double)rand_r(&seed) / RAND_MAX);
      const T delta = (T)(R * (2 * rr - 1.) * eps);
      const T DELTA = (T)(1.0 + delta);
      w[i - 1] = (T)(n - 1) * DELTA;
    }
    for (int i = 1; i <= 2; i++) {
      const int j = rand_r(&seed) % n;
      w[j] += (T)((double)rand_r(&seed) / RAND_MAX) * n;
    }
    T scale = 0;
    for (int i = 1; i <= n; i++) scale = (T)fmax((double)scale, fabs((double)w[i - 1]));
    scale = (T)fmax((double)scale, 1.);
    for (int i = 1; i <= n; i++) w[i - 1] /= scale;
    T *ht = (T *)malloc(sizeof(T) * (size_t)n);
    for (int i = 1; i <= n; i++) ht[i - 1] = (T)sqrt((double)i);
    T *hi = (T *)malloc(sizeof(T) * (size_t)n);
    T *hj = (T *)malloc(sizeof(T) * (size_t)n);
    /* Helmert-type orthogonal basis rows, main.cpp:104-146 */
    for (int i = 1; i <= n; i++) {
      if (i == 1) { for (int k = 1; k <= n; k++) hi[k - 1] = (T)(1. / ht[n - 1]); }
      else {
        const T s = (T)(i - 1); const T h = ht[i - 2] * ht[i - 1];
        for (int k = 1; k <= i - 1; k++) hi[k - 1] = (T)(1. / h);
        hi[i - 1] = -s / h;
        for (int k = i + 1; k <= n; k++) hi[k - 1] = 0;
      }
      for (int j = 1; j <= n; j++) {
        if (j == 1) { for (int k = 1; k <= n; k++) hj[k - 1] = (T)(1. / ht[n - 1]); }
        else {
          const T s = (T)(j - 1); const T h = ht[j - 2] * ht[j - 1];
          for (int k = 1; k <= j - 1; k++) hj[k - 1] = (T)(1. / h);
          hj[j - 1] = -s / h;
          for (int k = j + 1; k <= n; k++) hj[k - 1] = 0;
        }
        T t = 0;
        for (int k = 1; k <= n; k++) t += w[k - 1] * (hi[k - 1] * hj[k - 1]);
        a[(j - 1) + (size_t)(i - 1) * nm] = t;
      }
    }
    for (int i = 1; i <= n; i++)
      for (int j = 1; j <= n; j++) a[(j - 1) + (size_t)(i - 1) * nm] *= scale;
    free(w); free(ht); free(hi); free(hj);
    return;
  }
  for (int i = 0; i < n; i++) {
    for (int j = 0; j <= i; j++) {
      T x = 0;
      if (type == 0) {
        const T t = (T)((double)rand_r(&seed) / RAND_MAX);
        x = 2 * t - (T)1.0;
      } else if (type == 2) {
        x = (T)((j + 1 < i + 1) ? j + 1 : i + 1);
      }
      a[i + (size_t)nm * j] = x;
      a[j + (size_t)nm * i] = x;
    }
  }
}

#undef A_
#undef Z_
#undef D_
#undef E_
#undef W_
#undef P_
