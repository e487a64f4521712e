"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``oracle/liboracle.so`` (the C restatement of the reference's
tred1 -> tql2/imtql2 -> hhtr2sy -> selection-sort path, see
``eigen_oracle_body.h``) and adds the FP64 LAPACK ``dsyev`` oracle from scipy
and the seeded synthetic matrix families used by the tests and the bench.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of
``bench.py`` import this module; the CUDA library never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_LIBS = {}

METHOD_TQL2, METHOD_IMTQL2, METHOD_JACOBI = 0, 1, 2


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib(fast=False):
    """The parity build (liboracle.so), or with fast=True the timed CPU
    baseline build (liboracle_fast.so, -O3 -march=native), compiled here
    for this machine's CPU on first use."""
    global _LIB
    if fast:
        if "fast" not in _LIBS:
            subprocess.check_call(["make", "-s", "-C", _HERE, "fast"])
            _LIBS["fast"] = _load(os.path.join(_HERE, "liboracle_fast.so"))
        return _LIBS["fast"]
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = _load(path)
    return _LIB


def _load(path):
    L = ctypes.CDLL(path)
    P = ctypes.c_void_p
    I = ctypes.c_int
    for sfx in ("_d", "_f"):
        getattr(L, "oracle_eigen_batch" + sfx).argtypes = [I, I, I, I, P, P, I, I, I, P, I]
        getattr(L, "oracle_eigen_batch" + sfx).restype = ctypes.c_long
        getattr(L, "oracle_check" + sfx).argtypes = [I, I, I, I, P, P, P, P, P, P]
        getattr(L, "oracle_set_mat" + sfx).argtypes = [P, I, I, I, I]
        getattr(L, "oracle_tred1" + sfx).argtypes = [I, I, P, P, P]
        getattr(L, "oracle_tql2" + sfx).argtypes = [I, I, P, P, P, I, P]
        getattr(L, "oracle_tql2" + sfx).restype = I
        getattr(L, "oracle_imtql2" + sfx).argtypes = [I, I, P, P, P, I, P]
        getattr(L, "oracle_imtql2" + sfx).restype = I
        getattr(L, "oracle_select_sort" + sfx).argtypes = [I, P, P]
    L.oracle_num_threads.restype = I
    return L


def _sfx(dtype):
    dtype = np.dtype(dtype)
    if dtype == np.float64:
        return "_d"
    if dtype == np.float32:
        return "_f"
    raise TypeError(dtype)


def _ptr(x):
    return ctypes.c_void_p(x.ctypes.data)


def eigen_batch(a, n, nm=None, method=METHOD_TQL2, sort=True, max_sweep=100, nthreads=0, fast=False):
    """Solve a batch in place on the CPU.

    ``a``: contiguous array of L column-major nm x n matrices (shape (L, n, nm)
    in C order, i.e. a[k, j, i] = a_k(i, j)).  Returns (w, info, rotations);
    ``a`` is overwritten with the eigenvectors, as the reference does.
    """
    assert a.flags.c_contiguous
    nm = n if nm is None else nm
    L = a.size // (nm * n)
    w = np.zeros((L, n), dtype=a.dtype)
    info = np.zeros(L, dtype=np.int32)
    f = getattr(lib(fast), "oracle_eigen_batch" + _sfx(a.dtype))
    rots = f(L, nm, n, n, _ptr(a), _ptr(w), method, int(bool(sort)), max_sweep, _ptr(info), nthreads)
    return w, info, rots


def check(a0, w, z, n, nm=None):
    """Residual/orthogonality gate of eigen_GPU_check.cu: (err1, err2, flags)."""
    nm = n if nm is None else nm
    L = a0.size // (nm * n)
    e1 = np.zeros(L)
    e2 = np.zeros(L)
    fl = np.zeros(L, dtype=np.int32)
    a0 = np.ascontiguousarray(a0)
    w = np.ascontiguousarray(w)
    z = np.ascontiguousarray(z)
    getattr(lib(), "oracle_check" + _sfx(a0.dtype))(L, nm, n, n, _ptr(a0), _ptr(w), _ptr(z),
                                                    _ptr(e1), _ptr(e2), _ptr(fl))
    return e1, e2, fl


def select_sort(d):
    """Reference DO_SORT selection sort on one eigenvalue vector: (sorted d, pos 0-based)."""
    d = np.array(d, copy=True)
    pos = np.zeros(d.size, dtype=np.int32)
    getattr(lib(), "oracle_select_sort" + _sfx(d.dtype))(d.size, _ptr(d), _ptr(pos))
    return d, pos - 1


REF_SYM_RAND, REF_LETKF, REF_FRANK = 0, 1, 2


def ref_matrices(L, n, kind, dtype=np.float64, nm=None, seed0=0):
    """The reference's own generators (main.cpp:63-195), matrix k seeded with k+seed0."""
    nm = n if nm is None else nm
    a = np.zeros((L, n, nm), dtype=dtype)
    f = getattr(lib(), "oracle_set_mat" + _sfx(dtype))
    for k in range(L):
        f(ctypes.c_void_p(a[k].ctypes.data), nm, n, kind, k + seed0)
    return a


# ---------------------------------------------------------------------------
# Seeded synthetic families of the benchmark configurations.  Arrays are
# (L, n, n) C-order holding column-major matrices; all are symmetric so the
# layout question only matters for the triangle that is read.

def sym_uniform(L, n, seed, dtype=np.float64):
    """A = (B + B^T)/2, B iid U[-1, 1]."""
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1.0, 1.0, size=(L, n, n))
    return np.ascontiguousarray(((b + b.transpose(0, 2, 1)) * 0.5).astype(dtype))


def letkf_like(L, n, seed, dtype=np.float64, k=None):
    """A = (k-1) I + Y^T Y with Y k x n iid N(0,1)/sqrt(n), k = n."""
    k = n if k is None else k
    rng = np.random.default_rng(seed)
    y = rng.standard_normal(size=(L, k, n)) / np.sqrt(n)
    a = np.einsum("lki,lkj->lij", y, y) + (k - 1) * np.eye(n)[None]
    return np.ascontiguousarray(a.astype(dtype))


def _random_orthogonal(rng, L, n):
    g = rng.standard_normal(size=(L, n, n))
    q, r = np.linalg.qr(g)
    return q * np.sign(np.diagonal(r, axis1=1, axis2=2))[:, None, :]


def logspaced_spectrum(L, n, seed, dtype=np.float64, lo=1.0, hi=1e6):
    """A = Q diag(lambda) Q^T, lambda log-spaced in [lo, hi] with random signs."""
    rng = np.random.default_rng(seed)
    q = _random_orthogonal(rng, L, n)
    lam = np.logspace(np.log10(lo), np.log10(hi), n)[None, :] * rng.choice([-1.0, 1.0], size=(L, n))
    a = np.einsum("lij,lj,lkj->lik", q, lam, q)
    a = 0.5 * (a + a.transpose(0, 2, 1))
    return np.ascontiguousarray(a.astype(dtype))


def clustered_spectrum(L, n, seed, dtype=np.float64, cluster=8, sep=1e-8, gap=1e-1):
    """Clusters of `cluster` eigenvalues `sep` apart inside gaps of `gap`."""
    rng = np.random.default_rng(seed)
    q = _random_orthogonal(rng, L, n)
    idx = np.arange(n)
    lam = (idx // cluster) * gap + (idx % cluster) * sep + 1.0
    a = np.einsum("lij,j,lkj->lik", q, lam, q)
    a = 0.5 * (a + a.transpose(0, 2, 1))
    return np.ascontiguousarray(a.astype(dtype))


THETA_DIM = 4


def theta_family_basis(n=64, family_seed=2024):
    """The fixed members of the parameterised family A(theta) = A0 +
    sum_j theta_j E_j (j = 1..4): A0 = (G + G^T)/sqrt(2n), G iid N(0,1)
    (a Wigner matrix, spectrum close to [-2, 2]); E_j = (H_j + H_j^T)
    scaled to unit Frobenius norm, H_j iid N(0,1).  Returns (A0, E) with
    E of shape (4, n, n), all float64 and symmetric."""
    rng = np.random.default_rng(family_seed)
    g = rng.standard_normal((n, n))
    a0 = (g + g.T) / np.sqrt(2.0 * n)
    e = np.empty((THETA_DIM, n, n))
    for j in range(THETA_DIM):
        h = rng.standard_normal((n, n))
        h = h + h.T
        e[j] = h / np.linalg.norm(h)
    return a0, e


def theta_family(L, n=64, seed=0, dtype=np.float32, family_seed=2024, return_theta=False):
    """L matrices A(theta) = A0 + sum_j theta_j E_j, theta iid U[-0.1, 0.1]^4
    (A0, E_j from theta_family_basis).  (L, n, n) C-order holding the
    symmetric matrices; with return_theta also the (L, 4) parameters."""
    a0, e = theta_family_basis(n, family_seed)
    rng = np.random.default_rng(seed)
    th = rng.uniform(-0.1, 0.1, size=(L, THETA_DIM))
    a = a0[None] + np.einsum("lj,jik->lik", th, e)
    a = np.ascontiguousarray(a.astype(dtype))
    return (a, th) if return_theta else a


def frank(L, n, dtype=np.float64):
    i = np.arange(1, n + 1)
    a = np.minimum.outer(i, i).astype(dtype)
    return np.ascontiguousarray(np.broadcast_to(a, (L, n, n)).copy())


def frank_eigenvalues(n):
    """Analytic eigenvalues of the Frank matrix min(i,j), ascending
    (eigen_GPU_check.cu:17-32)."""
    i = np.arange(1, n + 1)
    theta = (2 * (n + 1 - i) - 1) * np.pi / (2 * n + 1)
    return np.sort(1.0 / (2.0 * (1.0 - np.cos(theta))))


def lapack_eigh(a, n, dtype=None):
    """Per-matrix FP64 LAPACK dsyev (upper triangle of the column-major
    matrix); returns (w ascending, V) in float64."""
    from scipy.linalg import lapack
    a = np.asarray(a, dtype=np.float64).reshape(-1, n, n)
    L = a.shape[0]
    w = np.zeros((L, n))
    v = np.zeros((L, n, n))
    for k in range(L):
        # a[k] holds the column-major matrix, so its C-order view is A^T and the
        # Fortran-order matrix is a[k].T; dsyev reads uplo='U' of that.
        mk = np.asfortranarray(a[k].T)
        wk, vk, inf = lapack.dsyev(mk, compute_v=1, lower=0)
        assert inf == 0
        w[k] = wk
        v[k] = vk.T  # back to (col, row) storage: v[k][j] = eigenvector j
    return w, v


def residuals(a0, w, z, n):
    """Scale-relative FP64 residuals: max|AV - V diag(w)| / ||A||_2-ish and
    ||V^T V - I||_max, per matrix.  a0 uses the upper triangle."""
    a0 = np.asarray(a0, dtype=np.float64).reshape(-1, n, n)
    z = np.asarray(z, dtype=np.float64).reshape(-1, n, n)
    w = np.asarray(w, dtype=np.float64).reshape(-1, n)
    A = np.triu(np.transpose(a0, (0, 2, 1)))            # row-major upper
    A = A + np.transpose(np.triu(A, 1), (0, 2, 1))
    V = np.transpose(z, (0, 2, 1))                      # V[:, i, j] = v_j(i)
    R = A @ V - V * w[:, None, :]
    anorm = np.maximum(np.abs(w).max(axis=1), np.finfo(np.float64).tiny)
    res = np.linalg.norm(R, axis=(1, 2)) / anorm
    orth = np.linalg.norm(np.transpose(V, (0, 2, 1)) @ V - np.eye(n)[None], axis=(1, 2))
    return res, orth


def symdmt(v, d, n):
    """z = V diag(d) V^T per matrix, the reference prototype symdmt.cu:5-80
    (z(i,j) = sum_k a(i,k) d(k) a(j,k)), in FP64.  v: (L, n, nm) column-major
    eigenvectors (v[k, j, i] = V_k(i, j)), d: (L, n).  Returns (L, n, n)
    column-major (z[k, j, i] = Z_k(i, j))."""
    v = np.asarray(v, dtype=np.float64)[:, :n, :n]       # [k, col j, row i]
    d = np.asarray(d, dtype=np.float64).reshape(-1, n)
    V = np.transpose(v, (0, 2, 1))                        # V[k, i, j]
    Z = (V * d[:, None, :]) @ np.transpose(V, (0, 2, 1))
    return np.transpose(Z, (0, 2, 1))
