"""CPU unit tests of the library's own device code compiled for the host:
the phase-2 QL rotation generator (eigb_ql.cuh) and the phase-1 team code
(eigb_tridiag.cuh, run by one std::thread per GPU thread with std::barrier
for the CTA barrier).  They check the algorithms against the oracle without
a GPU; the -m gpu tests check the compiled kernels."""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "tests", "host")
NVCC = "/usr/local/cuda/bin/nvcc"


@pytest.fixture(scope="module")
def hostlibs():
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    td = tempfile.mkdtemp(prefix="eigb_host_")
    libs = {}
    for name in ("ql_host", "tridiag_host", "apply_host"):
        out = os.path.join(td, f"lib{name}.so")
        subprocess.check_call([NVCC, "-O2", "-std=c++20", "-Xcompiler", "-fPIC", "-shared",
                               "-Wno-deprecated-gpu-targets", "-diag-suppress", "20014,20011",
                               "-o", out, os.path.join(HOST, name + ".cu")])
        libs[name] = ctypes.CDLL(out)
    P, I = ctypes.c_void_p, ctypes.c_int
    for s in ("_d", "_f"):
        f = getattr(libs["ql_host"], "host_ql" + s)
        f.argtypes = [I, P, P, I, I, I, I, P, P, P]
        f.restype = I
        f = getattr(libs["ql_host"], "host_ql_fast" + s)
        f.argtypes = [I, P, P, I, I, I, P, P, P]
        f.restype = I
        getattr(libs["tridiag_host"], "host_tridiag" + s).argtypes = [I, I, I, P, I, I, P, P]
        getattr(libs["tridiag_host"], "host_tridiag_reg" + s).argtypes = [I, P, I, P, P]
        getattr(libs["apply_host"], "host_apply" + s).argtypes = [I, P, P, I, I, I]
        getattr(libs["apply_host"], "host_apply" + s).restype = I
    return libs


def _p(x):
    return ctypes.c_void_p(x.ctypes.data)


def tred(O, a0, n):
    a = np.ascontiguousarray(a0.copy())
    d = np.zeros(n, a.dtype)
    e = np.zeros(n, a.dtype)
    f = O.lib().oracle_tred1_d if a.dtype == np.float64 else O.lib().oracle_tred1_f
    f(n, n, _p(a), _p(d), _p(e))
    return d, e


def host_ql(libs, d, e, method, cap, chunk=0, max_sweep=100):
    n = d.size
    d = d.copy()
    e = e.copy()
    rec = np.zeros(2 * cap, d.dtype)
    nrec = np.zeros(1, np.int32)
    ierr = np.zeros(1, np.int32)
    f = libs["ql_host"].host_ql_d if d.dtype == np.float64 else libs["ql_host"].host_ql_f
    st = f(n, _p(d), _p(e), method, max_sweep, cap, chunk, _p(rec), _p(nrec), _p(ierr))
    return st, d, rec[: 2 * int(nrec[0])].reshape(-1, 2), int(ierr[0])


def apply_records(rec, n, dtype):
    z = np.eye(n)
    q = 0
    ity = np.int64 if dtype == np.float64 else np.int32
    while q < rec.shape[0]:
        i0, cnt = (int(x) for x in rec[q].view(ity))
        q += 1
        for t in range(cnt):
            c, s = (float(x) for x in rec[q])
            q += 1
            i = i0 - t
            h0, h1 = z[:, i].copy(), z[:, i + 1].copy()
            z[:, i + 1] = s * h0 + c * h1
            z[:, i] = c * h0 - s * h1
    return z


@pytest.mark.parametrize("n", [2, 3, 8, 17, 40])
@pytest.mark.parametrize("method", [0, 1])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_ql_generator_matches_oracle(oracle_mod, hostlibs, n, method, dtype):
    O = oracle_mod
    a0 = O.sym_uniform(1, n, seed=n + 10 * method)[0].astype(dtype)
    d, e = tred(O, a0, n)
    cap = 2 * n * n + 4 * n + 32
    st, dq, rec, ierr = host_ql(hostlibs, d, e, method, cap)
    assert st == 0 and ierr == 0
    # same eigenvalues as the oracle's QL on the same (d, e)
    do, eo = d.copy(), e.copy()
    z = np.zeros((n, n), dtype)
    f = getattr(O.lib(), ("oracle_imtql2" if method else "oracle_tql2") + ("_d" if dtype == np.float64 else "_f"))
    assert f(n, n, _p(do), _p(eo), _p(z), 100, None) == 0
    eps = np.finfo(dtype).eps
    assert np.abs(np.sort(dq) - np.sort(do)).max() <= 64 * n * eps * np.abs(do).max()
    # the records rebuild the eigenvectors of T
    T = np.diag(d.astype(np.float64)) + np.diag(e[:-1].astype(np.float64), 1) + np.diag(e[:-1].astype(np.float64), -1)
    zr = apply_records(rec, n, dtype)
    assert np.abs(T @ zr - zr * dq.astype(np.float64)).max() <= 200 * n * eps * np.abs(dq).max()


@pytest.mark.parametrize("method", [0, 1])
def test_ql_resume_in_chunks_is_identical(oracle_mod, hostlibs, method):
    """The phase-3 fallback regenerates the stream in small chunks; segment
    boundaries move, but every rotation and eigenvalue is bit-identical."""
    O = oracle_mod
    n = 24
    d, e = tred(O, O.sym_uniform(1, n, seed=5)[0], n)
    cap = 2 * n * n + 4 * n + 32
    _, d1, r1, _ = host_ql(hostlibs, d, e, method, cap)
    _, d2, r2, _ = host_ql(hostlibs, d, e, method, 100 * cap, chunk=7)
    assert np.array_equal(d1, d2)
    z1, z2 = apply_records(r1, n, np.float64), apply_records(r2, n, np.float64)
    assert np.array_equal(z1, z2)
    st, _, _, _ = host_ql(hostlibs, d, e, method, 40)  # too small: reported as overflow
    assert st == 1


def test_ql_sweep_limit_reports_index(oracle_mod, hostlibs):
    n = 10
    d = np.full(n, np.nan)
    e = np.ones(n)
    e[-1] = 0
    st, _, _, ierr = host_ql(hostlibs, d, e, 0, 100000, max_sweep=3)
    assert st == 0 and ierr == 1


@pytest.mark.parametrize("n,nthr,split,blk", [(2, 32, 1, 2), (3, 32, 1, 3), (8, 32, 1, 8), (32, 32, 1, 32),
                                              (33, 64, 1, 33), (64, 64, 1, 64), (100, 128, 1, 100), (64, 96, 1, 64),
                                              (33, 256, 4, 33), (64, 256, 4, 64), (100, 512, 4, 100),
                                              (77, 192, 2, 77), (128, 512, 4, 128),
                                              # leading block in "shared memory", outer band in G
                                              (100, 512, 4, 60), (77, 192, 2, 1), (64, 256, 4, 0),
                                              (96, 128, 1, 95), (130, 640, 4, 100)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_tridiag_team_code(oracle_mod, hostlibs, n, nthr, split, blk, dtype):
    """Phase 1 (eigb_tridiag.cuh) with the whole matrix, part of it or none
    of it in the shared-memory array."""
    O = oracle_mod
    a0 = O.sym_uniform(1, n, seed=n)[0].astype(dtype)
    ld = n | 1
    S = np.zeros((n, ld), dtype)          # S[c, r] = element (r, c), column-major with ld
    S[:, :n] = a0
    d = np.zeros(n, dtype)
    e = np.zeros(n, dtype)
    f = hostlibs["tridiag_host"].host_tridiag_d if dtype == np.float64 else hostlibs["tridiag_host"].host_tridiag_f
    f(n, nthr, split, _p(S), ld, blk, _p(d), _p(e))
    eps = np.finfo(dtype).eps
    scale = np.abs(a0).max() * n
    M = S[:, :n].T.astype(np.float64)     # M[r, c] with r = row
    Q = M.T
    T = np.diag(d.astype(np.float64)) + np.diag(e[:-1].astype(np.float64), 1) + np.diag(e[:-1].astype(np.float64), -1)
    # backward stable: A = Q T Q^T with Q orthogonal, to rounding level
    assert np.abs(Q @ T @ Q.T - a0).max() <= 64 * eps * scale
    assert np.abs(Q.T @ Q - np.eye(n)).max() <= 64 * eps * n
    # same spectrum as the oracle's tridiagonal (the reduction is the same up
    # to rounding; summation order differs)
    do, eo = tred(O, a0, n)
    To = np.diag(do.astype(np.float64)) + np.diag(eo[:-1].astype(np.float64), 1) + np.diag(eo[:-1].astype(np.float64), -1)
    assert np.abs(np.linalg.eigvalsh(T) - np.linalg.eigvalsh(To)).max() <= 64 * eps * scale


@pytest.mark.parametrize("n,nm", [(33, 33), (40, 41), (64, 64), (65, 66), (96, 96), (100, 101), (128, 128)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_tridiag_register_variant(oracle_mod, hostlibs, n, nm, dtype):
    """The register-resident phase 1 (eigb_tridiag_reg.cuh): reads the upper
    triangle of a (nm x n, column-major), leaves Q (A = Q T Q^T) in its place."""
    O = oracle_mod
    a0 = O.sym_uniform(1, n, seed=n + 1)[0].astype(dtype)
    A = np.full((n, nm), np.nan, dtype)  # A[c, r] = element (r, c)
    A[:, :n] = a0
    for c in range(n):
        A[c, c + 1:n] = np.nan            # strict lower triangle is never read
    d = np.zeros(n, dtype)
    e = np.zeros(n, dtype)
    f = hostlibs["tridiag_host"].host_tridiag_reg_d if dtype == np.float64 else hostlibs["tridiag_host"].host_tridiag_reg_f
    f(n, _p(A), nm, _p(d), _p(e))
    eps = np.finfo(dtype).eps
    scale = np.abs(a0).max() * n
    Q = A[:, :n].T.astype(np.float64)
    T = np.diag(d.astype(np.float64)) + np.diag(e[:-1].astype(np.float64), 1) + np.diag(e[:-1].astype(np.float64), -1)
    assert np.abs(Q @ T @ Q.T - a0).max() <= 64 * eps * scale
    assert np.abs(Q.T @ Q - np.eye(n)).max() <= 64 * eps * n
    assert np.isnan(A[:, n:]).all()     # padding rows untouched
    do, eo = tred(O, a0, n)
    To = np.diag(do.astype(np.float64)) + np.diag(eo[:-1].astype(np.float64), 1) + np.diag(eo[:-1].astype(np.float64), -1)
    assert np.abs(np.linalg.eigvalsh(T) - np.linalg.eigvalsh(To)).max() <= 64 * eps * scale


@pytest.mark.parametrize("n", [2, 5, 16, 33, 64])
@pytest.mark.parametrize("method", [0, 1])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_fast_generator_is_bit_identical(oracle_mod, hostlibs, n, method, dtype):
    """Phase 2's single-call generator emits exactly the records and
    eigenvalues of the resumable generator used by the fallback path."""
    O = oracle_mod
    a0 = O.sym_uniform(1, n, seed=3 * n)[0].astype(dtype)
    d, e = tred(O, a0, n)
    cap = 2 * n * n + 4 * n + 32
    _, d1, r1, i1 = host_ql(hostlibs, d, e, method, cap)
    d2, e2 = d.copy(), e.copy()
    rec = np.zeros(2 * cap, dtype)
    nrec = np.zeros(1, np.int32)
    ierr = np.zeros(1, np.int32)
    f = hostlibs["ql_host"].host_ql_fast_d if dtype == np.float64 else hostlibs["ql_host"].host_ql_fast_f
    assert f(n, _p(d2), _p(e2), method, 100, cap, _p(rec), _p(nrec), _p(ierr)) == 0
    assert int(ierr[0]) == i1
    assert np.array_equal(d2, d1)
    assert np.array_equal(rec[: 2 * int(nrec[0])].reshape(-1, 2).view(np.uint8), r1.view(np.uint8))
    # too small a capacity is reported, not truncated
    assert f(n, _p(d.copy()), _p(e.copy()), method, 100, 3, _p(rec), _p(nrec), _p(ierr)) == (1 if n > 2 else 0) or n <= 2


@pytest.mark.parametrize("n", [3, 8, 17, 33, 64, 100])
@pytest.mark.parametrize("method", [0, 1])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_pipelined_apply_matches_sequential(oracle_mod, hostlibs, n, method, dtype):
    """Phase 3 applies each sweep as one rotation chain whose operands are
    loaded a block ahead; the result equals applying every rotation in
    order, also when the stream is staged in small chunks."""
    O = oracle_mod
    a0 = O.sym_uniform(1, n, seed=7 * n + method)[0].astype(dtype)
    d, e = tred(O, a0, n)
    cap = 2 * n * n + 4 * n + 32
    st, dq, rec, ierr = host_ql(hostlibs, d, e, method, cap)
    assert st == 0
    rng = np.random.default_rng(n)
    q0 = rng.standard_normal((n, n)).astype(dtype)     # any start matrix, row-major
    ref = q0.astype(np.float64) @ apply_records(rec, n, dtype)
    f = hostlibs["apply_host"].host_apply_d if dtype == np.float64 else hostlibs["apply_host"].host_apply_f
    flat = np.ascontiguousarray(rec)
    eps = np.finfo(dtype).eps
    first = None
    for kg in (0, 2, 4, 8):
        for ch in (4 * (n + 1), n + 1, 10 ** 6):
            z = np.ascontiguousarray(q0.copy())
            segs = f(n, _p(z), _p(flat), flat.shape[0], ch, kg)
            assert segs > 0
            assert np.abs(z - ref).max() <= 64 * n * eps * np.abs(ref).max()
            # chunking and the group size change which sweeps are applied
            # together; the pipelines do the same operations in the same
            # order, so the results are identical
            if first is None:
                first = z
            assert np.array_equal(z, first), (kg, ch)
