"""The tensor-core precision form: FP64-accurate Rayleigh products on the
int8 tensor cores (eigen_GPU_batch_rayleigh_DP) and the FP32 solve refined
to FP64 accuracy (eigen_GPU_batch_refine_DP), both through the C ABI.

Tolerances:
  * products: |S - X^T A X| <= 2 n eps (|X|^T |A| |X|) elementwise (the
    standard bound of an FP64 product), against an extended-precision
    (80-bit) reference; the same for G = X^T X
  * refined eigenpairs (relative to ||A||_2 = max |lambda|): per-pair
    residual ||A v - lambda v||_2 <= 1e-12 (1e-13 for the clustered C4
    family, its configuration's target), orthogonality max |V^T V - I| <=
    max(4e-15 n, 1e-13) (the plain FP64 path's level), eigenvalues within 64 n eps of LAPACK dsyev's, cluster
    subspaces (C4) within sin 1e-10 of LAPACK's
  * fallback: a matrix that does not converge is solved by the plain FP64
    path, whose results it then equals bit for bit
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def E():
    import eigeng_b200
    return eigeng_b200


def full(a0, n):
    A = np.triu(np.transpose(np.asarray(a0, np.float64)[:, :n, :n], (0, 2, 1)))
    return A + np.transpose(np.triu(A, 1), (0, 2, 1))


@pytest.mark.parametrize("n", [2, 8, 32, 33, 64, 100, 128, 129, 200, 256])
def test_rayleigh_products_fp64_accurate(oracle_mod, n):
    O = oracle_mod
    L = 4
    rng = np.random.default_rng(n)
    a0 = O.logspaced_spectrum(L, n, seed=n) if n % 2 else O.sym_uniform(L, n, seed=n)
    x0 = rng.standard_normal((L, n, n)) * np.exp(rng.uniform(-20, 5, size=(L, n, 1)))  # columns of mixed scale
    s, g = E().rayleigh(torch.from_numpy(a0).cuda(), torch.from_numpy(np.ascontiguousarray(x0)).cuda(), n)
    torch.cuda.synchronize()
    s, g = s.cpu().numpy(), g.cpu().numpy()
    A = full(a0, n).astype(np.longdouble)
    X = np.transpose(x0, (0, 2, 1)).astype(np.longdouble)   # X[k] = column-major matrix
    Xt = np.transpose(X, (0, 2, 1))
    S_ref = Xt @ A @ X
    G_ref = Xt @ X
    bS = 2 * n * np.finfo(np.float64).eps * (np.abs(Xt) @ np.abs(A) @ np.abs(X))
    bG = 2 * n * np.finfo(np.float64).eps * (np.abs(Xt) @ np.abs(X))
    S_got = np.transpose(s, (0, 2, 1)).astype(np.longdouble)  # s[k] holds column-major S
    G_got = np.transpose(g, (0, 2, 1)).astype(np.longdouble)
    assert (np.abs(S_got - S_ref) <= bS).all(), float(np.max(np.abs(S_got - S_ref) / bS))
    assert (np.abs(G_got - G_ref) <= bG).all(), float(np.max(np.abs(G_got - G_ref) / bG))


def refined(a0, n, **kw):
    a = torch.from_numpy(np.ascontiguousarray(a0)).cuda()
    w, info, iters = E().solve_refined(a, n, **kw)
    torch.cuda.synchronize()
    return w.cpu().numpy(), a.cpu().numpy(), info.cpu().numpy(), iters.cpu().numpy()


def check_accuracy(oracle_mod, a0, n, w, z, res_bound=1e-12):
    O = oracle_mod
    A = full(a0, n)
    V = np.transpose(z[:, :n, :n], (0, 2, 1))
    wl, vl = O.lapack_eigh(a0, n)
    an = np.abs(wl).max(axis=1)
    r = np.linalg.norm(A @ V - V * w[:, None, :], axis=1).max(axis=1) / an
    o = np.abs(np.transpose(V, (0, 2, 1)) @ V - np.eye(n)).max(axis=(1, 2))
    assert r.max() <= res_bound, r.max()
    assert o.max() <= max(4e-15 * n, 1e-13), o.max()
    assert (np.abs(w - wl) <= 64 * n * np.finfo(np.float64).eps * an[:, None]).all()
    assert (np.diff(w, axis=1) >= 0).all()
    return wl, vl


FAMILIES = {
    "c1_uniform_n32": (lambda O: O.sym_uniform(64, 32, seed=201), 32),
    "c2_letkf_n128": (lambda O: O.letkf_like(64, 128, seed=202), 128),
    "uniform_n256": (lambda O: O.sym_uniform(16, 256, seed=203), 256),
    "logspaced_n128": (lambda O: O.logspaced_spectrum(16, 128, seed=204), 128),
    "uniform_n5": (lambda O: O.sym_uniform(64, 5, seed=205), 5),
    "uniform_n17": (lambda O: O.sym_uniform(64, 17, seed=206), 17),
    "letkf_n100": (lambda O: O.letkf_like(32, 100, seed=207), 100),
    "uniform_n200": (lambda O: O.sym_uniform(16, 200, seed=208), 200),
    "frank_n64": (lambda O: O.frank(8, 64), 64),
}


@pytest.mark.parametrize("fam", sorted(FAMILIES))
def test_refined_solve_matches_lapack(oracle_mod, fam):
    gen, n = FAMILIES[fam]
    a0 = gen(oracle_mod)
    w, z, info, iters = refined(a0, n)
    assert (info == 0).all()
    assert (iters >= 0).all() and (iters <= 3).all()
    print(fam, "iterations", np.bincount(iters, minlength=4).tolist())
    check_accuracy(oracle_mod, a0, n, w, z)


def test_refined_c4_clusters(oracle_mod):
    """C4: clusters of eight eigenvalues 1e-8 apart, n = 256, residual
    <= 1e-13 ||A||; the cluster Rayleigh-Ritz step resolves them (within
    the three refinement iterations, no fallback)."""
    n, cl = 256, 8
    a0 = oracle_mod.clustered_spectrum(64, n, seed=209)
    w, z, info, iters = refined(a0, n)
    assert (info == 0).all()
    assert ((iters >= 1) & (iters <= 3)).all(), np.bincount(iters)
    A = full(a0, n)
    V = np.transpose(z, (0, 2, 1))
    r = np.linalg.norm(A @ V - V * w[:, None, :], axis=1).max(axis=1) / np.abs(w).max(axis=1)
    print("C4 worst residuals", np.sort(r)[-3:], "their iterations", iters[np.argsort(r)[-3:]],
          "iterations", np.bincount(iters, minlength=4).tolist())
    wl, vl = check_accuracy(oracle_mod, a0, n, w, z, res_bound=1e-13)
    V = np.transpose(z, (0, 2, 1))
    for k in range(a0.shape[0]):
        for c in range(n // cl):
            Vg = V[k][:, c * cl:(c + 1) * cl]
            Vl = vl[k][c * cl:(c + 1) * cl].T
            assert np.linalg.norm(Vg - Vl @ (Vl.T @ Vg), 2) <= 1e-10


def test_refined_fallback_equals_plain_path(oracle_mod):
    """With an unreachable tolerance every matrix goes to the fallback,
    whose results are the plain FP64 path's, bit for bit; with the
    fallback off they are reported (info -1) and left unsolved."""
    n = 48
    a0 = oracle_mod.sym_uniform(37, n, seed=210)
    w, z, info, iters = refined(a0, n, max_iter=1, tol=1e-300)
    assert (iters == 0).all() and (info == 0).all()
    a = torch.from_numpy(a0.copy()).cuda()
    wp, ip = E().solve(a, n)
    torch.cuda.synchronize()
    assert np.array_equal(w, wp.cpu().numpy())
    assert np.array_equal(z, a.cpu().numpy())
    w2, z2, info2, iters2 = refined(a0, n, max_iter=1, tol=1e-300, fallback=False)
    assert (info2 == -1).all() and (iters2 == 0).all()
    assert np.array_equal(z2, a0)  # untouched


def test_refined_partial_fallback_and_nan(oracle_mod):
    """A NaN matrix fails its FP32 solve and goes to the fallback, which
    reports it; the other matrices are refined normally."""
    n = 64
    a0 = oracle_mod.sym_uniform(20, n, seed=211)
    a0[7, 3, 2] = a0[7, 2, 3] = np.nan
    w, z, info, iters = refined(a0, n)
    ok = np.arange(20) != 7
    assert info[7] != 0 and iters[7] == 0
    assert (info[ok] == 0).all() and (iters[ok] >= 1).all()
    check_accuracy(oracle_mod, a0[ok], n, w[ok], z[ok])


def test_refined_chunks_and_n1(oracle_mod):
    """Several internal chunks give the one-chunk results bit for bit; n = 1."""
    n = 40
    a0 = oracle_mod.sym_uniform(50, n, seed=212)
    w1, z1, _, it1 = refined(a0, n)
    w2, z2, _, it2 = refined(a0, n, chunk=16)
    assert np.array_equal(w1, w2) and np.array_equal(z1, z2) and np.array_equal(it1, it2)
    a1 = np.array([[[3.5]], [[-2.0]]])
    w, z, info, iters = refined(a1, 1)
    assert np.array_equal(w[:, 0], [3.5, -2.0]) and np.array_equal(z[:, 0, 0], [1.0, 1.0])
