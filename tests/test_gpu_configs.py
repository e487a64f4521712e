"""Parity on every benchmark configuration family, at the configuration's
own order and precision, with at least 64 matrices per case: the CUDA
library (through its C ABI) against FP64 LAPACK dsyev per matrix and the
CPU oracle.

  C1  (B + B^T)/2, B iid U[-1,1]            n = 32   FP64
  C2  LETKF-like (n-1) I + Y^T Y            n = 128  FP64 and FP32
  C3  Q diag(l) Q^T, l log-spaced 1..1e6,   n in {200, 256, 384, 512}
      random signs, one mixed-size call             FP64
  C4  clusters of 8 eigenvalues 1e-8 apart  n = 256  FP64
      in gaps of 1e-1
  C5  A0 + sum_j theta_j E_j                n = 64   FP32

Tolerances (all relative to ||A||_2 = max |lambda|):
  * per-eigenpair residual ||A v - lambda v||_2 <= 1e-12 (FP64), 2e-5 (FP32)
  * orthogonality max |V^T V - I| <= 4e-15 n (FP64), 2e-5 (FP32)
  * eigenvalues within 64 n eps of LAPACK's
  * C4: each cluster's invariant subspace, compared through the largest
    principal angle with LAPACK's: sin <= 1e-10 (the eigenvectors inside a
    cluster 1e-8 wide are determined only up to rotation at this accuracy,
    so per-vector comparisons would be meaningless there)
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def E():
    import eigeng_b200
    return eigeng_b200


def full(a0, n):
    """Symmetric FP64 matrices from the upper triangles of column-major storage."""
    A = np.triu(np.transpose(np.asarray(a0, np.float64)[:, :n, :n], (0, 2, 1)))
    return A + np.transpose(np.triu(A, 1), (0, 2, 1))


def metrics(A, w, z, n):
    """(per-pair residual, orthogonality) relative to ||A||_2, per matrix."""
    V = np.transpose(np.asarray(z, np.float64)[:, :n, :n], (0, 2, 1))
    w = np.asarray(w, np.float64)
    an = np.abs(np.linalg.eigvalsh(A)).max(axis=1)
    r = np.linalg.norm(A @ V - V * w[:, None, :], axis=1).max(axis=1) / an
    o = np.abs(np.transpose(V, (0, 2, 1)) @ V - np.eye(n)).max(axis=(1, 2))
    return r, o


def bounds(dtype, n):
    if dtype == np.float64:
        return 1e-12, 4e-15 * n
    return 2e-5, 2e-5


def check_family(oracle_mod, a0, n, dtype):
    O = oracle_mod
    a = torch.from_numpy(np.ascontiguousarray(a0.astype(dtype))).cuda()
    w, info = E().solve(a, n)
    torch.cuda.synchronize()
    w, z, info = w.cpu().numpy(), a.cpu().numpy(), info.cpu().numpy()
    assert (info == 0).all()
    A = full(a0.astype(dtype), n)
    r, o = metrics(A, w, z, n)
    rb, ob = bounds(dtype, n)
    assert r.max() <= rb, r.max()
    assert o.max() <= ob, o.max()
    wl, vl = O.lapack_eigh(a0.astype(dtype), n)
    eps = np.finfo(dtype).eps
    scale = np.abs(wl).max(axis=1, keepdims=True)
    assert (np.abs(w - wl) <= 64 * n * eps * scale).all()
    # and the CPU oracle (the reference's method)
    ao = np.ascontiguousarray(a0.astype(dtype)).copy()
    wo, io, _ = O.eigen_batch(ao, n)
    assert (io == 0).all()
    assert (np.abs(w - wo) <= 64 * n * eps * scale).all()
    return w, z, wl, vl


def test_c1_uniform_n32_fp64(oracle_mod):
    check_family(oracle_mod, oracle_mod.sym_uniform(64, 32, seed=101), 32, np.float64)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_c2_letkf_n128(oracle_mod, dtype):
    check_family(oracle_mod, oracle_mod.letkf_like(64, 128, seed=102), 128, dtype)


def test_c3_logspaced_mixed_sizes_fp64(oracle_mod):
    """One eigen_GPU_batch_uneven_DP call over 64 matrices of orders 200,
    256, 384 and 512 (interleaved), each checked on its own."""
    O = oracle_mod
    orders = [200, 256, 384, 512] * 16
    mats = {nn: O.logspaced_spectrum(16, nn, seed=103 + nn) for nn in set(orders)}
    used = {nn: 0 for nn in mats}
    seq = []
    for nn in orders:
        seq.append((nn, mats[nn][used[nn]]))
        used[nn] += 1
    flat = np.concatenate([m.reshape(-1) for _, m in seq])
    a = torch.from_numpy(flat.copy()).cuda()
    w, info = E().solve_uneven(a, orders)
    torch.cuda.synchronize()
    assert (info.cpu().numpy() == 0).all()
    z_all, w_all = a.cpu().numpy(), w.cpu().numpy()
    oa = ow = 0
    for nn, m in seq:
        z = z_all[oa:oa + nn * nn].reshape(1, nn, nn)
        wk = w_all[ow:ow + nn].reshape(1, nn)
        oa += nn * nn
        ow += nn
        A = full(m[None], nn)
        r, o = metrics(A, wk, z, nn)
        rb, ob = bounds(np.float64, nn)
        assert r.max() <= rb and o.max() <= ob, (nn, r.max(), o.max())
        wl, _ = O.lapack_eigh(m[None], nn)
        assert np.abs(wk - wl).max() <= 64 * nn * np.finfo(np.float64).eps * np.abs(wl).max()


def test_c4_clustered_n256_fp64_cluster_subspaces(oracle_mod):
    n, cl = 256, 8
    a0 = oracle_mod.clustered_spectrum(64, n, seed=104)
    w, z, wl, vl = check_family(oracle_mod, a0, n, np.float64)
    V = np.transpose(z[:, :n, :n], (0, 2, 1))
    for k in range(a0.shape[0]):
        for c in range(n // cl):
            Vg = V[k][:, c * cl:(c + 1) * cl]
            Vl = vl[k][c * cl:(c + 1) * cl].T           # lapack_eigh returns rows = eigenvectors
            # sine of the largest principal angle: ||(I - Vl Vl^T) Vg||_2
            s = np.linalg.norm(Vg - Vl @ (Vl.T @ Vg), 2)
            assert s <= 1e-10, (k, c, s)


def test_c5_theta_family_n64_fp32(oracle_mod):
    check_family(oracle_mod, oracle_mod.theta_family(64, 64, seed=105), 64, np.float32)
