"""Matrix functions of a solved batch, Z = V diag(f(w)) V^T
(eigen_GPU_batch_symfunc_*, the reference's symdmt.cu:5-80), checked
against the FP64 restatement oracle.symdmt on the GPU's own eigenpairs."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def E():
    import eigeng_b200
    return eigeng_b200


F = {0: lambda x, p: x, 1: lambda x, p: np.power(x, p), 2: lambda x, p: np.exp(p * x)}


@pytest.mark.parametrize("n,nm", [(1, 1), (5, 7), (33, 33), (64, 64), (65, 70), (128, 128), (200, 201)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("func,p", [(0, 0.0), (1, 0.5), (1, -1.0), (2, 0.01)])
def test_symfunc_matches_oracle(oracle_mod, n, nm, dtype, func, p):
    O = oracle_mod
    L = 5
    a0 = np.zeros((L, n, nm))
    a0[:, :, :n] = O.letkf_like(L, n, seed=n)           # symmetric positive definite
    a = torch.from_numpy(a0.astype(dtype)).cuda()
    w, info = E().solve(a, n, nm)
    assert (info == 0).all()
    z = torch.full_like(a, float("nan"))
    E().symfunc(a, w, n, func=func, p=p, nm=nm, z=z)
    torch.cuda.synchronize()
    wn = w.cpu().numpy().astype(np.float64)
    d = F[func](wn, p)
    ref = O.symdmt(a.cpu().numpy(), d, n)
    got = z.cpu().numpy()
    eps = np.finfo(dtype).eps
    scale = np.abs(d).max(axis=1)[:, None, None]
    assert (np.abs(got[:, :n, :n] - ref) <= 32 * n * eps * scale).all()
    assert np.isnan(got[:, :, n:]).all()                  # padding rows untouched
    assert np.array_equal(got[:, :n, :n], np.transpose(got[:, :n, :n], (0, 2, 1)))  # exactly symmetric


def test_square_root_squares_back(oracle_mod):
    """LETKF use: the symmetric square root of an SPD matrix."""
    O = oracle_mod
    n, L = 96, 4
    a0 = O.letkf_like(L, n, seed=3)
    a = torch.from_numpy(a0.copy()).cuda()
    w, _ = E().solve(a, n)
    z = E().symfunc(a, w, n, func=E().FUNC_POW, p=0.5)
    zn = z.cpu().numpy()
    A = np.transpose(a0, (0, 2, 1))
    A = np.triu(A) + np.transpose(np.triu(A, 1), (0, 2, 1))
    S = np.transpose(zn, (0, 2, 1))
    assert np.abs(S @ S - A).max() <= 1e-12 * np.abs(A).max() * n


def test_symfunc_rejects_bad_arguments():
    import eigeng_b200 as Em
    v = torch.zeros((1, 4, 4), dtype=torch.float64, device="cuda")
    w = torch.zeros((1, 4), dtype=torch.float64, device="cuda")
    lib = Em.lib()
    st = lib.eigen_GPU_batch_symfunc_DP(1, 4, 4, v.data_ptr(), w.data_ptr(), v.data_ptr(), 1, 0.5, None)
    assert st == 1                                          # z aliases v
    z = torch.empty_like(v)
    assert lib.eigen_GPU_batch_symfunc_DP(1, 4, 4, v.data_ptr(), w.data_ptr(), z.data_ptr(), 7, 0.5, None) == 1
    assert lib.eigen_GPU_batch_symfunc_DP(1, 3, 4, v.data_ptr(), w.data_ptr(), z.data_ptr(), 1, 0.5, None) == 1
