"""Packed upper-triangle input (eigen_GPU_batch_packed_*) and the
interleaved layout (eigen_GPU_batch_interleaved_*): the same
eigenpairs, bit for bit, as the full-storage solve of the same matrices,
for every phase-1 form (warp, registers, shared-memory block with the band
in global memory) and for Jacobi and n = 1; the packed input is not
modified."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def E():
    import eigeng_b200
    return eigeng_b200


@pytest.mark.parametrize("n,ldz", [(1, 1), (2, 3), (5, 5), (32, 32), (33, 35), (100, 100), (128, 129), (129, 129),
                                   (200, 200), (256, 256)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_packed_matches_full(oracle_mod, n, ldz, dtype):
    O = oracle_mod
    L = 7
    a0 = np.zeros((L, n, ldz))
    a0[:, :, :n] = O.sym_uniform(L, n, seed=n + 17)
    a = torch.from_numpy(a0.astype(dtype)).cuda()
    ap = E().pack_upper(a, n, ldz)
    ap0 = ap.clone()
    z, w, info = E().solve_packed(ap, n, ldz)
    wf, infof = E().solve(a, n, ldz)
    torch.cuda.synchronize()
    assert torch.equal(ap, ap0)
    assert torch.equal(info, infof) and (info == 0).all()
    assert torch.equal(w, wf)
    assert torch.equal(z[:, :, :n], a[:, :, :n])


@pytest.mark.parametrize("method", [1, 2])
def test_packed_other_methods(oracle_mod, method):
    O = oracle_mod
    n = 24
    a = torch.from_numpy(O.sym_uniform(5, n, seed=3)).cuda()
    ap = E().pack_upper(a, n)
    z, w, info = E().solve_packed(ap, n, method=method)
    wf, infof = E().solve(a, n, method=method)
    torch.cuda.synchronize()
    assert torch.equal(w, wf) and torch.equal(z, a) and torch.equal(info, infof)


@pytest.mark.parametrize("n,L", [(1, 7), (5, 33), (32, 100), (64, 70), (130, 45), (256, 9)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_interleaved_matches_full(oracle_mod, n, L, dtype):
    O = oracle_mod
    a0 = O.sym_uniform(L, n, seed=n + 5).astype(dtype)       # (L, n, n) column-major matrices
    a = torch.from_numpy(a0.copy()).cuda()
    ai = a.reshape(L, n * n).t().contiguous()                 # element e of matrix k at ai[e, k]
    zi, wi, info = E().solve_interleaved(ai, n)
    wf, infof = E().solve(a, n)
    torch.cuda.synchronize()
    assert torch.equal(info, infof) and (info == 0).all()
    assert torch.equal(wi.t(), wf)
    assert torch.equal(zi.t().reshape(L, n, n), a)


@pytest.mark.parametrize("n,ldz", [(2, 2), (17, 17), (32, 33), (33, 33), (64, 64), (65, 66), (128, 128),
                                   (129, 129), (200, 200), (256, 256), (300, 300)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_packed_check_matches_the_gate(oracle_mod, n, ldz, dtype):
    """The packed solve with the gate in the same call: the same eigenpairs
    as eigen_GPU_batch_packed_*, and err1, err2 and flags of
    eigen_GPU_check_ex_* on the full matrices, bit for bit (the same
    kernels read the packed triangle instead of the full matrix)."""
    O = oracle_mod
    L = 5
    a0 = np.zeros((L, n, ldz))
    a0[:, :, :n] = O.sym_uniform(L, n, seed=n + 29)
    a = torch.from_numpy(a0.astype(dtype)).cuda()
    ap = E().pack_upper(a, n, ldz)
    ap0 = ap.clone()
    z, w, info, e1, e2, fl = E().solve_packed_checked(ap, n, ldz)
    zp, wp, ip = E().solve_packed(ap, n, ldz)
    torch.cuda.synchronize()
    # rows n .. ldz-1 of each column of z are padding, never written
    assert torch.equal(ap, ap0) and torch.equal(z[:, :, :n], zp[:, :, :n]) and torch.equal(w, wp)
    assert (info == 0).all()
    g1, g2, gf = E().check(a, w, z, n, ldz)
    torch.cuda.synchronize()
    assert torch.equal(fl, gf) and (fl == 0).all()
    assert torch.equal(e1, g1) and torch.equal(e2, g2)

