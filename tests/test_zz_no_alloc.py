"""eigen_GPU_batch_noalloc_DP: the entry point for callers that cannot
allocate device memory (its workspace is a static array inside the
library).  Its results must match the regular entry point's within the
parity tolerances of the other GPU tests, on two calls in a row -- the
second call reuses the array the first one left behind.  Kept in its own
file, collected last, so that a run stopping at the first failure has
already run every other test."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _inputs(L, n, seed):
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1.0, 1.0, size=(L, n, n))
    return np.ascontiguousarray(0.5 * (b + b.transpose(0, 2, 1)))


def _regular(a0, n):
    import eigeng_b200 as E
    a = torch.from_numpy(a0.copy()).cuda()
    w, info = E.solve(a, n)
    torch.cuda.synchronize()
    return w.cpu().numpy(), a.cpu().numpy(), info.cpu().numpy()


def _noalloc(a0, n):
    import eigeng_b200 as E
    L = a0.shape[0]
    a = torch.from_numpy(a0.copy()).cuda()
    w = torch.empty((L, n), dtype=torch.float64, device="cuda")
    info = torch.full((L,), -7, dtype=torch.int32, device="cuda")
    st = E.eigen_GPU_batch_noalloc(a, w, n, info=info)
    torch.cuda.synchronize()
    assert st == 0
    return w.cpu().numpy(), a.cpu().numpy(), info.cpu().numpy()


def _close(ref, got, n):
    w_r, z_r, i_r = ref
    w_g, z_g, i_g = got
    eps = np.finfo(np.float64).eps
    scale = np.abs(w_r).max(axis=1, keepdims=True)
    assert np.array_equal(i_g, i_r) and (i_g == 0).all()
    assert (np.abs(w_g - w_r) <= 64 * n * eps * scale).all()
    for k in range(w_r.shape[0]):
        wl = w_r[k]
        gaps = np.minimum(np.diff(wl, prepend=-np.inf), np.diff(wl, append=np.inf))
        for j in range(n):
            dot = abs(float(np.dot(z_g[k, j], z_r[k, j])))
            assert 1.0 - dot <= max(256 * eps * n * scale[k, 0] / max(gaps[j], 1e-300), 100 * eps * n)


def test_noalloc_matches_regular_entry_point_twice():
    # first call: a batch larger than the static workspace holds at once
    # (n = 128: about 120 matrices per piece), second call: another size
    for L, n, seed in ((300, 128, 1), (50, 40, 2)):
        a0 = _inputs(L, n, seed)
        _close(_regular(a0, n), _noalloc(a0, n), n)


def test_noalloc_largest_matrix_fits():
    """One matrix of the largest supported order, n = 1024, fits the static
    workspace on its own (two calls of one matrix each, then one of two,
    which the library runs one matrix per piece): results match the
    regular entry point and FP64 LAPACK."""
    from scipy.linalg import lapack
    n = 1024
    a0 = _inputs(2, n, 5)
    ref = _regular(a0, n)
    for k in range(2):
        got = _noalloc(a0[k:k + 1], n)
        _close(tuple(x[k:k + 1] for x in ref), got, n)
    _close(ref, _noalloc(a0, n), n)
    wl, _, inf = lapack.dsyev(np.asfortranarray(a0[0].T), compute_v=0)
    assert inf == 0
    assert np.abs(ref[0][0] - wl).max() <= 64 * n * np.finfo(np.float64).eps * np.abs(wl).max()


def test_noalloc_rejects_sizes_beyond_limit():
    import eigeng_b200 as E
    a = torch.zeros((1, 4, 4), dtype=torch.float64, device="cuda")
    w = torch.zeros((1, 4), dtype=torch.float64, device="cuda")
    assert E.eigen_GPU_batch_noalloc(a, w, 4, nm=4, m=5) == 1   # m > n: cudaErrorInvalidValue
    big = torch.zeros((1, 1100, 1100), dtype=torch.float64, device="cuda")
    wb = torch.zeros((1, 1100), dtype=torch.float64, device="cuda")
    assert E.eigen_GPU_batch_noalloc(big, wb, 1100) == 1        # n above the supported 1024
