"""Uneven batches (eigen_GPU_batch_uneven_*): matrices of different orders
back to back in one call give, matrix by matrix, exactly the results of
the uniform solve of the same matrices."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def E():
    import eigeng_b200
    return eigeng_b200


def _check(O, ns, dtype, method=0, seed=0, **kw):
    rng = np.random.default_rng(seed)
    mats = [O.sym_uniform(1, int(n), seed=int(rng.integers(1 << 30)))[0].astype(dtype) for n in ns]
    flat = np.concatenate([m.reshape(-1) for m in mats])
    a = torch.from_numpy(flat.copy()).cuda()
    w, info = E().solve_uneven(a, ns, method=method, **kw)
    torch.cuda.synchronize()
    ao = np.cumsum([0] + [int(n) * int(n) for n in ns])
    wo = np.cumsum([0] + [int(n) for n in ns])
    an, wn, inn = a.cpu().numpy(), w.cpu().numpy(), info.cpu().numpy()
    for n in sorted(set(int(x) for x in ns)):
        idx = [k for k, x in enumerate(ns) if int(x) == n]
        ref = torch.from_numpy(np.stack([mats[k] for k in idx])).cuda()
        wr, ir = E().solve(ref, n, method=method, rec_cap=kw.get("rec_cap", 0))
        torch.cuda.synchronize()
        refn, wrn = ref.cpu().numpy(), wr.cpu().numpy()
        for j, k in enumerate(idx):
            assert np.array_equal(an[ao[k]:ao[k + 1]].reshape(n, n), refn[j]), (n, k)
            assert np.array_equal(wn[wo[k]:wo[k + 1]], wrn[j]), (n, k)
            assert inn[k] == ir[j].item() == 0


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_uneven_matches_uniform(oracle_mod, dtype):
    rng = np.random.default_rng(1)
    ns = list(rng.integers(1, 300, size=70)) + [1, 2, 32, 33, 128, 129, 256, 256, 5, 5, 5]
    rng.shuffle(ns)
    _check(oracle_mod, ns, dtype, seed=2)


@pytest.mark.parametrize("wave,mpw", [(7, 0), (40, 1), (1, 32)])
def test_uneven_waves_and_queue_widths(oracle_mod, wave, mpw):
    """Waves of at most `wave` matrices (groups cut across waves, the
    workspace reused), and the QL queue at 1 and 32 matrices per warp:
    the same bits as the uniform solve."""
    rng = np.random.default_rng(4)
    ns = [int(x) for x in rng.integers(2, 200, size=30)] + [1, 1, 64, 64, 64, 64, 64, 64, 64, 64, 64]
    rng.shuffle(ns)
    _check(oracle_mod, ns, np.float64, seed=5, wave=wave, ql_mpw=mpw)


def test_uneven_imtql2_and_overflowing_records(oracle_mod):
    """imtql2 through the queue; and every matrix's records overflowing a
    small capacity (rec_cap), which the apply phase then regenerates."""
    rng = np.random.default_rng(8)
    ns = [int(x) for x in rng.integers(2, 150, size=20)]
    _check(oracle_mod, ns, np.float64, method=1, seed=9)
    _check(oracle_mod, ns, np.float64, method=0, seed=10, rec_cap=8)


def test_uneven_jacobi_and_errors(oracle_mod):
    _check(oracle_mod, [4, 9, 32, 9, 17], np.float64, method=2, seed=3)
    zeros = lambda k: torch.zeros(k, dtype=torch.float64, device="cuda")  # noqa: E731
    with pytest.raises(E().EigenGError):      # Jacobi is n <= 32
        E().solve_uneven(zeros(40 * 40 + 4), [40, 2], method=2)
    with pytest.raises(E().EigenGError):      # above the size limit
        E().solve_uneven(zeros(1025 * 1025), [1025])


def test_uneven_tensor_memory_bit_identical(oracle_mod):
    """The apply phase of every order group gives the same bits with the
    rows of Z in tensor memory (default) as in shared memory."""
    rng = np.random.default_rng(7)
    ns = [int(x) for x in rng.integers(33, 300, size=24)] + [64, 96, 128, 200, 256]
    mats = [oracle_mod.sym_uniform(1, n, seed=int(rng.integers(1 << 30)))[0] for n in ns]
    flat = np.concatenate([m.reshape(-1) for m in mats])
    a1 = torch.from_numpy(flat.copy()).cuda()
    a2 = torch.from_numpy(flat.copy()).cuda()
    w1, i1 = E().solve_uneven(a1, ns)
    w2, i2 = E().solve_uneven(a2, ns, zmem=E().ZMEM_SHARED)
    torch.cuda.synchronize()
    assert torch.equal(a1, a2) and torch.equal(w1, w2) and torch.equal(i1, i2)
