"""No path reads workspace memory it has not written: every solve gives the
same bits with a workspace filled with 0xFF bytes (NaN as FP64 and FP32,
-1 as integers) as with a zeroed one.  A read of a stale entry, even one
multiplied by zero, shows as NaN or as a changed result.  (A refinement
update once read the unused entries of its cluster rotations: matrices
failed over to the fallback depending on what the workspace had held.)"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def E():
    import eigeng_b200
    return eigeng_b200


def _pair(make_wk, run):
    """run(wk) with a zeroed and with a 0xFF-filled workspace; returns both."""
    wk = make_wk()
    wk.zero_()
    r0 = run(wk)
    wk.fill_(255)
    r1 = run(wk)
    torch.cuda.synchronize()
    return r0, r1


def _same(r0, r1):
    for x, y in zip(r0, r1):
        assert torch.equal(x, y)


@pytest.mark.parametrize("n,dtype", [(16, np.float64), (64, np.float64), (128, np.float32), (200, np.float64),
                                     (256, np.float64), (700, np.float64)])
def test_plain_solve(oracle_mod, n, dtype):
    a0 = oracle_mod.sym_uniform(3 if n > 256 else 8, n, seed=n).astype(dtype)
    L = a0.shape[0]
    td = torch.float64 if dtype == np.float64 else torch.float32

    def run(wk):
        a = torch.from_numpy(a0.copy()).cuda()
        w = torch.empty((L, n), dtype=td, device="cuda")
        info = torch.zeros(L, dtype=torch.int32, device="cuda")
        assert E().eigen_GPU_batch_ex(a, w, wk, n, info=info) == 0
        return a, w, info
    _same(*_pair(lambda: E().workspace(L, n, n, td), run))


@pytest.mark.parametrize("family,n", [("clustered", 256), ("letkf", 128), ("uniform", 40)])
def test_refined_solve(oracle_mod, family, n):
    O = oracle_mod
    a0 = {"clustered": lambda: O.clustered_spectrum(16, n, seed=7), "letkf": lambda: O.letkf_like(16, n, seed=7),
          "uniform": lambda: O.sym_uniform(16, n, seed=7)}[family]()

    def run(wk):
        a = torch.from_numpy(np.ascontiguousarray(a0)).cuda()
        w, info, it = E().solve_refined(a, n, wk=wk)
        return a, w, info, it
    r0, r1 = _pair(lambda: E().refine_workspace(a0.shape[0], n, n), run)
    _same(r0, r1)
    if family == "clustered":
        assert (r1[3].cpu().numpy() >= 1).all()  # no fallback


def test_uneven_solve(oracle_mod):
    rng = np.random.default_rng(3)
    ns = [int(x) for x in rng.integers(1, 260, size=24)] + [1, 32, 33, 128, 256]
    mats = [oracle_mod.sym_uniform(1, n, seed=int(rng.integers(1 << 30)))[0] for n in ns]
    flat = np.concatenate([m.reshape(-1) for m in mats])
    import ctypes
    nsa = (ctypes.c_int * len(ns))(*ns)

    def make():
        o = E().Opts(0, 1, 100, 0, 0, 0, 0, 0)
        lw = ctypes.c_size_t(0)
        assert E().lib().eigen_GPU_batch_uneven_BufferSize_DP(len(ns), nsa, ctypes.byref(o), ctypes.byref(lw)) == 0
        return torch.empty(max(lw.value, 16), dtype=torch.uint8, device="cuda")

    def run(wk):
        a = torch.from_numpy(flat.copy()).cuda()
        w = torch.empty(sum(ns), dtype=torch.float64, device="cuda")
        info = torch.zeros(len(ns), dtype=torch.int32, device="cuda")
        o = E().Opts(0, 1, 100, 0, 0, 0, 0, 0)
        st = E().lib().eigen_GPU_batch_uneven_DP(len(ns), nsa, E()._ptr(a), E()._ptr(w), E()._ptr(wk),
                                                 wk.numel(), E()._ptr(info), ctypes.byref(o), E()._stream(None))
        assert st == 0
        return a, w, info
    _same(*_pair(make, run))


def test_learned_solve(oracle_mod):
    import eigeng_b200.learned as lw
    n = 64
    a0, e = oracle_mod.theta_family_basis(n)
    a0t, et = torch.from_numpy(a0).cuda(), torch.from_numpy(e).cuda()
    v0 = lw.basis_eigenvectors(a0t)
    fam = lw.family_buffer(a0t, et, v0)
    A = oracle_mod.theta_family(32, n, seed=5)
    net = lw.MLP(512, 512, n * n, seed=5)

    def run(wk):
        a = torch.from_numpy(A.copy()).cuda()
        w, info, sweeps, resid = lw.solve_learned(a, n, fam, net, wk=wk)
        return a, w, info, sweeps
    _same(*_pair(lambda: lw.learned_workspace(32, n, n, net.dims), run))
