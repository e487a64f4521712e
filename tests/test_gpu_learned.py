"""The learned warm start on the GPU, through the C ABI
(include/eigen_GPU_learned.h):

  * the network's forward pass and gradient against the CPU reference
    (oracle/mlp_ref.py, itself checked by finite differences) with the same
    BF16 rounding of each product's operands: relative error of the
    gradient vector <= 1e-3 (FP32 against FP64 accumulation);
  * training with the library's Adam step lowers the loss;
  * the learned solve on the C5 family A(theta) = A0 + sum theta_j E_j
    (n = 64, FP32): every matrix passes the residual gate (max_j ||A x_j -
    w_j x_j|| <= 1e-6 max|w|, checked again here in FP64 against the
    input), eigenvalues within 1e-5 max|w| of FP64 LAPACK, orthogonality
    <= 1e-5;
  * ablation: with the trained network the polish needs fewer Jacobi
    sweeps than from A0's eigenbasis, which needs fewer than from the
    identity;
  * fallback: matrices that fail the gate are solved by the plain path.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def L():
    import eigeng_b200.learned as learned
    return learned


def test_mlp_forward_and_gradient_match_cpu_reference():
    import mlp_ref as M
    lw = L()
    torch.manual_seed(0)
    net = lw.MLP(64, 64, 256, seed=7)
    rows = 64
    x = (torch.rand((rows, lw.D0), device="cuda") - 0.5)
    x[:, 4:] = 0
    t = torch.randn((rows, 256), device="cuda") * 0.1
    flat = net.flat().double().cpu().numpy()
    y = net.forward(x)
    g, sse = net.gradient(x, t)
    torch.cuda.synchronize()
    yr, _ = M.forward(flat, net.dims, x.cpu().numpy(), bf16=True)
    gr, sser = M.gradient(flat, net.dims, x.cpu().numpy(), t.cpu().numpy(), bf16=True)
    yg = y.cpu().numpy()
    assert np.abs(yg - yr).max() <= 1e-3 * np.abs(yr).max()
    gg = g.double().cpu().numpy()
    rel = np.linalg.norm(gg - gr) / np.linalg.norm(gr)
    assert rel <= 1e-3, rel
    assert abs(float(sse.item()) - sser) <= 1e-3 * sser
    # each block of the gradient (weights and biases of every layer) on its own
    o = 0
    for shp in ((64, 16), (64,), (64, 64), (64,), (256, 64), (256,)):
        k = int(np.prod(shp))
        blk = slice(o, o + k)
        assert np.linalg.norm(gg[blk] - gr[blk]) <= 2e-3 * np.linalg.norm(gr[blk]) + 1e-12, shp
        o += k


def test_mlp_training_lowers_the_loss():
    lw = L()
    torch.manual_seed(1)
    net = lw.MLP(64, 64, 64, seed=3)
    n = 2048
    th = torch.rand((n, 4), device="cuda") - 0.5
    x = torch.zeros((n, lw.D0), device="cuda")
    x[:, :4] = th
    # a smooth target of the four inputs
    t = torch.stack([torch.sin(3 * th[:, i % 4]) * torch.cos(2 * th[:, (i + 1) % 4]) for i in range(64)], dim=1)
    hist = lw.train(net, x, t.contiguous(), epochs=30, batch=256, lr=3e-3, lr_final=3e-4)
    assert hist[-1] <= 0.05 * hist[0], hist


@pytest.fixture(scope="module")
def family(oracle_mod):
    lw = L()
    a0, e = oracle_mod.theta_family_basis(64)
    a0t = torch.from_numpy(a0).cuda()
    et = torch.from_numpy(e).cuda()
    v0 = lw.basis_eigenvectors(a0t)
    return a0t, et, v0, lw.family_buffer(a0t, et, v0)


@pytest.fixture(scope="module")
def trained(family):
    lw = L()
    a0, e, v0, fam = family
    x, t = lw.make_dataset(a0, e, v0, 16384, seed=11)
    net = lw.MLP(256, 256, 64 * 64, seed=5)
    hist = lw.train(net, x, t, epochs=12, batch=512, lr=2e-3, lr_final=1e-4)
    assert hist[-1] < hist[0]
    return net


def _check(oracle_mod, a0, z, w, n, tol=1e-6):
    A = np.asarray(a0, dtype=np.float64)
    V = np.transpose(np.asarray(z, dtype=np.float64), (0, 2, 1))
    wv = np.asarray(w, dtype=np.float64)
    an = np.abs(np.linalg.eigvalsh(A)).max(axis=1)
    r = np.linalg.norm(A @ V - V * wv[:, None, :], axis=1).max(axis=1) / an
    o = np.abs(np.transpose(V, (0, 2, 1)) @ V - np.eye(n)).max(axis=(1, 2))
    wl = np.linalg.eigvalsh(A)
    return r, o, np.abs(wv - wl).max(axis=1) / an


def test_learned_solve_and_ablation(oracle_mod, family, trained):
    lw = L()
    a0, e, v0, fam = family
    n = 64
    A = oracle_mod.theta_family(256, n, seed=99)                      # FP32, the C5 family
    res = {}
    for warm in (lw.WARM_NETWORK, 1, 2):
        a = torch.from_numpy(A.copy()).cuda()
        w, info, sweeps, resid = lw.solve_learned(a, n, fam, trained if warm == 0 else None, warm=warm)
        torch.cuda.synchronize()
        info, sweeps = info.cpu().numpy(), sweeps.cpu().numpy()
        r, o, dw = _check(oracle_mod, A, a.cpu().numpy(), w.cpu().numpy(), n)
        assert (info == 0).all()
        passed = sweeps >= 0
        # gate-passing matrices: the gate's 1e-6 plus the FP32 rounding of the
        # output; the others come from the plain FP32 path, at its accuracy
        assert r[passed].max() <= 2e-6, (warm, r[passed].max())
        assert r.max() <= 2e-5 and o.max() <= 2e-5 and dw.max() <= 1e-5, (warm, r.max(), o.max(), dw.max())
        res[warm] = (passed.mean(), sweeps[passed].mean() if passed.any() else np.inf)
        print("warm", warm, "gate pass rate", res[warm][0], "mean sweeps", res[warm][1])
    assert res[0][0] >= 0.95
    assert res[0][1] < res[1][1] < res[2][1], res


def test_learned_fallback(oracle_mod, family):
    """With one Jacobi sweep from the identity most matrices fail the gate;
    the plain path then solves them (sweeps -1), results as accurate as that
    path's, and with the fallback off they are left unsolved (info -1)."""
    lw = L()
    a0, e, v0, fam = family
    n = 64
    A = oracle_mod.theta_family(32, n, seed=98)
    a = torch.from_numpy(A.copy()).cuda()
    w, info, sweeps, resid = lw.solve_learned(a, n, fam, None, warm=2, max_sweeps=1)
    torch.cuda.synchronize()
    sw = sweeps.cpu().numpy()
    assert (sw == -1).sum() >= 16 and (info.cpu().numpy() == 0).all()
    r, o, dw = _check(oracle_mod, A, a.cpu().numpy(), w.cpu().numpy(), n)
    assert r.max() <= 2e-5 and dw.max() <= 1e-5
    a2 = torch.from_numpy(A.copy()).cuda()
    w2, info2, sweeps2, _ = lw.solve_learned(a2, n, fam, None, warm=2, max_sweeps=1, fallback=False)
    torch.cuda.synchronize()
    failed = sweeps2.cpu().numpy() == -1
    assert (info2.cpu().numpy()[failed] == -1).all()
