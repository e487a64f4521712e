"""The learned warm start: a small MLP, trained by this library's own
kernels on eigenpairs this library computes, predicts the eigenvectors of
members of a parameterised matrix family

    A(theta) = A0 + sum_{j=1..4} theta_j E_j,

which eigen_GPU_batch_learned_FP then polishes (tensor-core products and
Jacobi) and gates (residual check, plain-path fallback).  This module is
the host side: ctypes bindings of include/eigen_GPU_learned.h and the
training driver.  Every computation runs in the library's kernels; torch
supplies device memory, random parameters and index sampling only.
"""
from __future__ import annotations

import ctypes

import torch

from . import EigenGError, LearnedOpts, WARM_NETWORK, _ptr, _stream, lib, solve

D0 = 16  # network input: ten times the four family coordinates, zero padded


class MLP:
    """Parameters (one device buffer) of the network d0 -> d1 -> d2 -> d3."""

    def __init__(self, d1, d2, d3, seed=1, device=None, d0=D0):
        self.dims = (d0, d1, d2, d3)
        sz = ctypes.c_size_t(0)
        st = lib().eigen_GPU_mlp_size(*self.dims, ctypes.byref(sz))
        if st != 0:
            raise EigenGError(f"eigen_GPU_mlp_size failed with cudaError {st}")
        self.params = torch.empty(sz.value, dtype=torch.uint8, device=device or "cuda")
        st = lib().eigen_GPU_mlp_init(*self.dims, _ptr(self.params), seed, _stream(None))
        if st != 0:
            raise EigenGError(f"eigen_GPU_mlp_init failed with cudaError {st}")
        self.step = 0
        self._ws = {}

    @property
    def n_params(self):
        d0, d1, d2, d3 = self.dims
        return d1 * d0 + d1 + d2 * d1 + d2 + d3 * d2 + d3

    def flat(self):
        """The FP32 weights and biases, flat (W1 b1 W2 b2 W3 b3), a view."""
        return self.params[: 4 * self.n_params].view(torch.float32)

    def unpack(self, flat=None):
        """(W1, b1, W2, b2, W3, b3) views of a flat FP32 vector."""
        d0, d1, d2, d3 = self.dims
        f = self.flat() if flat is None else flat
        out, o = [], 0
        for shape in ((d1, d0), (d1,), (d2, d1), (d2,), (d3, d2), (d3,)):
            k = 1
            for x in shape:
                k *= x
            out.append(f[o:o + k].view(*shape))
            o += k
        return tuple(out)

    def ws(self, rows):
        if rows not in self._ws:
            sz = ctypes.c_size_t(0)
            st = lib().eigen_GPU_mlp_ws_size(*self.dims, rows, ctypes.byref(sz))
            if st != 0:
                raise EigenGError(f"eigen_GPU_mlp_ws_size failed with cudaError {st}")
            self._ws[rows] = torch.empty(sz.value, dtype=torch.uint8, device=self.params.device)
        return self._ws[rows]

    def forward(self, x):
        rows = x.shape[0]
        y = torch.empty((rows, self.dims[3]), dtype=torch.float32, device=x.device)
        ws = self.ws(rows)
        st = lib().eigen_GPU_mlp_forward(*self.dims, _ptr(self.params), rows, _ptr(x), _ptr(y), _ptr(ws), ws.numel(),
                                         _stream(None))
        if st != 0:
            raise EigenGError(f"eigen_GPU_mlp_forward failed with cudaError {st}")
        return y

    def gradient(self, x, t):
        """(flat FP32 gradient of the mean squared error, sum of squared errors)."""
        rows = x.shape[0]
        g = torch.zeros(self.n_params, dtype=torch.float32, device=x.device)
        sse = torch.zeros(1, dtype=torch.float64, device=x.device)
        ws = self.ws(rows)
        st = lib().eigen_GPU_mlp_gradient(*self.dims, _ptr(self.params), rows, _ptr(x), _ptr(t), _ptr(g), _ptr(sse),
                                          _ptr(ws), ws.numel(), _stream(None))
        if st != 0:
            raise EigenGError(f"eigen_GPU_mlp_gradient failed with cudaError {st}")
        return g, sse

    def train_step(self, x, t, lr, sse=None):
        rows = x.shape[0]
        self.step += 1
        ws = self.ws(rows)
        st = lib().eigen_GPU_mlp_train_step(*self.dims, _ptr(self.params), rows, _ptr(x), _ptr(t), float(lr),
                                            self.step, _ptr(sse), _ptr(ws), ws.numel(), _stream(None))
        if st != 0:
            raise EigenGError(f"eigen_GPU_mlp_train_step failed with cudaError {st}")


def family_buffer(a0, e, v0):
    """The family argument of eigen_GPU_batch_learned_FP: A0, E_1..E_4, V0
    (torch tensors, n x n each, symmetric A0 and E_j; V0 with the
    eigenvectors of A0 in its columns), FP32 column-major, back to back."""
    n = a0.shape[0]
    parts = [a0] + [e[j] for j in range(e.shape[0])] + [v0]
    return torch.stack([p.to(torch.float32).t().contiguous().reshape(-1) for p in parts]).reshape(-1).contiguous()


def basis_eigenvectors(a0):
    """V0: eigenvectors of A0 (columns, ascending eigenvalues), by this
    library's FP64 solve; returns an n x n FP64 tensor (row i, column j)."""
    n = a0.shape[0]
    a = a0.to(torch.float64).t().contiguous().reshape(1, n, n).clone()
    w, info = solve(a, n)
    torch.cuda.synchronize()
    if int(info.abs().sum()) != 0:
        raise EigenGError("the solve of A0 did not converge")
    return a[0].t().contiguous()  # a[0][j] is eigenvector j


def family_members(a0, e, theta):
    """A(theta) for each row of theta (L x 4): L x n x n, column-major
    storage of symmetric matrices (identical to row-major)."""
    return (a0[None] + torch.einsum("lj,jik->lik", theta.to(a0.dtype), e)).contiguous()


def targets(v, v0):
    """Training targets of solved members (v: L x n x n eigenvectors as the
    solver returns them, FP32): L x n*n, eigen_GPU_learned_targets_FP."""
    L, n = v.shape[0], v.shape[1]
    c = torch.empty((L, n * n), dtype=torch.float32, device=v.device)
    v0c = v0.to(torch.float32).t().contiguous()  # column-major
    st = lib().eigen_GPU_learned_targets_FP(L, n, _ptr(v), n, _ptr(v0c), _ptr(c), _stream(None))
    if st != 0:
        raise EigenGError(f"eigen_GPU_learned_targets_FP failed with cudaError {st}")
    return c


def features(theta):
    """Network inputs: 10 theta, zero padded to D0 columns."""
    x = torch.zeros((theta.shape[0], D0), dtype=torch.float32, device=theta.device)
    x[:, :theta.shape[1]] = 10.0 * theta.to(torch.float32)
    return x


def make_dataset(a0, e, v0, count, seed, chunk=8192):
    """count solver-generated training pairs: theta ~ U[-0.1, 0.1]^4, the
    members solved by this library's FP64 path, targets V0^T V (signs
    fixed).  Returns (features count x D0, targets count x n*n), FP32."""
    n = a0.shape[0]
    g = torch.Generator(device=a0.device)
    g.manual_seed(seed)
    xs, ts = [], []
    for s in range(0, count, chunk):
        m = min(chunk, count - s)
        th = (torch.rand((m, e.shape[0]), generator=g, device=a0.device, dtype=torch.float64) - 0.5) * 0.2
        a = family_members(a0.to(torch.float64), e.to(torch.float64), th)
        w, info = solve(a, n)
        if int(info.abs().sum()) != 0:
            raise EigenGError("a training solve did not converge")
        xs.append(features(th))
        ts.append(targets(a.to(torch.float32), v0))
    return torch.cat(xs), torch.cat(ts)


def train(mlp, x, t, epochs=20, batch=1024, lr=1e-3, lr_final=1e-5, seed=0, log=None):
    """Adam on minibatches of the dataset (x, t) with the library's train
    step; the learning rate decays geometrically from lr to lr_final.
    Returns the mean squared error of each epoch."""
    count = x.shape[0]
    g = torch.Generator(device=x.device)
    g.manual_seed(seed)
    steps_per_epoch = max(1, count // batch)
    total = epochs * steps_per_epoch
    sse = torch.zeros(1, dtype=torch.float64, device=x.device)
    hist = []
    k = 0
    for ep in range(epochs):
        perm = torch.randperm(count, generator=g, device=x.device)
        sse.zero_()
        for s in range(steps_per_epoch):
            idx = perm[s * batch:(s + 1) * batch]
            rate = lr * (lr_final / lr) ** (k / max(1, total - 1))
            mlp.train_step(x[idx].contiguous(), t[idx].contiguous(), rate, sse)
            k += 1
        mse = float(sse.item()) / (steps_per_epoch * batch * t.shape[1])
        hist.append(mse)
        if log:
            log(f"epoch {ep}: mse {mse:.3e}")
    return hist


def learned_workspace(L, nm, n, mlp_dims, opts=None, device=None):
    sz = ctypes.c_size_t(0)
    o = opts if opts is not None else LearnedOpts(WARM_NETWORK, 0, 0.0, 0.0, 1, 0)
    st = lib().eigen_GPU_batch_learned_BufferSize_FP(L, nm, n, mlp_dims[1], mlp_dims[2], ctypes.byref(o),
                                                     ctypes.byref(sz))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_learned_BufferSize_FP failed with cudaError {st}")
    return torch.empty(max(sz.value, 16), dtype=torch.uint8, device=device or "cuda")


def solve_learned(a, n, family, mlp=None, warm=WARM_NETWORK, max_sweeps=0, tol=0.0, jacobi_tol=0.0, fallback=True,
                  chunk=0, wk=None, stream=None, d1=512, d2=512):
    """eigen_GPU_batch_learned_FP on the FP32 batch a (L x n x n, in place):
    returns (w, info, sweeps, resid)."""
    L = a.numel() // (n * n)
    if a.dtype != torch.float32 or not a.is_cuda or not a.is_contiguous():
        raise EigenGError("a must be a contiguous FP32 CUDA tensor")
    if mlp is not None:
        d1, d2 = mlp.dims[1], mlp.dims[2]
    o = LearnedOpts(warm, max_sweeps, tol, jacobi_tol, 1 if fallback else 0, chunk)
    if wk is None:
        wk = learned_workspace(L, n, n, (D0, d1, d2, n * n), o, a.device)
    w = torch.empty((L, n), dtype=torch.float32, device=a.device)
    info = torch.zeros(L, dtype=torch.int32, device=a.device)
    sweeps = torch.zeros(L, dtype=torch.int32, device=a.device)
    resid = torch.zeros(L, dtype=torch.float64, device=a.device)
    st = lib().eigen_GPU_batch_learned_FP(L, n, n, _ptr(a), _ptr(w), _ptr(family),
                                          _ptr(mlp.params if mlp is not None else None), d1, d2, _ptr(wk), wk.numel(),
                                          _ptr(info), _ptr(sweeps), _ptr(resid), ctypes.byref(o), _stream(stream))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_learned_FP failed with cudaError {st}")
    return w, info, sweeps, resid
