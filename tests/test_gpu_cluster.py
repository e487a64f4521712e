"""Phase 1 on a thread-block cluster (k1_cl: the matrix in the cluster's
distributed shared memory, 32 < n <= 512) against the oracle and FP64
LAPACK, with the one-CTA forms forced for comparison through the tuned
options' `reduce` entry.  Same tolerances as test_gpu_parity: eigenvalues
within 64 n eps max|w| of the oracle, eigenvectors by the gap-scaled dot
product bound, the reference's gate without flags, and for FP64 residual
and orthogonality below 2e-11."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from test_gpu_parity import assert_vectors_match, device_gate, gpu_solve  # noqa: E402


def E():
    import eigeng_b200
    return eigeng_b200


def _forced(n, dtype, reduce):
    return [dict(esize=8 if dtype == np.float64 else 4, n=n, split=0, zmem=0, ql_mpw=0, reduce=reduce)]


@pytest.mark.parametrize("n", [33, 64, 65, 100, 128, 129, 200, 256, 300, 384, 400, 512])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_cluster_form_parity(oracle_mod, n, dtype):
    O = oracle_mod
    L = 4 if n <= 256 else 2
    a0 = O.sym_uniform(L, n, seed=3000 + n).astype(dtype)
    E().tune_set(_forced(n, dtype, E().REDUCE_CLUSTER))
    try:
        w, z, info = gpu_solve(a0, n)
    finally:
        E().tune_set([])
    assert (info == 0).all()
    ao = a0.copy()
    wo, _, _ = O.eigen_batch(ao, n)
    eps = np.finfo(dtype).eps
    scale = np.abs(wo).max(axis=1, keepdims=True)
    assert (np.abs(w - wo) <= 64 * n * eps * scale).all()
    assert (np.diff(w, axis=1) >= 0).all()
    assert_vectors_match(z, ao, wo, n, eps)
    e1, e2, fl = device_gate(a0, w, z, n)
    assert (fl == 0).all(), (e1, e2)
    if dtype == np.float64:
        res, orth = O.residuals(a0, w, z, n)
        assert res.max() < 2e-11 and orth.max() < 2e-11, (res.max(), orth.max())


@pytest.mark.parametrize("n", [129, 256, 512])
def test_cta_form_through_the_table(oracle_mod, n):
    """The one-CTA form (shared memory plus a band in global memory), also
    the automatic choice, asked for through the table."""
    O = oracle_mod
    a0 = O.sym_uniform(2, n, seed=4000 + n)
    E().tune_set(_forced(n, np.float64, E().REDUCE_CTA))
    try:
        w, z, info = gpu_solve(a0, n)
    finally:
        E().tune_set([])
    assert (info == 0).all()
    res, orth = O.residuals(a0, w, z, n)
    assert res.max() < 2e-11 and orth.max() < 2e-11


@pytest.mark.parametrize("n", [140, 256])
def test_cluster_form_families_and_packed(oracle_mod, n):
    """The reference's matrix families through the cluster form, from the
    full and from the packed upper-triangle input, pass the gate."""
    O = oracle_mod
    E().tune_set(_forced(n, np.float64, E().REDUCE_CLUSTER))
    try:
        for a0 in (O.letkf_like(4, n, seed=5), O.ref_matrices(2, n, O.REF_FRANK), O.logspaced_spectrum(4, n, seed=9),
                   O.clustered_spectrum(2, n, seed=4)):
            w, z, info = gpu_solve(a0, n)
            assert (info == 0).all()
            e1, e2, fl = device_gate(a0, w, z, n)
            assert (fl == 0).all(), (n, e1, e2)
            ap = E().pack_upper(torch.from_numpy(np.ascontiguousarray(a0)).cuda(), n)
            zp, wp, ip = E().solve_packed(ap, n)
            torch.cuda.synchronize()
            assert torch.equal(wp.cpu(), torch.from_numpy(w)) and np.array_equal(zp.cpu().numpy(), z)
    finally:
        E().tune_set([])
