"""Parity of the CUDA library (through its C ABI) with the CPU oracle and
with FP64 LAPACK, on seeded inputs.

Tolerances (floating point; the index work -- the DO_SORT permutation -- is
checked bit-exactly):
  * eigenvalues: |w_gpu - w_oracle| <= 64 * n * eps_T * max|w|
  * eigenvectors: sign-invariant, 1 - |<v_gpu, v_oracle>| <= C * eps_T * n * max|w| / gap
  * residual and orthogonality: the reference's own gate
    (eigen_GPU_check.cu:65-74) run on the device, no flags allowed.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

DT = {np.float64: torch.float64, np.float32: torch.float32}


def E():
    import eigeng_b200
    return eigeng_b200


def gpu_solve(a0, n, nm=None, method=0, sort=True, max_sweep=100, rec_cap=0, chunk=0, split=0, zmem=0):
    a = torch.from_numpy(np.ascontiguousarray(a0)).cuda()
    w, info = E().solve(a, n, nm, method=method, sort=sort, max_sweep=max_sweep, rec_cap=rec_cap, chunk=chunk,
                        split=split, zmem=zmem)
    torch.cuda.synchronize()
    return w.cpu().numpy(), a.cpu().numpy(), info.cpu().numpy()


def device_gate(a0, w, z, n, nm=None):
    e1, e2, fl = E().check(torch.from_numpy(np.ascontiguousarray(a0)).cuda(),
                           torch.from_numpy(np.ascontiguousarray(w)).cuda(),
                           torch.from_numpy(np.ascontiguousarray(z)).cuda(), n, nm)
    torch.cuda.synchronize()
    return e1.cpu().numpy(), e2.cpu().numpy(), fl.cpu().numpy()


def assert_vectors_match(z_gpu, z_ref, w_ref, n, eps, c=256.0):
    scale = np.abs(w_ref).max(axis=1)
    for k in range(z_gpu.shape[0]):
        wl = np.sort(w_ref[k])
        gaps = np.minimum(np.diff(wl, prepend=-np.inf), np.diff(wl, append=np.inf))
        for j in range(n):
            dot = abs(float(np.dot(z_gpu[k, j, :n].astype(np.float64), z_ref[k, j, :n].astype(np.float64))))
            bound = c * eps * n * scale[k] / max(gaps[j], 1e-300)
            assert 1.0 - dot <= max(bound, 100 * eps * n), (k, j, dot, bound)


SIZES = [2, 3, 4, 5, 7, 8, 9, 15, 16, 17, 24, 31, 32, 33, 40, 47, 48, 63, 64, 65, 96, 100, 127, 128, 129, 160,
         161, 200, 256]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("method", [0, 1])
def test_parity_with_oracle(oracle_mod, n, dtype, method):
    O = oracle_mod
    L = 6 if n <= 128 else 3
    a0 = O.sym_uniform(L, n, seed=1000 + n).astype(dtype)
    w, z, info = gpu_solve(a0, n, method=method)
    assert (info == 0).all()
    ao = a0.copy()
    wo, info_o, _ = O.eigen_batch(ao, n, method=method)
    eps = np.finfo(dtype).eps
    scale = np.abs(wo).max(axis=1, keepdims=True)
    assert (np.abs(w - wo) <= 64 * n * eps * scale).all()
    assert (np.diff(w, axis=1) >= 0).all()  # DO_SORT: ascending
    assert_vectors_match(z, ao, wo, n, eps)
    e1, e2, fl = device_gate(a0, w, z, n)
    assert (fl == 0).all(), (e1, e2)
    if dtype == np.float64:
        wl, _ = O.lapack_eigh(a0, n)
        assert (np.abs(w - wl) <= 64 * n * eps * scale).all()
        res, orth = O.residuals(a0, w, z, n)
        assert res.max() < 2e-11 and orth.max() < 2e-11


@pytest.mark.parametrize("n,dtype", [(1024, np.float64), (1024, np.float32), (700, np.float64), (513, np.float64)])
def test_largest_sizes(oracle_mod, n, dtype):
    """Up to the size limit n = 1024: Z kept in the workspace (large FP64),
    several row blocks per matrix in shared memory, two rows per thread,
    phase 1 with most of the matrix outside shared memory."""
    O = oracle_mod
    a0 = O.sym_uniform(2, n, seed=n).astype(dtype)
    w, z, info = gpu_solve(a0, n)
    assert (info == 0).all()
    eps = np.finfo(dtype).eps
    wl, _ = O.lapack_eigh(a0.astype(np.float64), n)
    scale = np.abs(wl).max(axis=1, keepdims=True)
    assert (np.abs(w - wl) <= 64 * n * eps * scale).all()
    res, orth = O.residuals(a0.astype(np.float64), w.astype(np.float64), z.astype(np.float64), n)
    assert res.max() < 256 * n * eps and orth.max() < 256 * n * eps, (res.max(), orth.max())
    e1, e2, fl = device_gate(a0, w, z, n)
    assert (fl == 0).all(), (e1, e2)


@pytest.mark.parametrize("n", [4, 16, 32, 33, 64, 128])
def test_families_pass_reference_gate(oracle_mod, n):
    O = oracle_mod
    for a0 in (O.letkf_like(8, n, seed=5), O.ref_matrices(4, n, O.REF_LETKF), O.ref_matrices(4, n, O.REF_FRANK),
               O.ref_matrices(4, n, O.REF_SYM_RAND), O.logspaced_spectrum(4, n, seed=9)):
        for dt in (np.float64, np.float32):
            a = a0.astype(dt)
            w, z, info = gpu_solve(a, n)
            assert (info == 0).all()
            e1, e2, fl = device_gate(a, w, z, n)
            assert (fl == 0).all(), (n, dt, e1, e2)


def _sort_cases(n, dtype):
    rng = np.random.default_rng(n)
    cases = [np.eye(n)[None].repeat(2, 0)]                          # all eigenvalues tie
    dg = np.zeros((2, n, n))
    vals = np.round(rng.uniform(-3, 3, size=(2, n)))                 # many exact ties
    for k in range(2):
        dg[k] = np.diag(vals[k])
    cases.append(dg)
    b = rng.uniform(-1, 1, size=(2, n, n))
    cases.append(0.5 * (b + b.transpose(0, 2, 1)))                   # distinct
    return [np.ascontiguousarray(c.astype(dtype)) for c in cases]


@pytest.mark.parametrize("n", [3, 8, 17, 32, 33, 50, 128])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_sort_permutation_bit_exact(oracle_mod, n, dtype):
    """DO_SORT ordering/indexing is bit-exact: for the eigenvalues the solver
    computed (sort off), the sorted run returns exactly w[pos] and the
    columns z[:, pos] where pos is the reference's selection sort
    (tql2_tiled.hpp:149-176) of those values, ties included."""
    O = oracle_mod
    for a0 in _sort_cases(n, dtype):
        wu, zu, _ = gpu_solve(a0, n, sort=False)
        ws, zs, _ = gpu_solve(a0, n, sort=True)
        for k in range(a0.shape[0]):
            srt, pos = O.select_sort(wu[k])
            assert np.array_equal(ws[k], srt)
            assert np.array_equal(zs[k], zu[k][pos])


@pytest.mark.parametrize("n", [5, 16, 32])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_jacobi_parity(oracle_mod, n, dtype):
    O = oracle_mod
    a0 = O.sym_uniform(8, n, seed=77 + n).astype(dtype)
    for sort in (False, True):
        w, z, info = gpu_solve(a0, n, method=2, sort=sort)
        ao = a0.copy()
        wo, info_o, _ = O.eigen_batch(ao, n, method=2, sort=sort)
        assert (info == 0).all() and (info_o == 0).all()
        eps = np.finfo(dtype).eps
        scale = np.abs(wo).max(axis=1, keepdims=True)
        ws, wos = np.sort(w, axis=1), np.sort(wo, axis=1)
        assert (np.abs(ws - wos) <= 64 * n * eps * scale).all()
        if sort:
            # the reference gate scales by max(|w_1|, |w_n|), which assumes
            # ascending eigenvalues (eigen_GPU_check.cu:65-70)
            e1, e2, fl = device_gate(a0, w, z, n)
            assert (fl == 0).all()
            assert_vectors_match(z, ao, wo, n, eps)
        else:
            res, orth = O.residuals(a0, w, z, n)
            assert res.max() <= 100 * n * eps and orth.max() <= 100 * n * eps


@pytest.mark.parametrize("n,nm", [(7, 8), (31, 32), (33, 34), (65, 70), (200, 201)])
def test_leading_dimension_and_lower_triangle(oracle_mod, n, nm):
    """nm > n padding rows are left untouched and the strict lower triangle
    is never read (eigen_GPU_batch.cu contract: upper triangle only)."""
    O = oracle_mod
    L = 3
    base = O.sym_uniform(L, n, seed=n)
    a0 = np.full((L, n, nm), 7.25)
    a0[:, :, :n] = base
    junk = a0.copy()
    for k in range(L):
        for j in range(n):
            junk[k, j, j + 1:n] = np.nan  # a(i, j) with i > j: strict lower triangle
    w1, z1, _ = gpu_solve(a0, n, nm)
    w2, z2, _ = gpu_solve(junk, n, nm)
    assert np.array_equal(w1, w2) and np.array_equal(z1, z2)
    assert (z1[:, :, n:] == 7.25).all()
    wo, _, _ = O.eigen_batch(base.copy(), n)
    assert np.abs(w1 - wo).max() <= 64 * n * np.finfo(np.float64).eps * np.abs(wo).max()


def test_n1_and_n2(oracle_mod):
    a = np.array([[[3.5]], [[-2.0]]])
    w, z, info = gpu_solve(a, 1)
    assert np.array_equal(w[:, 0], [3.5, -2.0]) and (z == 1.0).all()
    a2 = np.array([[[2.0, 1.0], [1.0, 2.0]], [[0.0, 0.0], [0.0, 0.0]], [[1.0, 0.0], [0.0, -1.0]]])
    w, z, info = gpu_solve(a2, 2)
    assert np.allclose(w, [[1.0, 3.0], [0.0, 0.0], [-1.0, 1.0]], atol=1e-15)
    e1, e2, fl = device_gate(a2, w, z, 2)
    assert (fl == 0).all()


def test_dropin_abi_and_size_query():
    """eigen_GPU_batch_DP / _FP exactly as the reference is called
    (README:77-88): size query through w, then the solve."""
    import eigeng_b200 as e
    for dt, tdt in ((np.float64, torch.float64), (np.float32, torch.float32)):
        for n in (1, 20, 64):
            L = 10
            q = e.query_lwork(L, n, n, n, tdt)
            assert q == e.buffer_size(L, n, n, n, tdt)
            if n == 1:
                assert q == 0
                continue
            rng = np.random.default_rng(n)
            b = rng.uniform(-1, 1, size=(L, n, n))
            a0 = (0.5 * (b + b.transpose(0, 2, 1))).astype(dt)
            a = torch.from_numpy(a0).cuda()
            w = torch.empty((L, n), dtype=tdt, device="cuda")
            wk = torch.empty(q, dtype=torch.uint8, device="cuda")
            e.eigen_GPU_batch(a, w, wk, n)
            w2, z2, _ = gpu_solve(a0, n)
            torch.cuda.synchronize()
            assert np.array_equal(w.cpu().numpy(), w2) and np.array_equal(a.cpu().numpy(), z2)


def test_reference_check_api_writes_flags():
    """eigen_GPU_check_DP keeps the reference's contract: the verdict goes
    into the first four floats of each matrix of the input copy."""
    import ctypes
    import eigeng_b200 as e
    n, L = 16, 4
    rng = np.random.default_rng(1)
    b = rng.uniform(-1, 1, size=(L, n, n))
    a0 = 0.5 * (b + b.transpose(0, 2, 1))
    w, z, _ = gpu_solve(a0, n)
    z_bad = z.copy()
    z_bad[2, 3] += 0.5 * z_bad[2, 4]  # mix two eigenvectors of matrix 2
    ad = torch.from_numpy(a0.copy()).cuda()
    wd = torch.from_numpy(w).cuda()
    zd = torch.from_numpy(z_bad).cuda()
    e.lib().eigen_GPU_check_DP(L, n, n, n, ctypes.c_void_p(ad.data_ptr()), ctypes.c_void_p(wd.data_ptr()),
                              ctypes.c_void_p(zd.data_ptr()), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    flags = ad.view(torch.float32).reshape(L, -1)[:, :4].cpu().numpy()
    assert (flags[[0, 1, 3], :2] == 0).all()
    assert flags[2, 0] > 0 and flags[2, 1] > 0


@pytest.mark.parametrize("n,nm,m", [(20, 20, 20), (30, 33, 17), (40, 43, 40), (48, 50, 31), (64, 64, 64),
                                     (100, 100, 77), (128, 130, 128), (200, 201, 200)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_gate_norms_match_numpy(oracle_mod, n, nm, m, dtype):
    """eigen_GPU_check_ex (one warp per matrix for n <= 32, one CTA per
    matrix for n <= 64, 128 x 128 tiles above, all on the FP64 tensor
    cores): ||A Z - Z D||_F over the first m pairs and ||Z^T Z - I||_F
    (m x m) in FP64, on eigenvectors perturbed by ~1e-6 so that the norms
    are far above rounding; m < n and padded leading dimensions in each
    form."""
    import ctypes
    import eigeng_b200 as e
    O = oracle_mod
    L = 5
    a0 = np.zeros((L, n, nm))
    a0[:, :, :n] = O.sym_uniform(L, n, seed=n + 1)
    w, z, _ = gpu_solve(a0.astype(dtype), n, nm)
    rng = np.random.default_rng(n)
    zp = (z.astype(np.float64) + 1e-6 * rng.standard_normal(z.shape)).astype(dtype)
    ad = torch.from_numpy(a0.astype(dtype)).cuda()
    wd = torch.from_numpy(w).cuda()
    zd = torch.from_numpy(np.ascontiguousarray(zp)).cuda()
    e1 = torch.empty(L, dtype=torch.float64, device="cuda")
    e2 = torch.empty(L, dtype=torch.float64, device="cuda")
    fl = torch.empty(L, dtype=torch.int32, device="cuda")
    sfx = "DP" if dtype == np.float64 else "FP"
    P = ctypes.c_void_p
    st = getattr(e.lib(), "eigen_GPU_check_ex_" + sfx)(L, nm, n, m, P(ad.data_ptr()), P(wd.data_ptr()),
                                                       P(zd.data_ptr()), P(e1.data_ptr()), P(e2.data_ptr()),
                                                       P(fl.data_ptr()), P(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert st == 0
    A = np.transpose(a0.astype(dtype).astype(np.float64), (0, 2, 1))[:, :n, :n]
    A = np.triu(A) + np.transpose(np.triu(A, 1), (0, 2, 1))
    Z = np.transpose(zp.astype(np.float64), (0, 2, 1))[:, :n, :m]
    D = w.astype(np.float64)[:, :m]
    r1 = np.linalg.norm(A @ Z - Z * D[:, None, :], axis=(1, 2))
    r2 = np.linalg.norm(np.transpose(Z, (0, 2, 1)) @ Z - np.eye(m)[None], axis=(1, 2))
    assert np.allclose(e1.cpu().numpy(), r1, rtol=1e-6) and np.allclose(e2.cpu().numpy(), r2, rtol=1e-6)


def test_invalid_arguments_rejected():
    import eigeng_b200 as e
    a = torch.zeros((2, 8, 8), dtype=torch.float64, device="cuda")
    w = torch.zeros((2, 8), dtype=torch.float64, device="cuda")
    wk = e.workspace(2, 8, 8, torch.float64)
    INVALID = 1  # cudaErrorInvalidValue
    assert e.eigen_GPU_batch_ex(a, w, wk, 8, 8, 9) == INVALID           # m > n
    assert e.eigen_GPU_batch_ex(a, w, wk[:16], 8) == INVALID            # workspace too small
    assert e.eigen_GPU_batch_ex(a, w, None, 8) == INVALID               # no workspace
    assert e.eigen_GPU_batch_ex(a, w, wk, 8, method=7) == INVALID       # unknown method
    big = torch.zeros((1, 40, 40), dtype=torch.float64, device="cuda")
    assert e.eigen_GPU_batch_ex(big, w, None, 40, method=e.JACOBI) == INVALID  # Jacobi is n <= 32
    torch.cuda.synchronize()


@pytest.mark.parametrize("n", [6, 40])
def test_nan_input_reports_status_and_terminates(oracle_mod, n):
    O = oracle_mod
    a0 = O.sym_uniform(3, n, seed=2)
    a0[1, 2, 1] = np.nan  # a(1, 2) in the upper triangle
    w, z, info = gpu_solve(a0, n)
    assert info[1] != 0 and info[0] == 0 and info[2] == 0
    ao = a0.copy()
    wo, io, _ = O.eigen_batch(ao, n)
    assert np.abs(w[[0, 2]] - wo[[0, 2]]).max() <= 64 * n * 2.3e-16 * np.abs(wo[[0, 2]]).max()


@pytest.mark.parametrize("n", [12, 32, 48, 128])
@pytest.mark.parametrize("method", [0, 1])
def test_record_overflow_path_is_identical(oracle_mod, n, method):
    """With a tiny record capacity every matrix takes the in-kernel
    regeneration path; the rotations and hence the results are identical."""
    O = oracle_mod
    a0 = O.sym_uniform(5, n, seed=31)
    w1, z1, i1 = gpu_solve(a0, n, method=method)
    w2, z2, i2 = gpu_solve(a0, n, method=method, rec_cap=16)
    assert np.array_equal(i1, i2)
    assert np.array_equal(w1, w2)
    assert np.array_equal(z1, z2)


@pytest.mark.parametrize("n,nm", [(40, 40), (100, 103), (200, 200), (256, 256)])
def test_apply_row_split_is_bit_identical(oracle_mod, n, nm):
    """The apply phase may split a matrix's rows over several thread blocks
    (each applies every rotation to its own rows): results do not depend
    on the split, with or without the in-kernel regeneration path."""
    O = oracle_mod
    a0 = np.zeros((6, n, nm))
    a0[:, :, :n] = O.sym_uniform(6, n, seed=n + 3)
    w1, z1, i1 = gpu_solve(a0, n, nm)
    for split in (2, 3, 5):
        w2, z2, i2 = gpu_solve(a0, n, nm, split=split)
        assert np.array_equal(w1, w2) and np.array_equal(z1, z2) and np.array_equal(i1, i2), split
    w3, z3, i3 = gpu_solve(a0, n, nm, split=3, rec_cap=4 * n)   # records overflow: regenerated per block
    assert np.array_equal(w1, w3) and np.array_equal(z1, z3) and np.array_equal(i1, i3)


@pytest.mark.parametrize("n,nm,dtype", [(33, 33, np.float64), (64, 64, np.float64), (100, 103, np.float64),
                                        (128, 128, np.float64), (129, 130, np.float64), (200, 200, np.float64),
                                        (256, 256, np.float64), (40, 40, np.float32), (128, 128, np.float32),
                                        (300, 301, np.float32), (512, 512, np.float32)])
def test_tensor_memory_apply_is_bit_identical(oracle_mod, n, nm, dtype):
    """Where a row fits, the apply phase keeps Z in tensor memory (one row
    per TMEM lane) with the operations of the shared-memory form, in the
    same order: results agree bit for bit with the shared-memory form, with
    a row split and with the in-kernel regeneration path too."""
    O = oracle_mod
    a0 = np.zeros((5, n, nm), dtype)
    a0[:, :, :n] = O.sym_uniform(5, n, seed=n + 11).astype(dtype)
    shared = E().ZMEM_SHARED
    w1, z1, i1 = gpu_solve(a0, n, nm, zmem=shared)
    w2, z2, i2 = gpu_solve(a0, n, nm)
    assert np.array_equal(w1, w2) and np.array_equal(z1, z2) and np.array_equal(i1, i2)
    w3, z3, i3 = gpu_solve(a0, n, nm, split=3)
    assert np.array_equal(w1, w3) and np.array_equal(z1, z3) and np.array_equal(i1, i3)
    w4, z4, i4 = gpu_solve(a0, n, nm, rec_cap=4 * n)   # records overflow: regenerated in the kernel
    w5, z5, i5 = gpu_solve(a0, n, nm, rec_cap=4 * n, zmem=shared)
    assert np.array_equal(w4, w5) and np.array_equal(z4, z5) and np.array_equal(i4, i5)
    assert np.array_equal(w1, w4) and np.array_equal(z1, z4)


def test_chunked_batch_and_determinism(oracle_mod):
    """Batches split into several workspace chunks (including a ragged last
    chunk) give the same results as one chunk, and identical matrices give
    identical results."""
    O = oracle_mod
    for n, L, chunk in ((20, 23, 5), (70, 11, 4), (200, 5, 2)):
        a0 = O.sym_uniform(L, n, seed=n)
        a0[3] = a0[0]
        w1, z1, i1 = gpu_solve(a0, n)
        w2, z2, i2 = gpu_solve(a0, n, chunk=chunk)
        assert np.array_equal(w1, w2) and np.array_equal(z1, z2) and np.array_equal(i1, i2)
        assert np.array_equal(w1[3], w1[0]) and np.array_equal(z1[3], z1[0])


def test_solve_host_matches_device_solve(oracle_mod):
    """solve_host (host buffers, chunks solved concurrently on their own
    streams) gives exactly the device solve's results, with a ragged last
    chunk and padding rows."""
    O = oracle_mod
    n, nm, L = 48, 50, 37
    a0 = np.zeros((L, n, nm))
    a0[:, :, :n] = O.sym_uniform(L, n, seed=11)
    w1, z1, _ = gpu_solve(a0, n, nm)
    ah = torch.from_numpy(a0.copy()).pin_memory()
    wh = E().solve_host(ah, n, nm, chunk=10)
    torch.cuda.synchronize()
    assert np.array_equal(wh.numpy(), w1)
    assert np.array_equal(ah.numpy()[:, :, :n], z1[:, :, :n])
    af = torch.from_numpy(a0.astype(np.float32))             # not pinned: copies still complete
    wf = E().solve_host(af, n, nm)
    torch.cuda.synchronize()
    w2, _, _ = gpu_solve(a0.astype(np.float32), n, nm)
    assert np.array_equal(wf.numpy(), w2)


@pytest.mark.parametrize("n,L,chunk", [(48, 37, 2), (16, 4096, 0)])
def test_solve_host_buffer_reuse_and_status(oracle_mod, n, L, chunk):
    """More chunks than the ten device buffers (each buffer, and its status
    buffer, reused after its copy-out; each of the eight streams' workspace
    reused by the stream's next chunk), and the default 17-chunk schedule of
    a batch of 2048 or more with the QL phase at eight matrices per warp:
    bit for bit the device solve, status copied back per matrix.  One matrix
    carries a NaN, which QL reports in its status."""
    O = oracle_mod
    a0 = O.sym_uniform(L, n, seed=23)
    bad = L // 3
    a0[bad, 1, 0] = a0[bad, 0, 1] = np.nan
    w1, z1, i1 = gpu_solve(a0, n)
    ah = torch.from_numpy(a0.copy()).pin_memory()
    ih = torch.full((L,), -5, dtype=torch.int32).pin_memory()
    wh = E().solve_host(ah, n, chunk=chunk, info_host=ih)
    torch.cuda.synchronize()
    ok = np.arange(L) != bad
    assert np.array_equal(ih.numpy(), i1)
    assert i1[bad] != 0 and (i1[ok] == 0).all()
    assert np.array_equal(wh.numpy()[ok], w1[ok])
    assert np.array_equal(ah.numpy()[ok], z1[ok])


def _stage_parts(a0, n, nm, dtype, method):
    """Solves a0 with eigen_GPU_batch_stage_*: the reductions in two parts on
    two streams, the QL phase over the whole batch, the apply phase in three
    parts."""
    e = E()
    L = a0.shape[0]
    a = torch.from_numpy(np.ascontiguousarray(a0)).cuda()
    w = torch.zeros((L, n), dtype=DT[dtype], device="cuda")
    info = torch.full((L,), -7, dtype=torch.int32, device="cuda")
    wk = e.workspace(L, nm, n, DT[dtype], chunk=L)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    torch.cuda.synchronize()
    assert e.stage(a, w, wk, n, e.STAGE_REDUCE, 0, 5, nm=nm, info=info, method=method, stream=s1) == 0
    assert e.stage(a, w, wk, n, e.STAGE_REDUCE, 5, 0, nm=nm, info=info, method=method, stream=s2) == 0
    s1.wait_stream(s2)
    assert e.stage(a, w, wk, n, e.STAGE_QL, 0, 0, nm=nm, info=info, method=method, stream=s1) == 0
    for c0, c1 in ((0, 2), (2, 9), (9, L)):
        assert e.stage(a, w, wk, n, e.STAGE_APPLY, c0, c1 - c0, nm=nm, info=info, method=method, stream=s1) == 0
    torch.cuda.synchronize()
    return w.cpu().numpy(), a.cpu().numpy(), info.cpu().numpy()


@pytest.mark.parametrize("n,nm,method", [(1, 1, 0), (20, 20, 0), (20, 21, 2), (48, 50, 0), (48, 48, 1),
                                         (128, 128, 0), (200, 201, 0)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_stage_parts_match_whole_solve(oracle_mod, n, nm, method, dtype):
    """The phases run in parts (eigen_GPU_batch_stage_*), split differently
    per phase and on two streams, give the one-call solve's results bit for
    bit (warp, register, shared/tensor-memory paths; Jacobi and n = 1 run at
    the apply part)."""
    O = oracle_mod
    L = 13
    a0 = np.zeros((L, n, nm), dtype=dtype)
    a0[:, :, :n] = O.sym_uniform(L, n, seed=n + nm).astype(dtype)
    w1, z1, i1 = gpu_solve(a0, n, nm, method=method)
    w2, z2, i2 = _stage_parts(a0, n, nm, dtype, method)
    assert np.array_equal(w1, w2) and np.array_equal(z1, z2) and np.array_equal(i1, i2)


def test_stage_rejects_bad_parts():
    import ctypes
    e = E()
    L, n = 6, 40
    a = torch.zeros((L, n, n), dtype=torch.float64, device="cuda")
    w = torch.zeros((L, n), dtype=torch.float64, device="cuda")
    wk = e.workspace(L, n, n, torch.float64, chunk=L)
    INVALID = 1  # cudaErrorInvalidValue
    assert e.stage(a, w, wk, n, e.STAGE_REDUCE, 4, 3) == INVALID     # past the end of the batch
    assert e.stage(a, w, wk, n, e.STAGE_REDUCE, -1, 2) == INVALID    # negative first
    assert e.stage(a, w, wk, n, 0, 0, 2) == INVALID                  # no phase
    assert e.stage(a, w, wk, n, 8, 0, 2) == INVALID                  # unknown phase bit
    assert e.stage(a, w, wk[:64], n, e.STAGE_REDUCE, 0, 2) == INVALID  # workspace too small
    # a plan that keeps the batch in several chunks cannot run a part
    o = e.Opts(0, 1, 100, 0, 2, 0, 0)
    st = e.lib().eigen_GPU_batch_stage_DP(L, n, n, n, a.data_ptr(), w.data_ptr(), wk.data_ptr(),
                                          wk.numel(), None, ctypes.byref(o), e.STAGE_REDUCE, 0, 2, None)
    assert st == INVALID
    torch.cuda.synchronize()


@pytest.mark.parametrize("n,dtype", [(20, np.float64), (64, np.float32), (128, np.float64)])
def test_ql_matrices_per_warp_bit_identical(oracle_mod, n, dtype):
    """opts.ql_mpw (QL matrices per warp) changes only the launch: every
    power of two up to 32 gives the automatic choice's results; other
    values are rejected."""
    O = oracle_mod
    e = E()
    L = 37
    a0 = O.sym_uniform(L, n, seed=3 * n).astype(dtype)
    w1, z1, i1 = gpu_solve(a0, n)
    for q in (1, 2, 4, 8, 16, 32):
        a = torch.from_numpy(np.ascontiguousarray(a0)).cuda()
        w = torch.empty((L, n), dtype=DT[dtype], device="cuda")
        info = torch.zeros(L, dtype=torch.int32, device="cuda")
        wk = e.workspace(L, n, n, DT[dtype])
        assert e.eigen_GPU_batch_ex(a, w, wk, n, info=info, ql_mpw=q) == 0
        torch.cuda.synchronize()
        assert np.array_equal(w.cpu().numpy(), w1) and np.array_equal(a.cpu().numpy(), z1), q
        assert np.array_equal(info.cpu().numpy(), i1)
    for q in (3, 64):
        assert e.eigen_GPU_batch_ex(a, w, wk, n, ql_mpw=q) == 1  # cudaErrorInvalidValue
    torch.cuda.synchronize()
