"""Fixtures from the reference's own GPU build (EigenG-Batched, default tql2
+ DO_SORT, compiled for sm_100a; tests/golden/make_ref_golden.py) pin both
the CPU oracle and the CUDA library to the reference's actual outputs:
eigenvalues within 64 n eps max|w|, eigenvectors sign-invariant within a
gap-scaled bound, identical ascending order."""
import importlib.util
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "ref_gpu_golden.npz")


def _mk():
    spec = importlib.util.spec_from_file_location("make_ref_golden", os.path.join(HERE, "golden", "make_ref_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _cases():
    m = _mk()
    return [(k, n, a0) for k, n, a0 in m.cases()]


CASES = None


def cases():
    global CASES
    if CASES is None:
        CASES = _cases()
    return CASES


@pytest.fixture(scope="module")
def fixtures():
    return np.load(FIX)


def _check_against(ref_w, ref_z, w, z, n, dtype):
    eps = np.finfo(dtype).eps
    scale = np.maximum(np.abs(ref_w).max(axis=1), np.finfo(np.float64).tiny)
    assert (np.abs(w - ref_w).max(axis=1) <= 64 * n * eps * scale).all()
    for k in range(ref_w.shape[0]):
        wl = ref_w[k].astype(np.float64)
        gaps = np.minimum(np.diff(wl, prepend=-np.inf), np.diff(wl, append=np.inf))
        for j in range(n):
            dot = abs(float(np.dot(z[k, j, :n].astype(np.float64), ref_z[k, j, :n].astype(np.float64))))
            bound = 512 * eps * n * scale[k] / max(gaps[j], 1e-300)
            assert 1.0 - dot <= max(bound, 200 * eps * n), (k, j, dot, bound)


def test_fixture_inputs_regenerate_exactly(fixtures):
    m = _mk()
    for key, n, a0 in cases():
        assert str(fixtures[key + "__sha"]) == m.sha(a0), key


@pytest.mark.parametrize("idx", range(88))
def test_oracle_matches_reference_gpu_build(oracle_mod, fixtures, idx):
    key, n, a0 = cases()[idx]
    O = oracle_mod
    ref_w, ref_z = fixtures[key + "__w"], fixtures[key + "__z"]
    a = a0.copy()
    w, info, _ = O.eigen_batch(a, n)
    assert (info == 0).all()
    _check_against(ref_w, ref_z, w, a, n, a0.dtype)
    # the reference's own output passes its own gate
    e1, e2, fl = O.check(a0, ref_w, ref_z, n)
    assert (fl == 0).all(), (key, e1, e2)


@pytest.mark.gpu
def test_cuda_library_matches_reference_gpu_build(fixtures):
    import torch
    import eigeng_b200 as E
    for key, n, a0 in cases():
        a = torch.from_numpy(a0.copy()).cuda()
        w, info = E.solve(a, n)
        torch.cuda.synchronize()
        assert (info.cpu().numpy() == 0).all(), key
        _check_against(fixtures[key + "__w"], fixtures[key + "__z"], w.cpu().numpy(), a.cpu().numpy(), n, a0.dtype)


# ---------------------------------------------------------------------------
# The "ext" set: the reference's USE_IMTQL 1 build (imtql2 + DO_SORT) at
# n = 3 .. 256, and its default build at n = 256 (the warp-per-matrix
# hhsy2tr_ / tql2_ / hhtr2sy_ path, eigen_GPU_batch.cu:138-245).

FIX_EXT = os.path.join(HERE, "golden", "ref_gpu_golden_ext.npz")
EXT = None


def ext_cases():
    global EXT
    if EXT is None:
        EXT = list(_mk().ext_cases())
    return EXT


@pytest.fixture(scope="module")
def fixtures_ext():
    if not os.path.exists(FIX_EXT):
        pytest.skip("ref_gpu_golden_ext.npz not generated (tests/golden/make_ref_golden.py ext, on a GPU)")
    return np.load(FIX_EXT)


def test_ext_fixture_inputs_regenerate_exactly(fixtures_ext):
    m = _mk()
    for key, n, a0, _ in ext_cases():
        assert str(fixtures_ext[key + "__sha"]) == m.sha(a0), key


@pytest.mark.parametrize("idx", range(52))
def test_oracle_matches_reference_ext(oracle_mod, fixtures_ext, idx):
    key, n, a0, meth = ext_cases()[idx]
    O = oracle_mod
    a = a0.copy()
    w, info, _ = O.eigen_batch(a, n, method=O.METHOD_IMTQL2 if meth == "imtql2" else O.METHOD_TQL2)
    assert (info == 0).all()
    _check_against(fixtures_ext[key + "__w"], fixtures_ext[key + "__z"], w, a, n, a0.dtype)
    e1, e2, fl = O.check(a0, fixtures_ext[key + "__w"], fixtures_ext[key + "__z"], n)
    assert (fl == 0).all(), (key, e1, e2)


@pytest.mark.gpu
def test_cuda_library_matches_reference_ext(fixtures_ext):
    import torch
    import eigeng_b200 as E
    for key, n, a0, meth in ext_cases():
        a = torch.from_numpy(a0.copy()).cuda()
        w, info = E.solve(a, n, method=E.IMTQL2 if meth == "imtql2" else E.TQL2)
        torch.cuda.synchronize()
        assert (info.cpu().numpy() == 0).all(), key
        _check_against(fixtures_ext[key + "__w"], fixtures_ext[key + "__z"], w.cpu().numpy(), a.cpu().numpy(), n,
                       a0.dtype)
