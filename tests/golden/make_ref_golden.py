"""Generates the fixtures of the reference's own GPU build (EigenG-Batched
eigen_GPU_batch_DP/FP compiled for sm_100a by oracle/build_ref.sh into
oracle/_ref/) on seeded inputs:

  tests/golden/ref_gpu_golden.npz      default build (tql2 + DO_SORT),
                                       n = 3 .. 128 (set "tql2")
  tests/golden/ref_gpu_golden_ext.npz  the USE_IMTQL 1 build (imtql2 +
                                       DO_SORT), n = 3 .. 256, and the
                                       default build at n = 256, the
                                       warp-per-matrix hhsy2tr_/tql2_/hhtr2sy_
                                       path of eigen_GPU_batch.cu:138-245
                                       (set "ext")

Run on a machine with a GPU:

    python tests/golden/make_ref_golden.py [tql2|ext] [out.npz]

The CPU oracle and the CUDA library are checked against these fixtures
(tests/test_golden.py).  n == 2 is left out: the reference's n <= 32 path
returns the input matrix unchanged for n == 2 (tred1_tiled.hpp:25-34,
hhtr2sy_tiled.hpp:27-35).
"""
import ctypes
import hashlib
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libeigenGbatch_ref.so")
REF_LIB_IMTQL = os.path.join(ROOT, "oracle", "_ref", "libeigenGbatch_ref_imtql.so")
OUT = {"tql2": os.path.join(ROOT, "tests", "golden", "ref_gpu_golden.npz"),
       "ext": os.path.join(ROOT, "tests", "golden", "ref_gpu_golden_ext.npz")}


def ref_solve(lib, a0, n):
    """Calls the reference exactly as its README does: size query, solve."""
    L = a0.shape[0]
    dt = a0.dtype
    fn = lib.eigen_GPU_batch_DP if dt == np.float64 else lib.eigen_GPU_batch_FP
    fn.restype = None
    lw = ctypes.c_size_t(0)
    fn(L, n, n, n, None, ctypes.byref(lw), None, None)
    a = torch.from_numpy(a0.copy()).cuda()
    w = torch.zeros((L, n), dtype=a.dtype, device="cuda")
    wk = torch.zeros(max(lw.value, 16), dtype=torch.uint8, device="cuda")
    fn(L, n, n, n, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(wk.data_ptr()),
       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return w.cpu().numpy(), a.cpu().numpy()


def ext_cases():
    """(key, n, input, method) of the "ext" set: method "imtql2" for the
    USE_IMTQL 1 build, "tql2" for the default build at n = 256."""
    for n in (3, 8, 17, 32, 33, 64, 100, 128, 256):
        L = 3 if n <= 33 else (2 if n <= 64 else 1)
        fams = {
            "symu": lambda: O.sym_uniform(L, n, seed=700 + n),
            "letkf": lambda: O.letkf_like(L, n, seed=800 + n),
        }
        if n <= 64:
            fams["refrand"] = lambda: O.ref_matrices(L, n, O.REF_SYM_RAND, seed0=7)
        for fam, gen in fams.items():
            a = gen()
            for dt in (np.float64, np.float32):
                a_t = np.ascontiguousarray(a.astype(dt))
                yield f"imtql2_{np.dtype(dt).name}_{fam}_{n}", n, a_t, "imtql2"
                if n == 256:
                    yield f"tql2_{np.dtype(dt).name}_{fam}_{n}", n, a_t, "tql2"


def cases():
    """(key, n, input) for every fixture; inputs come from the seeded
    generators of oracle/oracle.py, so only their sha256 is stored."""
    for n in (3, 5, 8, 16, 17, 31, 32, 33, 48, 64, 100, 128):
        L = 3 if n <= 33 else (2 if n <= 64 else 1)
        fams = {
            "symu": lambda: O.sym_uniform(L, n, seed=500 + n),
            "letkf": lambda: O.letkf_like(L, n, seed=600 + n),
        }
        if n <= 64:
            fams["frank"] = lambda: O.ref_matrices(L, n, O.REF_FRANK)
            fams["refrand"] = lambda: O.ref_matrices(L, n, O.REF_SYM_RAND)
        for fam, gen in fams.items():
            a = gen()
            for dt in (np.float64, np.float32):
                yield f"{np.dtype(dt).name}_{fam}_{n}", n, np.ascontiguousarray(a.astype(dt))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    which = sys.argv[1] if len(sys.argv) > 1 else "tql2"
    out = sys.argv[2] if len(sys.argv) > 2 else OUT[which]
    libs = {"tql2": ctypes.CDLL(REF_LIB)}
    if which == "ext":
        libs["imtql2"] = ctypes.CDLL(REF_LIB_IMTQL)
        todo = list(ext_cases())
    else:
        todo = [(k, n, a0, "tql2") for k, n, a0 in cases()]
    res = {}
    for key, n, a0, meth in todo:
        w, z = ref_solve(libs[meth], a0, n)
        res[key + "__sha"] = np.array(sha(a0))
        res[key + "__w"] = w
        res[key + "__z"] = z
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    np.savez_compressed(out, **res)
    print("wrote", out, len(res) // 3, "cases")


if __name__ == "__main__":
    main()
