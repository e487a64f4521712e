"""Python host mirror of the B200 batched symmetric eigensolver.

Thin ctypes binding of ``lib/libeigenGbatch.so`` (the C ABI declared in
``include/eigen_GPU_batch.h`` and ``include/eigen_GPU_check.h``).  The names
follow the reference's C/C++ interface (EigenG-Batched
``eigen_GPU_batch.h:26-30``, ``eigen_GPU_batch.hpp:104-157``,
``eigen_GPU_check.cu:183-197``); tensors are CUDA ``torch`` tensors and the
stream defaults to torch's current stream.  PyTorch only supplies device
memory and streams: every computation runs in the library's own kernels, and
nothing here falls back to another implementation -- a missing library is
an error.
"""
from __future__ import annotations

import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libeigenGbatch.so")

TQL2, IMTQL2, JACOBI = 0, 1, 2
ZMEM_AUTO, ZMEM_SHARED = 0, 1  # where the apply phase keeps Z (eigen_GPU_batch_opts.zmem)
REDUCE_AUTO, REDUCE_CTA, REDUCE_CLUSTER = 0, 1, 2  # phase-1 kernel (eigen_GPU_tune_entry.reduce)
# phases of eigen_GPU_batch_stage_* (EIGEN_GPU_STAGE_*)
STAGE_REDUCE, STAGE_QL, STAGE_APPLY, STAGE_ALL = 1, 2, 4, 7

_lib = None


class EigenGError(RuntimeError):
    pass


class Opts(ctypes.Structure):
    """eigen_GPU_batch_opts of include/eigen_GPU_batch.h."""
    _fields_ = [("method", ctypes.c_int), ("sort", ctypes.c_int), ("max_sweep", ctypes.c_int),
                ("rec_cap", ctypes.c_int), ("chunk", ctypes.c_int), ("split", ctypes.c_int),
                ("zmem", ctypes.c_int), ("ql_mpw", ctypes.c_int)]


class RefineOpts(ctypes.Structure):
    """eigen_GPU_refine_opts of include/eigen_GPU_batch.h."""
    _fields_ = [("max_iter", ctypes.c_int), ("tol", ctypes.c_double), ("fallback", ctypes.c_int),
                ("chunk", ctypes.c_int)]


class LearnedOpts(ctypes.Structure):
    """eigen_GPU_learned_opts of include/eigen_GPU_learned.h."""
    _fields_ = [("warm", ctypes.c_int), ("max_sweeps", ctypes.c_int), ("tol", ctypes.c_double),
                ("jacobi_tol", ctypes.c_double), ("fallback", ctypes.c_int), ("chunk", ctypes.c_int)]


WARM_NETWORK, WARM_BASIS, WARM_IDENTITY = 0, 1, 2


class TuneEntry(ctypes.Structure):
    """eigen_GPU_tune_entry of include/eigen_GPU_batch.h."""
    _fields_ = [("esize", ctypes.c_int), ("n", ctypes.c_int), ("split", ctypes.c_int), ("zmem", ctypes.c_int),
                ("ql_mpw", ctypes.c_int), ("reduce", ctypes.c_int)]


def lib():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise EigenGError(f"{LIB_PATH} is missing: build it with `make -C eigeng-batched_b200`")
        L = ctypes.CDLL(LIB_PATH)
        P, I, SZ = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
        for s in ("DP", "FP"):
            f = getattr(L, "eigen_GPU_batch_" + s)
            f.argtypes = [I, I, I, I, P, P, P, P]
            f.restype = None
            f = getattr(L, "eigen_GPU_batch_BufferSize_" + s)
            f.argtypes = [I, I, I, I, ctypes.POINTER(SZ)]
            f.restype = I
            f = getattr(L, "eigen_GPU_batch_ex_BufferSize_" + s)
            f.argtypes = [I, I, I, I, ctypes.POINTER(Opts), ctypes.POINTER(SZ)]
            f.restype = I
            f = getattr(L, "eigen_GPU_batch_ex_" + s)
            f.argtypes = [I, I, I, I, P, P, P, SZ, P, ctypes.POINTER(Opts), P]
            f.restype = I
            f = getattr(L, "eigen_GPU_batch_stage_" + s)
            f.argtypes = [I, I, I, I, P, P, P, SZ, P, ctypes.POINTER(Opts), I, I, I, P]
            f.restype = I
            f = getattr(L, "eigen_GPU_check_" + s)
            f.argtypes = [I, I, I, I, P, P, P, P]
            f.restype = None
            f = getattr(L, "eigen_GPU_check_ex_" + s)
            f.argtypes = [I, I, I, I, P, P, P, P, P, P, P]
            f.restype = I
        for s_ in ("DP", "FP"):
            f = getattr(L, "eigen_GPU_batch_interleaved_BufferSize_" + s_)
            f.argtypes = [I, I, ctypes.POINTER(Opts), ctypes.POINTER(SZ)]
            f.restype = I
            f = getattr(L, "eigen_GPU_batch_interleaved_" + s_)
            f.argtypes = [I, I, P, P, P, P, SZ, P, ctypes.POINTER(Opts), P]
            f.restype = I
        for s_ in ("DP", "FP"):
            f = getattr(L, "eigen_GPU_batch_uneven_BufferSize_" + s_)
            f.argtypes = [I, P, ctypes.POINTER(Opts), ctypes.POINTER(SZ)]
            f.restype = I
            f = getattr(L, "eigen_GPU_batch_uneven_" + s_)
            f.argtypes = [I, P, P, P, P, SZ, P, ctypes.POINTER(Opts), P]
            f.restype = I
        for s_ in ("DP", "FP"):
            f = getattr(L, "eigen_GPU_batch_packed_" + s_)
            f.argtypes = [I, I, P, P, I, P, P, SZ, P, ctypes.POINTER(Opts), P]
            f.restype = I
        for s_ in ("DP", "FP"):
            f = getattr(L, "eigen_GPU_batch_packed_check_" + s_)
            f.argtypes = [I, I, P, P, I, P, P, SZ, P, ctypes.POINTER(Opts), P, P, P, P]
            f.restype = I
        for s_ in ("DP", "FP"):
            f = getattr(L, "eigen_GPU_batch_symfunc_" + s_)
            f.argtypes = [I, I, I, P, P, P, I, ctypes.c_double, P]
            f.restype = I
        for s_ in ("DP", "FP"):
            f = getattr(L, "eigen_GPU_batch_launch_params_" + s_)
            f.argtypes = [I, I] + [ctypes.POINTER(I)] * 6
            f.restype = I
        L.eigen_GPU_batch_refine_BufferSize_DP.argtypes = [I, I, I, ctypes.POINTER(RefineOpts), ctypes.POINTER(SZ)]
        L.eigen_GPU_batch_refine_BufferSize_DP.restype = I
        L.eigen_GPU_batch_refine_DP.argtypes = [I, I, I, P, P, P, SZ, P, P, ctypes.POINTER(RefineOpts), P]
        L.eigen_GPU_batch_refine_DP.restype = I
        L.eigen_GPU_batch_rayleigh_BufferSize_DP.argtypes = [I, I, I, ctypes.POINTER(SZ)]
        L.eigen_GPU_batch_rayleigh_BufferSize_DP.restype = I
        L.eigen_GPU_batch_rayleigh_DP.argtypes = [I, I, I, P, P, P, P, P, SZ, P]
        L.eigen_GPU_batch_rayleigh_DP.restype = I
        SZP = ctypes.POINTER(SZ)
        L.eigen_GPU_mlp_size.argtypes = [I, I, I, I, SZP]
        L.eigen_GPU_mlp_ws_size.argtypes = [I, I, I, I, I, SZP]
        L.eigen_GPU_mlp_init.argtypes = [I, I, I, I, P, ctypes.c_ulonglong, P]
        L.eigen_GPU_mlp_forward.argtypes = [I, I, I, I, P, I, P, P, P, SZ, P]
        L.eigen_GPU_mlp_gradient.argtypes = [I, I, I, I, P, I, P, P, P, P, P, SZ, P]
        L.eigen_GPU_mlp_train_step.argtypes = [I, I, I, I, P, I, P, P, ctypes.c_float, I, P, P, SZ, P]
        L.eigen_GPU_learned_targets_FP.argtypes = [I, I, P, I, P, P, P]
        L.eigen_GPU_batch_learned_BufferSize_FP.argtypes = [I, I, I, I, I, ctypes.POINTER(LearnedOpts), SZP]
        L.eigen_GPU_batch_learned_FP.argtypes = [I, I, I, P, P, P, P, I, I, P, SZ, P, P, P,
                                                 ctypes.POINTER(LearnedOpts), P]
        for f in ("eigen_GPU_mlp_size", "eigen_GPU_mlp_ws_size", "eigen_GPU_mlp_init", "eigen_GPU_mlp_forward",
                  "eigen_GPU_mlp_gradient", "eigen_GPU_mlp_train_step", "eigen_GPU_learned_targets_FP",
                  "eigen_GPU_batch_learned_BufferSize_FP", "eigen_GPU_batch_learned_FP"):
            getattr(L, f).restype = I
        L.eigen_GPU_batch_tune_set.argtypes = [P, I]
        L.eigen_GPU_batch_tune_set.restype = I
        L.eigen_GPU_batch_tune_get.argtypes = [I, I, ctypes.POINTER(TuneEntry)]
        L.eigen_GPU_batch_tune_get.restype = I
        L.eigen_GPU_batch_noalloc_DP.argtypes = [I, I, I, I, P, P, P, P]
        L.eigen_GPU_batch_noalloc_DP.restype = I
        L.eigen_GPU_batch_trace.argtypes = [P, I]
        L.eigen_GPU_batch_trace.restype = I
        _lib = L
    return _lib


class PhaseTrace:
    """Context manager recording the per-phase events of eigen_GPU_batch_trace
    for up to `chunks` chunks; `.ms()` returns [(p1, p2, p3) per chunk] in ms."""

    def __init__(self, chunks=1):
        self.events = [torch.cuda.Event(enable_timing=True) for _ in range(4 * chunks)]
        for e in self.events:  # torch creates the CUDA event on first record
            e.record()
        torch.cuda.synchronize()
        self._arr = (ctypes.c_void_p * len(self.events))(*[ctypes.c_void_p(e.cuda_event) for e in self.events])

    def __enter__(self):
        st = lib().eigen_GPU_batch_trace(self._arr, len(self.events))
        if st != 0:
            raise EigenGError(f"eigen_GPU_batch_trace failed with cudaError {st}")
        # events re-recorded by the solve come after this mark; the others
        # keep their earlier placeholder record
        self._mark = torch.cuda.Event(enable_timing=True)
        self._mark.record()
        return self

    def __exit__(self, *exc):
        lib().eigen_GPU_batch_trace(None, 0)
        return False

    def ms(self):
        """Phase times of every chunk the traced solve ran."""
        torch.cuda.synchronize()
        out = []
        for c in range(len(self.events) // 4):
            e = self.events[4 * c:4 * c + 4]
            if self._mark.elapsed_time(e[0]) < 0:  # not recorded by the solve
                break
            out.append(tuple(e[i].elapsed_time(e[i + 1]) for i in range(3)))
        return out


def exported_symbols():
    return [
        "eigen_GPU_batch_DP", "eigen_GPU_batch_FP",
        "eigen_GPU_batch_BufferSize_DP", "eigen_GPU_batch_BufferSize_FP",
        "eigen_GPU_batch_ex_DP", "eigen_GPU_batch_ex_FP",
        "eigen_GPU_batch_ex_BufferSize_DP", "eigen_GPU_batch_ex_BufferSize_FP",
        "eigen_GPU_batch_stage_DP", "eigen_GPU_batch_stage_FP",
        "eigen_GPU_check_DP", "eigen_GPU_check_FP",
        "eigen_GPU_check_ex_DP", "eigen_GPU_check_ex_FP",
        "eigen_GPU_batch_trace", "eigen_GPU_batch_noalloc_DP",
        "eigen_GPU_batch_launch_params_DP", "eigen_GPU_batch_launch_params_FP",
        "eigen_GPU_batch_refine_DP", "eigen_GPU_batch_refine_BufferSize_DP",
        "eigen_GPU_batch_rayleigh_DP", "eigen_GPU_batch_rayleigh_BufferSize_DP",
        "eigen_GPU_batch_tune_set", "eigen_GPU_batch_tune_get",
        "eigen_GPU_mlp_size", "eigen_GPU_mlp_ws_size", "eigen_GPU_mlp_init", "eigen_GPU_mlp_forward",
        "eigen_GPU_mlp_gradient", "eigen_GPU_mlp_train_step", "eigen_GPU_learned_targets_FP",
        "eigen_GPU_batch_learned_BufferSize_FP", "eigen_GPU_batch_learned_FP",
        "eigen_GPU_batch_symfunc_DP", "eigen_GPU_batch_symfunc_FP",
        "eigen_GPU_batch_packed_DP", "eigen_GPU_batch_packed_FP",
        "eigen_GPU_batch_packed_check_DP", "eigen_GPU_batch_packed_check_FP",
        "eigen_GPU_batch_uneven_DP", "eigen_GPU_batch_uneven_FP",
        "eigen_GPU_batch_uneven_BufferSize_DP", "eigen_GPU_batch_uneven_BufferSize_FP",
        "eigen_GPU_batch_interleaved_DP", "eigen_GPU_batch_interleaved_FP",
        "eigen_GPU_batch_interleaved_BufferSize_DP", "eigen_GPU_batch_interleaved_BufferSize_FP",
    ]


def _sfx(dtype):
    if dtype == torch.float64:
        return "DP"
    if dtype == torch.float32:
        return "FP"
    raise TypeError(f"unsupported dtype {dtype}")


def _ptr(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _stream(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def _dims(a, n, nm):
    nm = n if nm is None else nm
    if not a.is_cuda or not a.is_contiguous():
        raise EigenGError("a must be a contiguous CUDA tensor")
    if a.numel() % (nm * n):
        raise EigenGError("a.numel() is not a multiple of nm*n")
    return a.numel() // (nm * n), nm


def buffer_size(L, nm, n, m=None, dtype=torch.float64, rec_cap=0, method=TQL2, chunk=0):
    """eigen_GPU_batch_BufferSize<T>: workspace bytes (for the given options)."""
    m = n if m is None else m
    out = ctypes.c_size_t(0)
    if rec_cap or chunk or method != TQL2:
        o = Opts(method, 1, 100, rec_cap, chunk)
        st = getattr(lib(), "eigen_GPU_batch_ex_BufferSize_" + _sfx(dtype))(L, nm, n, m, ctypes.byref(o),
                                                                           ctypes.byref(out))
    else:
        st = getattr(lib(), "eigen_GPU_batch_BufferSize_" + _sfx(dtype))(L, nm, n, m, ctypes.byref(out))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_BufferSize failed with cudaError {st}")
    return out.value


def launch_params(L, n, dtype=torch.float64):
    """eigen_GPU_batch_get_Launch_params<T>: the reduction phase's launch
    geometry on the current device, as a dict (grpSZ, numTB, numGR, numTH,
    sizeSH, sizeL2)."""
    v = [ctypes.c_int(0) for _ in range(6)]
    st = getattr(lib(), "eigen_GPU_batch_launch_params_" + _sfx(dtype))(L, n, *[ctypes.byref(x) for x in v])
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_launch_params failed with cudaError {st}")
    return dict(zip(("grpSZ", "numTB", "numGR", "numTH", "sizeSH", "sizeL2"), (x.value for x in v)))


def query_lwork(L, nm, n, m=None, dtype=torch.float64):
    """The C size-query mode: wk == NULL writes the size through w (host)."""
    m = n if m is None else m
    out = ctypes.c_size_t(0xDEADBEEF)
    getattr(lib(), "eigen_GPU_batch_" + _sfx(dtype))(L, nm, n, m, None, ctypes.byref(out), None, None)
    return out.value


def workspace(L, nm, n, dtype, device=None, rec_cap=0, chunk=0):
    nb = buffer_size(L, nm, n, n, dtype, rec_cap, TQL2, chunk)
    return torch.empty(max(nb, 16), dtype=torch.uint8, device=device or "cuda")


def eigen_GPU_batch(a, w, wk, n, nm=None, m=None, stream=None):
    """Drop-in call: eigenvectors overwrite ``a``, eigenvalues go to ``w``."""
    L, nm = _dims(a, n, nm)
    m = n if m is None else m
    getattr(lib(), "eigen_GPU_batch_" + _sfx(a.dtype))(L, nm, n, m, _ptr(a), _ptr(w), _ptr(wk), _stream(stream))


def eigen_GPU_batch_ex(a, w, wk, n, nm=None, m=None, info=None, method=TQL2, sort=True, max_sweep=100,
                       stream=None, rec_cap=0, chunk=0, split=0, zmem=ZMEM_AUTO, ql_mpw=0):
    """Extended call; returns the cudaError_t status (0 on success)."""
    L, nm = _dims(a, n, nm)
    m = n if m is None else m
    o = Opts(method, 1 if sort else 0, max_sweep, rec_cap, chunk, split, zmem, ql_mpw)
    lw = 0 if wk is None else wk.numel() * wk.element_size()
    return getattr(lib(), "eigen_GPU_batch_ex_" + _sfx(a.dtype))(
        L, nm, n, m, _ptr(a), _ptr(w), _ptr(wk), lw, _ptr(info), ctypes.byref(o), _stream(stream))


def stage(a, w, wk, n, phases, first=0, count=0, nm=None, m=None, info=None, method=TQL2, sort=True,
          max_sweep=100, stream=None, rec_cap=0, split=0, zmem=ZMEM_AUTO, ql_mpw=0):
    """eigen_GPU_batch_stage_*: the phases in ``phases`` (STAGE_* bits) for
    matrices first .. first+count-1 (count <= 0: to the end) of the batch
    ``a``; ``wk`` is the whole batch's workspace (``workspace(..., chunk=L)``).
    Returns the cudaError_t status."""
    L, nm = _dims(a, n, nm)
    m = n if m is None else m
    o = Opts(method, 1 if sort else 0, max_sweep, rec_cap, L, split, zmem, ql_mpw)
    lw = 0 if wk is None else wk.numel() * wk.element_size()
    return getattr(lib(), "eigen_GPU_batch_stage_" + _sfx(a.dtype))(
        L, nm, n, m, _ptr(a), _ptr(w), _ptr(wk), lw, _ptr(info), ctypes.byref(o), phases, first, count,
        _stream(stream))


def eigen_GPU_batch_noalloc(a, w, n, nm=None, m=None, info=None, stream=None):
    """eigen_GPU_batch_noalloc_DP: solve with the library's static device
    workspace (FP64, tql2, sorted); returns the cudaError_t status."""
    L, nm = _dims(a, n, nm)
    m = n if m is None else m
    if a.dtype != torch.float64:
        raise TypeError("eigen_GPU_batch_noalloc_DP takes float64 matrices")
    return lib().eigen_GPU_batch_noalloc_DP(L, nm, n, m, _ptr(a), _ptr(w), _ptr(info), _stream(stream))


def solve(a, n, nm=None, method=TQL2, sort=True, max_sweep=100, wk=None, stream=None, rec_cap=0, chunk=0,
          split=0, zmem=ZMEM_AUTO):
    """Convenience wrapper: solves in place, returns (w, info)."""
    L, nm = _dims(a, n, nm)
    w = torch.empty((L, n), dtype=a.dtype, device=a.device)
    info = torch.zeros(L, dtype=torch.int32, device=a.device)
    if wk is None and method != JACOBI:
        wk = workspace(L, nm, n, a.dtype, a.device, rec_cap, chunk)
    st = eigen_GPU_batch_ex(a, w, wk, n, nm, n, info, method, sort, max_sweep, stream, rec_cap, chunk, split,
                            zmem)
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_ex failed with cudaError {st}")
    return w, info


def refine_workspace(L, nm, n, max_iter=0, tol=0.0, fallback=True, chunk=0, device=None):
    o = RefineOpts(max_iter, tol, 1 if fallback else 0, chunk)
    lw = ctypes.c_size_t(0)
    st = lib().eigen_GPU_batch_refine_BufferSize_DP(L, nm, n, ctypes.byref(o), ctypes.byref(lw))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_refine_BufferSize_DP failed with cudaError {st}")
    return torch.empty(max(lw.value, 16), dtype=torch.uint8, device=device or "cuda")


def solve_refined(a, n, nm=None, max_iter=0, tol=0.0, fallback=True, chunk=0, wk=None, stream=None):
    """eigen_GPU_batch_refine_DP: FP32 solve refined to FP64 accuracy on the
    tensor cores, in place on the FP64 batch ``a``.  Returns (w, info,
    iters): iters[k] is the number of refinement iterations matrix k took,
    0 where it went to the plain FP64 fallback."""
    L, nm = _dims(a, n, nm)
    if a.dtype != torch.float64:
        raise TypeError("eigen_GPU_batch_refine_DP takes float64 matrices")
    w = torch.empty((L, n), dtype=a.dtype, device=a.device)
    info = torch.zeros(L, dtype=torch.int32, device=a.device)
    iters = torch.zeros(L, dtype=torch.int32, device=a.device)
    if wk is None:
        wk = refine_workspace(L, nm, n, max_iter, tol, fallback, chunk, a.device)
    o = RefineOpts(max_iter, tol, 1 if fallback else 0, chunk)
    st = lib().eigen_GPU_batch_refine_DP(L, nm, n, _ptr(a), _ptr(w), _ptr(wk), wk.numel(), _ptr(info), _ptr(iters),
                                         ctypes.byref(o), _stream(stream))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_refine_DP failed with cudaError {st}")
    return w, info, iters


def rayleigh(a, x, n, nm=None, want_s=True, want_g=True, stream=None):
    """eigen_GPU_batch_rayleigh_DP: (S, G) = (X^T A X, X^T X) per matrix,
    FP64-accurate products on the int8 tensor cores (None where not
    wanted); S and G are (L, n, n) holding column-major matrices."""
    L, nm = _dims(a, n, nm)
    lw = ctypes.c_size_t(0)
    st = lib().eigen_GPU_batch_rayleigh_BufferSize_DP(L, nm, n, ctypes.byref(lw))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_rayleigh_BufferSize_DP failed with cudaError {st}")
    wk = torch.empty(max(lw.value, 16), dtype=torch.uint8, device=a.device)
    s = torch.empty((L, n, n), dtype=torch.float64, device=a.device) if want_s else None
    g = torch.empty((L, n, n), dtype=torch.float64, device=a.device) if want_g else None
    st = lib().eigen_GPU_batch_rayleigh_DP(L, nm, n, _ptr(a), _ptr(x), _ptr(s), _ptr(g), _ptr(wk), lw.value,
                                           _stream(stream))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_rayleigh_DP failed with cudaError {st}")
    return s, g


def tune_set(entries):
    """eigen_GPU_batch_tune_set on the current device; entries: dicts with
    esize, n, split, zmem, ql_mpw and optionally reduce (REDUCE_*; an empty
    list clears the table)."""
    arr = (TuneEntry * max(1, len(entries)))(*[TuneEntry(e["esize"], e["n"], e["split"], e["zmem"], e["ql_mpw"],
                                                         e.get("reduce", REDUCE_AUTO)) for e in entries])
    st = lib().eigen_GPU_batch_tune_set(ctypes.cast(arr, ctypes.c_void_p), len(entries))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_tune_set failed with cudaError {st}")


def tune_get(esize, n):
    """The tuned entry for (esize, n) as a dict, or None."""
    e = TuneEntry()
    st = lib().eigen_GPU_batch_tune_get(esize, n, ctypes.byref(e))
    if st != 0:
        return None
    return {"esize": e.esize, "n": e.n, "split": e.split, "zmem": e.zmem, "ql_mpw": e.ql_mpw, "reduce": e.reduce}


def packed_size(n):
    return n * (n + 1) // 2


def pack_upper(a, n, nm=None):
    """Packed upper triangles (LAPACK 'U' order) of a batch in the full
    column-major layout: (L, n(n+1)/2), element (r, c), r <= c, at
    r + c(c+1)/2."""
    nm = n if nm is None else nm
    A = a.reshape(-1, n, nm)
    return torch.cat([A[:, c, :c + 1] for c in range(n)], dim=1).contiguous()


def solve_packed(ap, n, ldz=None, method=TQL2, sort=True, max_sweep=100, stream=None, rec_cap=0, chunk=0, split=0):
    """eigen_GPU_batch_packed: solves a batch given as packed upper
    triangles; returns (z, w, info) with z in the full layout."""
    if not ap.is_cuda or not ap.is_contiguous() or ap.numel() % packed_size(n):
        raise EigenGError("ap must be a contiguous CUDA tensor of L*n(n+1)/2 elements")
    L = ap.numel() // packed_size(n)
    ldz = n if ldz is None else ldz
    z = torch.empty((L, n, ldz), dtype=ap.dtype, device=ap.device)
    w = torch.empty((L, n), dtype=ap.dtype, device=ap.device)
    info = torch.zeros(L, dtype=torch.int32, device=ap.device)
    wk = workspace(L, ldz, n, ap.dtype, ap.device, rec_cap, chunk) if method != JACOBI else None
    o = Opts(method, 1 if sort else 0, max_sweep, rec_cap, chunk, split)
    lw = 0 if wk is None else wk.numel()
    st = getattr(lib(), "eigen_GPU_batch_packed_" + _sfx(ap.dtype))(
        L, n, _ptr(ap), _ptr(z), ldz, _ptr(w), _ptr(wk), lw, _ptr(info), ctypes.byref(o), _stream(stream))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_packed failed with cudaError {st}")
    return z, w, info


def solve_packed_checked(ap, n, ldz=None, method=TQL2, sort=True, max_sweep=100, stream=None, wk=None):
    """eigen_GPU_batch_packed_check: the packed solve and the accuracy gate
    in one call; returns (z, w, info, err1, err2, flags)."""
    if not ap.is_cuda or not ap.is_contiguous() or ap.numel() % packed_size(n):
        raise EigenGError("ap must be a contiguous CUDA tensor of L*n(n+1)/2 elements")
    L = ap.numel() // packed_size(n)
    ldz = n if ldz is None else ldz
    z = torch.empty((L, n, ldz), dtype=ap.dtype, device=ap.device)
    w = torch.empty((L, n), dtype=ap.dtype, device=ap.device)
    info = torch.zeros(L, dtype=torch.int32, device=ap.device)
    e1 = torch.empty(L, dtype=torch.float64, device=ap.device)
    e2 = torch.empty(L, dtype=torch.float64, device=ap.device)
    fl = torch.empty(L, dtype=torch.int32, device=ap.device)
    if wk is None and method != JACOBI:
        wk = workspace(L, ldz, n, ap.dtype, ap.device)
    o = Opts(method, 1 if sort else 0, max_sweep, 0, 0, 0)
    lw = 0 if wk is None else wk.numel()
    st = getattr(lib(), "eigen_GPU_batch_packed_check_" + _sfx(ap.dtype))(
        L, n, _ptr(ap), _ptr(z), ldz, _ptr(w), _ptr(wk), lw, _ptr(info), ctypes.byref(o), _ptr(e1), _ptr(e2),
        _ptr(fl), _stream(stream))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_packed_check failed with cudaError {st}")
    return z, w, info, e1, e2, fl


def solve_interleaved(ai, n, method=TQL2, sort=True, max_sweep=100, stream=None):
    """eigen_GPU_batch_interleaved: ai is a CUDA tensor of shape (n*n, L) with
    element (i, j) of matrix k at ai[i + j*n, k]; returns (zi, wi, info) in
    the same layout (wi of shape (n, L))."""
    if not ai.is_cuda or not ai.is_contiguous() or ai.dim() != 2 or ai.shape[0] != n * n:
        raise EigenGError("ai must be a contiguous CUDA tensor of shape (n*n, L)")
    L = ai.shape[1]
    o = Opts(method, 1 if sort else 0, max_sweep, 0, 0, 0)
    sfx = _sfx(ai.dtype)
    lw = ctypes.c_size_t(0)
    st = getattr(lib(), "eigen_GPU_batch_interleaved_BufferSize_" + sfx)(L, n, ctypes.byref(o), ctypes.byref(lw))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_interleaved_BufferSize failed with cudaError {st}")
    wk = torch.empty(max(lw.value, 16), dtype=torch.uint8, device=ai.device)
    zi = torch.empty_like(ai)
    wi = torch.empty((n, L), dtype=ai.dtype, device=ai.device)
    info = torch.zeros(L, dtype=torch.int32, device=ai.device)
    st = getattr(lib(), "eigen_GPU_batch_interleaved_" + sfx)(L, n, _ptr(ai), _ptr(zi), _ptr(wi), _ptr(wk), lw.value,
                                                             _ptr(info), ctypes.byref(o), _stream(stream))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_interleaved failed with cudaError {st}")
    return zi, wi, info


def solve_uneven(a, ns, method=TQL2, sort=True, max_sweep=100, stream=None, zmem=ZMEM_AUTO, ql_mpw=0, wave=0,
                 rec_cap=0):
    """eigen_GPU_batch_uneven: a is a flat CUDA tensor holding matrix k
    (order ns[k], column-major, leading dimension ns[k]) at offset
    sum_{j<k} ns[j]^2; solved in place.  Returns (w, info), w flat with the
    eigenvalues of matrix k at sum_{j<k} ns[j].  wave > 0 caps the matrices
    solved together (opts.chunk), and so the workspace."""
    nsa = (ctypes.c_int * len(ns))(*[int(x) for x in ns])
    L = len(ns)
    tot = sum(int(x) * int(x) for x in ns)
    if not a.is_cuda or not a.is_contiguous() or a.numel() != tot:
        raise EigenGError("a must be a contiguous CUDA tensor of sum(n^2) elements")
    o = Opts(method, 1 if sort else 0, max_sweep, int(rec_cap), int(wave), 0, zmem, ql_mpw)
    sfx = _sfx(a.dtype)
    lw = ctypes.c_size_t(0)
    st = getattr(lib(), "eigen_GPU_batch_uneven_BufferSize_" + sfx)(L, nsa, ctypes.byref(o), ctypes.byref(lw))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_uneven_BufferSize failed with cudaError {st}")
    wk = torch.empty(max(lw.value, 16), dtype=torch.uint8, device=a.device)
    w = torch.empty(sum(int(x) for x in ns), dtype=a.dtype, device=a.device)
    info = torch.zeros(L, dtype=torch.int32, device=a.device)
    st = getattr(lib(), "eigen_GPU_batch_uneven_" + sfx)(L, nsa, _ptr(a), _ptr(w), _ptr(wk), lw.value, _ptr(info),
                                                        ctypes.byref(o), _stream(stream))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_uneven failed with cudaError {st}")
    return w, info


FUNC_DIAG, FUNC_POW, FUNC_EXP = 0, 1, 2


def symfunc(v, w, n, func=FUNC_POW, p=0.5, nm=None, z=None, stream=None):
    """eigen_GPU_batch_symfunc: z_k = V_k diag(f(w_k)) V_k^T for a solved
    batch (v: eigenvectors, w: eigenvalues); returns z (allocated when None)."""
    L, nm = _dims(v, n, nm)
    if z is None:
        z = torch.empty_like(v)
    st = getattr(lib(), "eigen_GPU_batch_symfunc_" + _sfx(v.dtype))(L, nm, n, _ptr(v), _ptr(w), _ptr(z), func,
                                                                     float(p), _stream(stream))
    if st != 0:
        raise EigenGError(f"eigen_GPU_batch_symfunc failed with cudaError {st}")
    return z


def host_chunks(L, chunk=0):
    """Chunk boundaries of solve_host for a batch of L matrices: equal
    chunks of ``chunk`` (the last one ragged) when ``chunk`` > 0; else, from
    L = 2048 on, 17 chunks of about L/16 with half-size first and last ones;
    below that one chunk."""
    if chunk > 0:
        return list(range(0, L, chunk)) + [L]
    if L >= 2048:
        return [0] + [(L * (2 * k - 1) + 16) // 32 for k in range(1, 17)] + [L]
    return [0, L]


def solve_host(a_host, n, nm=None, w_host=None, chunk=0, method=TQL2, sort=True, max_sweep=100,
               stream=None, device=None, z_host=None, info_host=None):
    """Solves a batch held in host memory (pinned for the copies to be
    asynchronous): eigenvectors overwrite ``a_host`` (or go to ``z_host``,
    same shape, leaving ``a_host`` intact), eigenvalues go to ``w_host``
    (allocated pinned when None), which is returned.

    The batch goes through the device in chunks on separate streams -- copy
    in, solve (two streams), copy out -- so that the copies of one chunk
    overlap the solve of another; four device buffers rotate.  ``chunk`` > 0
    sets equal chunks.  The work starts after what is
    already queued on ``stream`` (default: the current stream) and
    ``stream`` waits for all of it, so events recorded there bracket the
    whole transfer and solve.  Results equal eigen_GPU_batch_ex's on the
    same matrices.  ``info_host`` (optional host int32 tensor of L entries,
    pinned for an asynchronous copy) receives each matrix's status as
    eigen_GPU_batch_ex reports it: 0, or the index at which QL exceeded
    max_sweep (NaN or Inf input shows up there too); read it after the
    caller's stream has completed."""
    nm = n if nm is None else nm
    if a_host.is_cuda or not a_host.is_contiguous() or a_host.numel() % (nm * n):
        raise EigenGError("a_host must be a contiguous host tensor of L*nm*n elements")
    L = a_host.numel() // (nm * n)
    a_host = a_host.view(L, n, nm)
    z_host = a_host if z_host is None else z_host.view(L, n, nm)
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    caller = stream if stream is not None else torch.cuda.current_stream(dev)
    dt = a_host.dtype
    if w_host is None:
        w_host = torch.empty((L, n), dtype=dt, pin_memory=True)
    # chunk boundaries: equal chunks of `chunk` matrices when given; else,
    # from L = 2048 on, chunks of L/16 with half-size first and last chunks
    # (17 in all) solved up to eight at a time on their own streams: the QL
    # phase of a chunk has a latency of about 2 ms at n = 128 whatever its
    # size and occupies few SMs, so the phases of the other chunks in flight
    # fill the GPU meanwhile, and the small end chunks shorten the copies
    # that nothing overlaps.  Host to host on B200, ms per batch, against
    # six chunks (1/16, 3/16, 1/4, 1/4, 3/16, 1/16) on two streams: FP64
    # n=128 L=4096 19.45 -> 16.26, n=32 L=16384 3.93 -> 3.89, n=64 L=20000
    # 18.73 -> 15.66, n=200 L=2048 61.1 -> 50.5, n=256 L=2048 104.7 -> 91.6;
    # FP32 n=128 L=4096 12.44 -> 10.43.  Four streams instead of eight lose
    # most of it (n=128 FP64 18.98 ms).
    bounds = host_chunks(L, chunk)
    nch = len(bounds) - 1
    C = max(bounds[i + 1] - bounds[i] for i in range(nch))
    # concurrent chunks, each with its own stream and workspace, and two
    # device buffers more than that, so that a chunk's copy in proceeds while
    # the chunks before it solve and copy out
    nrun = min(8, nch)
    nbuf = min(nrun + 2, nch)
    da = [torch.empty((C, n, nm), dtype=dt, device=dev) for _ in range(nbuf)]
    dw = [torch.empty((C, n), dtype=dt, device=dev) for _ in range(nbuf)]
    # QL phase with eight matrices per warp when chunks solve concurrently:
    # its lanes' chains then occupy fewer warps beside the other chunks'
    # kernels (measured on B200 at n=128 FP64, L=4096, two chunks in flight:
    # 19.8 ms against 20.8 with four, 21.1 with two, 21.3 automatic; with
    # eight in flight 16.26 ms against 16.15 with sixteen, which is slower
    # in FP32); one chunk alone keeps the automatic choice
    ql_mpw = 8 if nrun > 1 else 0
    if info_host is not None and (info_host.is_cuda or info_host.numel() != L or info_host.dtype != torch.int32):
        raise EigenGError("info_host must be a host int32 tensor of L entries")
    # per-matrix status, one buffer per device buffer: reused, like the
    # buffer itself, only after its copy-out (the chain s_in -> solve waits
    # for freed[b])
    info = [torch.zeros(C, dtype=torch.int32, device=dev) for _ in range(nbuf)]
    wk = [workspace(C, nm, n, dt, dev) if method != JACOBI else None for _ in range(nrun)]
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    s_runs = [torch.cuda.Stream(dev) for _ in range(nrun)]
    start = torch.cuda.Event()
    start.record(caller)
    for s_ in [s_in, s_out] + s_runs:
        s_.wait_event(start)
    freed = [None] * nbuf       # copy-out of the buffer's previous chunk
    for i in range(nch):
        c0, c1 = bounds[i], bounds[i + 1]
        b = i % nbuf
        cnt = c1 - c0
        if freed[b] is not None:
            s_in.wait_event(freed[b])
        with torch.cuda.stream(s_in):
            da[b][:cnt].copy_(a_host[c0:c1], non_blocking=True)
        loaded = torch.cuda.Event()
        loaded.record(s_in)
        s_run = s_runs[i % nrun]
        s_run.wait_event(loaded)
        st = eigen_GPU_batch_ex(da[b][:cnt], dw[b][:cnt], wk[i % nrun], n, nm, n, info[b][:cnt], method,
                                sort, max_sweep, s_run, ql_mpw=ql_mpw)
        if st != 0:
            raise EigenGError(f"eigen_GPU_batch_ex failed with cudaError {st}")
        solved = torch.cuda.Event()
        solved.record(s_run)
        s_out.wait_event(solved)
        with torch.cuda.stream(s_out):
            z_host[c0:c1].copy_(da[b][:cnt], non_blocking=True)
            w_host[c0:c1].copy_(dw[b][:cnt], non_blocking=True)
            if info_host is not None:
                info_host[c0:c1].copy_(info[b][:cnt], non_blocking=True)
        freed[b] = torch.cuda.Event()
        freed[b].record(s_out)
    done = torch.cuda.Event()
    done.record(s_out)
    caller.wait_event(done)
    # the device buffers are released only after the caller's stream has
    # waited for the last copy
    for t in da + dw + info + [x for x in wk if x is not None]:
        t.record_stream(caller)
    return w_host


def check(a0, w, z, n, nm=None, stream=None):
    """eigen_GPU_check_ex: per-matrix (err1, err2, flags) on the device."""
    L, nm = _dims(a0, n, nm)
    e1 = torch.empty(L, dtype=torch.float64, device=a0.device)
    e2 = torch.empty(L, dtype=torch.float64, device=a0.device)
    fl = torch.empty(L, dtype=torch.int32, device=a0.device)
    st = getattr(lib(), "eigen_GPU_check_ex_" + _sfx(a0.dtype))(
        L, nm, n, n, _ptr(a0), _ptr(w), _ptr(z), _ptr(e1), _ptr(e2), _ptr(fl), _stream(stream))
    if st != 0:
        raise EigenGError(f"eigen_GPU_check_ex failed with cudaError {st}")
    return e1, e2, fl
