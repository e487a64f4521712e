"""The C-ABI library loads and exports every entry point that include/*.h
declares (no compute call: this runs without a GPU)."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "eigeng-batched_b200", "lib", "libeigenGbatch.so")


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:void|cudaError_t)\s+(\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_reference_entry_points():
    names = declared_functions()
    for ref in ("eigen_GPU_batch_DP", "eigen_GPU_batch_FP", "eigen_GPU_check_DP", "eigen_GPU_check_FP"):
        assert ref in names


def test_library_exports_all_declared_symbols():
    assert os.path.exists(LIB), "build the library first (make -C eigeng-batched_b200)"
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_lists_exports():
    import eigeng_b200 as E
    assert sorted(E.exported_symbols()) == sorted(n for n in declared_functions())
    E.lib()


def test_cpp_header_compiles():
    """The C++ template header (eigen_GPU_batch.hpp) and the C headers
    compile as host code against the CUDA runtime headers."""
    import subprocess
    import tempfile
    src = ('#include "eigen_GPU_batch.hpp"\n#include "eigen_GPU_check.h"\n'
           "int main(){size_t lw=0; int g,b,r,t,s,l;\n"
           " (void)eigen_GPU_batch_BufferSize<double>(4,8,8,8,(double*)0,(double*)0,&lw);\n"
           " (void)eigen_GPU_batch_get_Launch_params<float>(4,8,g,b,r,t,s,l);\n"
           " eigen_GPU_batch<double>(4,8,8,8,(double*)0,(double*)0,(double*)0);\n return 0;}\n")
    with tempfile.TemporaryDirectory() as td:
        f = os.path.join(td, "t.cpp")
        open(f, "w").write(src)
        cmd = ["/usr/bin/g++", "-std=c++14", "-fsyntax-only", "-I" + os.path.join(ROOT, "include"),
               "-I/usr/local/cuda/include", f]
        subprocess.check_call(cmd)


def _cpp_launch_params_program(td):
    src = ('#include <stdio.h>\n#include "eigen_GPU_batch.hpp"\n'
           "int main(){ const int ns[] = {1, 5, 32, 33, 64, 96, 128, 129, 200, 256, 512, 1024};\n"
           " for (int i = 0; i < 12; i++) { int g,b,r,t,s,l;\n"
           "  if (eigen_GPU_batch_get_Launch_params<double>(4096, ns[i], g, b, r, t, s, l) != cudaSuccess) return 1;\n"
           "  printf(\"%d %d %d %d %d %d %d\\n\", ns[i], g, b, r, t, s, l); }\n"
           " int g,b,r,t,s,l; return eigen_GPU_batch_get_Launch_params<double>(0, 8, g, b, r, t, s, l) == cudaSuccess;}\n")
    f = os.path.join(td, "lp.cpp")
    open(f, "w").write(src)
    exe = os.path.join(td, "lp")
    import subprocess
    subprocess.check_call(["/usr/bin/g++", "-std=c++14", "-I" + os.path.join(ROOT, "include"),
                           "-I/usr/local/cuda/include", f, "-o", exe, "-L" + os.path.dirname(LIB),
                           "-Wl,-rpath," + os.path.dirname(LIB), "-leigenGbatch", "-L/usr/local/cuda/lib64",
                           "-lcudart"])
    return exe


def test_cpp_launch_params_program_builds(tmp_path):
    """The C++ template links against the library (its geometry query is an
    exported C function)."""
    _cpp_launch_params_program(str(tmp_path))


import pytest  # noqa: E402


@pytest.mark.gpu
def test_launch_params_report_the_launched_geometry(tmp_path):
    """eigen_GPU_batch_get_Launch_params<T> reports phase 1 as run() launches
    it: one thread per matrix for n = 1, a warp per matrix (four per block)
    for n <= 32, a CTA of 32*NB*NB threads (NB = ceil(n/32)) in the
    register form for 32 < n <= 128, and the CTA form's
    min(1024, ceil(n/32)*32*split) threads above (FP64 split 2 up to n =
    240, 4 up to 256, 2 up to 512, then 1), one block per matrix; with the cluster form asked
    for (tuned option reduce), ceil(n/32) blocks of 512 threads per
    matrix."""
    import subprocess
    out = subprocess.check_output([_cpp_launch_params_program(str(tmp_path))], text=True)
    rows = {int(x.split()[0]): [int(v) for v in x.split()[1:]] for x in out.strip().splitlines()}
    import math
    for n, (g, b, r, t, s, l) in rows.items():
        assert l > 0
        if n == 1:
            assert (g, b, r, t) == (1, 16, 256, 256)
        elif n <= 32:
            assert (g, b, r, t) == (32, 1024, 4, 128)
            assert s > 0
        elif n <= 128:
            nb = math.ceil(n / 32)
            assert (g, r, t) == (32 * nb * nb, 1, 32 * nb * nb), n
            assert 0 < b <= 4096
        else:
            split = 2 if n <= 240 else (4 if n <= 256 else (2 if n <= 512 else 1))
            th = min(1024, math.ceil(n / 32) * 32 * split)
            assert (g, r, t) == (th, 1, th), n
            assert 0 < b <= 4096
    import eigeng_b200 as E
    assert E.launch_params(4096, 128)["numTH"] == rows[128][3]
    E.tune_set([dict(esize=8, n=256, split=0, zmem=0, ql_mpw=0, reduce=E.REDUCE_CLUSTER)])
    try:
        lp = E.launch_params(4096, 256)
    finally:
        E.tune_set([])
    assert (lp["grpSZ"], lp["numGR"], lp["numTH"]) == (8 * 512, 1, 512) and lp["numTB"] % 8 == 0


@pytest.mark.parametrize("L,chunk", [(1, 0), (37, 0), (2047, 0), (2048, 0), (2049, 0), (3000, 0), (4096, 0),
                                     (100000, 0), (37, 2), (37, 5), (4096, 1000)])
def test_host_chunk_schedule(L, chunk):
    """solve_host's chunks tile [0, L) in order: the given size (last one
    ragged), else 17 chunks from L = 2048 on (half-size ends, the middle
    ones within one matrix of L/16), else one."""
    import eigeng_b200 as E
    b = E.host_chunks(L, chunk)
    assert b[0] == 0 and b[-1] == L
    sizes = [b[i + 1] - b[i] for i in range(len(b) - 1)]
    assert all(x > 0 for x in sizes)
    if chunk > 0:
        assert all(x == chunk for x in sizes[:-1]) and 0 < sizes[-1] <= chunk
    elif L >= 2048:
        assert len(sizes) == 17
        assert all(abs(x - L / 16) <= 1 for x in sizes[1:-1])
        assert all(abs(x - L / 32) <= 1 for x in (sizes[0], sizes[-1]))
    else:
        assert sizes == [L]
