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
