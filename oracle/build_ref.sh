#!/bin/sh
# Builds the reference's own GPU library (EigenG-Batched, its default
# configuration: tql2 + DO_SORT, eigen_GPU_batch.cu:1-11) for sm_100a from
# the reference sources where they lie, into oracle/_ref/ (git-ignored).
# Test infrastructure only: the library pins the CPU oracle through the
# fixture script tests/golden/make_ref_golden.py.  The numerics flags are
# those of the reference's Makefile_cuda:32-40; the stock Makefile would
# emit only compute_90 PTX with this nvcc (Makefile_cuda:23-30), and its
# `nvcc --ptx` step (Makefile_cuda:75) is not run.
set -e
REF=${REF:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
if [ ! -f "$REF/eigen_GPU_batch.cu" ]; then
  echo "reference sources not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
"$NVCC" -O3 -std=c++14 -gencode arch=compute_100a,code=sm_100a \
  --compiler-options -fno-strict-aliasing --compiler-options -fPIC \
  --extra-device-vectorization --restrict --maxrregcount=127 \
  --prec-div=true --prec-sqrt=true --fmad=true \
  -I"$REF" -shared -o "$OUT/libeigenGbatch_ref.so" "$REF/eigen_GPU_batch.cu" -lcudart
echo "built $OUT/libeigenGbatch_ref.so"
