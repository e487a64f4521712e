#!/bin/sh
# Builds the reference's own GPU library (EigenG-Batched) for sm_100a from
# the reference sources where they lie, into oracle/_ref/ (git-ignored):
#   libeigenGbatch_ref.so        its default configuration, tql2 + DO_SORT
#                                (eigen_GPU_batch.cu:1-11)
#   libeigenGbatch_ref_imtql.so  the USE_IMTQL 1 variant (imtql2 +
#                                DO_SORT); the macro is #defined inside
#                                eigen_GPU_batch.cu, so that one file is
#                                copied to a temporary directory, the
#                                define flipped, and compiled there against
#                                the reference's headers; the copy is
#                                deleted afterwards and never enters the
#                                repository
# Test infrastructure only: the libraries pin the CPU oracle through the
# fixture script tests/golden/make_ref_golden.py.  The numerics flags are
# those of the reference's Makefile_cuda:32-40; the stock Makefile would
# emit only compute_90 PTX with this nvcc (Makefile_cuda:23-30), and its
# `nvcc --ptx` step (Makefile_cuda:75) is not run.  The Jacobi variant
# (jac_tiled.hpp) is not built: its sweep loop has no iteration limit.
#
#   sh oracle/build_ref.sh <reference source directory>
#   REF=<reference source directory> sh oracle/build_ref.sh
set -e
REF=${1:-$REF}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
if [ -z "$REF" ] || [ ! -f "$REF/eigen_GPU_batch.cu" ]; then
  echo "reference sources not given or not found (argument or REF=...); skipping" >&2
  exit 0
fi
FLAGS="-O3 -std=c++14 -gencode arch=compute_100a,code=sm_100a \
  --compiler-options -fno-strict-aliasing --compiler-options -fPIC \
  --extra-device-vectorization --restrict --maxrregcount=127 \
  --prec-div=true --prec-sqrt=true --fmad=true"
mkdir -p "$OUT"
# shellcheck disable=SC2086
"$NVCC" $FLAGS -I"$REF" -shared -o "$OUT/libeigenGbatch_ref.so" "$REF/eigen_GPU_batch.cu" -lcudart
echo "built $OUT/libeigenGbatch_ref.so"

TMP=$(mktemp -d)
trap 'rm -rf "$TMP"' EXIT
sed 's/^#define[[:space:]]*USE_IMTQL[[:space:]]*0/#define USE_IMTQL 1/' "$REF/eigen_GPU_batch.cu" > "$TMP/eigen_GPU_batch.cu"
if ! grep -q '^#define USE_IMTQL 1' "$TMP/eigen_GPU_batch.cu"; then
  echo "could not switch USE_IMTQL in the copy; imtql2 variant not built" >&2
  exit 0
fi
# shellcheck disable=SC2086
"$NVCC" $FLAGS -I"$REF" -shared -o "$OUT/libeigenGbatch_ref_imtql.so" "$TMP/eigen_GPU_batch.cu" -lcudart
echo "built $OUT/libeigenGbatch_ref_imtql.so"
