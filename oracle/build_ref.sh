#!/usr/bin/env bash
# ORACLE — test and benchmark infrastructure only. Compiles the reference's own GPU
# circle FFT and sum-check kernels from their source in the reference tree, for sm_100a,
# and the host drivers that call them the way src/cuda/circlefft_gpu.zig and
# src/cuda/sumcheck_gpu.zig do, into oracle/_ref/ (git-ignored; the built files travel with the repository to the GPU
# host, which has no reference tree). Nothing is copied out of the reference tree.
#   REF: the reference checkout (default /root/reference)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${REF:-/root/reference}"
SRC="$REF/src/cuda/kernels/circlefft.cu"
OUT="$HERE/_ref"
if [ ! -f "$SRC" ]; then
  echo "build_ref.sh: $SRC not found; the reference GPU circle FFT is not built" >&2
  exit 0
fi
mkdir -p "$OUT"
NVCC="${NVCC:-nvcc}"
CUDA_HOME="${CUDA_HOME:-/usr/local/cuda}"
if [ ! "$OUT/circlefft.cubin" -nt "$SRC" ]; then
  "$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 -cubin -o "$OUT/circlefft.cubin" "$SRC"
fi
CXX="$(test -x /usr/bin/g++ && echo /usr/bin/g++ || echo g++)"
if [ ! "$OUT/libref_circlefft.so" -nt "$HERE/ref_circlefft_driver.cpp" ] || \
   [ ! "$OUT/libref_circlefft.so" -nt "$HERE/circle.hpp" ]; then
  "$CXX" -O2 -std=c++17 -fPIC -shared -I"$HERE" -I"$CUDA_HOME/include" \
    -o "$OUT/libref_circlefft.so" "$HERE/ref_circlefft_driver.cpp" -L"$CUDA_HOME/lib64/stubs" -lcuda
fi

SC_SRC="$REF/src/cuda/kernels/sumcheck.cu"
if [ -f "$SC_SRC" ]; then
  if [ ! "$OUT/sumcheck.cubin" -nt "$SC_SRC" ]; then
    "$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 -cubin -I"$REF/src/cuda/kernels" \
      -o "$OUT/sumcheck.cubin" "$SC_SRC"
  fi
  if [ ! "$OUT/libref_sumcheck.so" -nt "$HERE/ref_sumcheck_driver.cpp" ]; then
    "$CXX" -O2 -std=c++17 -fPIC -shared -I"$CUDA_HOME/include" \
      -o "$OUT/libref_sumcheck.so" "$HERE/ref_sumcheck_driver.cpp" -L"$CUDA_HOME/lib64/stubs" -lcuda
  fi
fi
