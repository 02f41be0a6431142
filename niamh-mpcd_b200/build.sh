#!/usr/bin/env bash
# Builds libmpcd_gpu.so (sm_100a) in-tree: niamh-mpcd_b200/libmpcd_gpu.so
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo -std=c++17 \
    -Xcompiler -fPIC -Xcompiler -Wall -shared \
    -I"$HERE/../include" -I"$HERE/csrc" \
    "$HERE/csrc/mpcd_api.cu" "$HERE/csrc/mpcd_noalloc.cu" "$HERE/csrc/mpcd_batch.cu" "$HERE/csrc/mpcd_tune.cu" "$HERE/csrc/mpcd_ckpt.cpp" "$HERE/csrc/mpcd_out.cpp" -o "$HERE/libmpcd_gpu.so" ${MPCD_NVCC_EXTRA:-}
