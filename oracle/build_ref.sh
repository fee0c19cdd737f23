#!/usr/bin/env bash
# Builds the checker libraries.  TEST INFRASTRUCTURE ONLY.
#
#   oracle/libpj_oracle.so        the C restatement (oracle/pj_oracle.c)
#   oracle/_ref/libref_cpu.so     the reference's own host code (murmur hash,
#                                 int_fastdiv slot, inner_join_cpu) behind
#                                 oracle/ref/ref_cpu_adapter.cu
#   oracle/_ref/libref_gpu_k4.so  the reference's own GPU join stages for
#   oracle/_ref/libref_gpu_k8.so  4- and 8-byte keys behind
#                                 oracle/ref/ref_gpu_adapter.cu (sm_100a)
#
# The reference libraries are compiled straight from the reference tree's
# headers (read-only, never copied); they are skipped when the tree is absent.
# Outputs go only to oracle/ and oracle/_ref/.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${PJ_REFERENCE_DIR:-/root/reference}"
NVCC="${NVCC:-nvcc}"
mkdir -p "$HERE/_ref"

gcc -O2 -std=c99 -fPIC -shared "$HERE/pj_oracle.c" -o "$HERE/libpj_oracle.so"

if [ ! -d "$REF/src" ]; then
    echo "build_ref.sh: reference tree $REF not found; reference checker libraries not rebuilt" >&2
    exit 0
fi

# -std=c++17 because CCCL 12.9 requires it (the reference Makefile says c++14);
# -lnvToolsExt is dropped: the reference only uses NVTX under -DUSE_NVTX.
"$NVCC" -std=c++17 -O2 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fopenmp,-fPIC -shared -I"$REF/src" \
    "$HERE/ref/ref_cpu_adapter.cu" -o "$HERE/_ref/libref_cpu.so" -lgomp

GPU_FLAGS=(-std=c++17 -O3 -Xcompiler -fPIC -shared --expt-extended-lambda --expt-relaxed-constexpr
           -gencode arch=compute_100a,code=sm_100a -I"$REF/src")
"$NVCC" "${GPU_FLAGS[@]}" "$HERE/ref/ref_gpu_adapter.cu" -o "$HERE/_ref/libref_gpu_k4.so"
"$NVCC" "${GPU_FLAGS[@]}" -DUSE_8B_KEYS "$HERE/ref/ref_gpu_adapter.cu" -o "$HERE/_ref/libref_gpu_k8.so"
echo "build_ref.sh: done"
