#!/usr/bin/env bash
# Compile the reference's operator library WITH its CUDA kernels, straight
# from the read-only reference checkout, for sm_100a, into
# oracle/_ref/libfhelium_ref_ops_cuda.so: the schema definitions, the CPU
# kernels and the CUDA kernels (csrc/ops/*/cuda/*.cu, relocatable device code
# as the reference's own build uses) of fhelium_{rns,ntt,ckks}_ops.  Only
# nvcc and g++ on the reference's own files: no CMake, no generated code.
# It replaces libfhelium_ref_cpu_ops.so in a process that times the
# reference's CUDA kernels (both define the same schemas, so a process loads
# one of them).
set -euo pipefail
REF=${FHELIUM_REFERENCE:-/root/reference}
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
if [ ! -d "$REF/csrc/ops" ]; then
  echo "reference sources not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
PY=${PYTHON:-python}
TORCH_INC=$($PY -c 'import torch, os; print(os.path.join(os.path.dirname(torch.__file__), "include"))')
TORCH_LIB=$($PY -c 'import torch, os; print(os.path.join(os.path.dirname(torch.__file__), "lib"))')
ABI=$($PY -c 'import torch; print(int(torch._C._GLIBCXX_USE_CXX11_ABI))')
CUDA_HOME=${CUDA_HOME:-/usr/local/cuda}
NVCC=${NVCC:-$CUDA_HOME/bin/nvcc}
CXX=${CXX_REF:-/usr/bin/g++}
ARCH="-gencode arch=compute_100a,code=sm_100a"
INC=(-I"$TORCH_INC" -I"$TORCH_INC/torch/csrc/api/include" -I"$REF/csrc" -I"$CUDA_HOME/include")
TMP="$OUT/cuda_build"
mkdir -p "$TMP"
CPP_SRCS=(
  "$REF"/csrc/ops/rns/rns_arithmetic.cpp
  "$REF"/csrc/ops/rns/rns_canonical_arithmetic.cpp
  "$REF"/csrc/ops/ntt/forward_ntt.cpp
  "$REF"/csrc/ops/ntt/inverse_ntt.cpp
  "$REF"/csrc/ops/ckks/ckks.cpp
  "$REF"/csrc/ops/rns/cpu/*.cpp
  "$REF"/csrc/ops/ntt/cpu/*.cpp
  "$REF"/csrc/ops/ckks/cpu/*.cpp
  "$REF"/csrc/ops/rns/cuda/*.cpp
  "$REF"/csrc/ops/ntt/cuda/*.cpp
  "$REF"/csrc/ops/ckks/cuda/*.cpp
)
CU_SRCS=("$REF"/csrc/ops/*/cuda/*.cu)
OBJS=()
CU_OBJS=()
for s in "${CPP_SRCS[@]}"; do
  o="$TMP/$(basename "$(dirname "$(dirname "$s")")")_$(basename "$(dirname "$s")")_$(basename "${s%.cpp}").o"
  $CXX -std=c++17 -O3 -fPIC -fopenmp -D_GLIBCXX_USE_CXX11_ABI=$ABI "${INC[@]}" -c "$s" -o "$o" &
  OBJS+=("$o")
done
for s in "${CU_SRCS[@]}"; do
  o="$TMP/$(basename "$(dirname "$(dirname "$s")")")_cu_$(basename "${s%.cu}").o"
  $NVCC $ARCH -std=c++17 -O3 -rdc=true -Xcompiler -fPIC -D_GLIBCXX_USE_CXX11_ABI=$ABI "${INC[@]}" \
    -c "$s" -o "$o" &
  CU_OBJS+=("$o")
done
wait
$NVCC $ARCH -dlink -Xcompiler -fPIC -o "$TMP/dlink.o" "${CU_OBJS[@]}"
$CXX -shared -fopenmp -o "$OUT/libfhelium_ref_ops_cuda.so" "${OBJS[@]}" "${CU_OBJS[@]}" "$TMP/dlink.o" \
  -L"$TORCH_LIB" -Wl,-rpath,"$TORCH_LIB" -ltorch -ltorch_cpu -ltorch_cuda -lc10 -lc10_cuda \
  -L"$CUDA_HOME/lib64" -lcudart
rm -rf "$TMP"
echo "built $OUT/libfhelium_ref_ops_cuda.so"
