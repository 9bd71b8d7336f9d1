#!/usr/bin/env bash
# Compile the reference's CPU operator sources (RNS, NTT, CKKS) straight from
# the read-only reference checkout into oracle/_ref/libfhelium_ref_cpu_ops.so.
# Only g++ on the reference's own .cpp files: no CMake, no generated code.
# The library registers the torch.ops.fhelium_{rns,ntt,ckks}_ops schemas with
# their CPU kernels; tests load it with torch.ops.load_library to pin the
# oracle restatement against the reference itself.
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
SRCS=(
  "$REF/csrc/ops/rns/rns_arithmetic.cpp"
  "$REF/csrc/ops/rns/rns_canonical_arithmetic.cpp"
  "$REF/csrc/ops/ntt/forward_ntt.cpp"
  "$REF/csrc/ops/ntt/inverse_ntt.cpp"
  "$REF/csrc/ops/ckks/ckks.cpp"
  "$REF/csrc/ops/rns/cpu/rns_arithmetic_cpu.cpp"
  "$REF/csrc/ops/rns/cpu/rns_canonical_arithmetic_cpu.cpp"
  "$REF/csrc/ops/ntt/cpu/indexed_ntt_cpu.cpp"
  "$REF/csrc/ops/ckks/cpu/ckks_cpu.cpp"
)
# System g++ by default; CXX_REF overrides it.
CXX=${CXX_REF:-/usr/bin/g++}
OBJS=()
for s in "${SRCS[@]}"; do
  o="$OUT/$(basename "${s%.cpp}").o"
  $CXX -std=c++17 -O3 -fPIC -fopenmp -D_GLIBCXX_USE_CXX11_ABI=$ABI \
    -I"$TORCH_INC" -I"$TORCH_INC/torch/csrc/api/include" -I"$REF/csrc" \
    -c "$s" -o "$o" &
  OBJS+=("$o")
done
wait
$CXX -shared -fopenmp -o "$OUT/libfhelium_ref_cpu_ops.so" "${OBJS[@]}" \
  -L"$TORCH_LIB" -Wl,-rpath,"$TORCH_LIB" -ltorch -ltorch_cpu -lc10
rm -f "${OBJS[@]}"
echo "built $OUT/libfhelium_ref_cpu_ops.so"
