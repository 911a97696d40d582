#!/usr/bin/env bash
# Test infrastructure only: compiles the REFERENCE extension (rpn_cuda_native) from its own
# sources, where they lie in the read-only reference checkout, into oracle/_ref/.  The result is
# used solely as a parity checker on the GPU box (tests and golden-fixture generation); no product
# code loads it.  The reference's own setup.py is not run: this recipe calls nvcc/g++ directly.
#
# Two variants are built:
#   oracle/_ref/fastmath/  -- the reference's shipped nvcc flags (-O3 --use_fast_math)
#   oracle/_ref/precise/   -- the same sources without --use_fast_math (IEEE sinf/expf/div ...)
#
# Usage: oracle/build_ref.sh REFERENCE_ROOT      (the reference checkout)
set -euo pipefail
REF_ROOT="${1:?usage: oracle/build_ref.sh REFERENCE_ROOT}"
SRC="$REF_ROOT/src/warpsymbolic/gpu/cuda"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
if [ ! -d "$SRC" ]; then
  echo "reference sources not found at $SRC; skipping" >&2
  exit 0
fi
PY=${PYTHON:-python}
read -r TORCH_INC TORCH_API_INC TORCH_LIB PY_INC EXT_SUFFIX ABI < <($PY - <<'EOF'
import os, sysconfig, torch
base = os.path.dirname(torch.__file__)
print(os.path.join(base, "include"), os.path.join(base, "include", "torch", "csrc", "api", "include"),
      os.path.join(base, "lib"), sysconfig.get_paths()["include"], sysconfig.get_config_var("EXT_SUFFIX"),
      int(torch._C._GLIBCXX_USE_CXX11_ABI))
EOF
)
CUDA_HOME=${CUDA_HOME:-/usr/local/cuda}
COMMON_DEFS="-DTORCH_EXTENSION_NAME=rpn_cuda_native -DTORCH_API_INCLUDE_EXTENSION_H -D_GLIBCXX_USE_CXX11_ABI=$ABI"
INCS="-I$TORCH_INC -I$TORCH_API_INC -I$CUDA_HOME/include -I$PY_INC"
CU_SOURCES="rpn_kernels pso_kernels fused_pso_kernels simplify_kernels genrand_kernels backward_kernels diversity_kernels lbfgs_kernels best_tracker_kernels"
CPP_SOURCES="bindings decoder"
JOBS=${JOBS:-8}

build_variant() {
  local name="$1"; shift
  local nvflags="$*"
  local dir="$OUT/$name"
  mkdir -p "$dir/obj"
  local stamp="$dir/rpn_cuda_native$EXT_SUFFIX"
  if [ -f "$stamp" ]; then echo "[build_ref] $name: up to date"; return; fi
  local pids=()
  for s in $CU_SOURCES; do
    nvcc -c "$SRC/$s.cu" -o "$dir/obj/$s.o" $COMMON_DEFS $INCS -std=c++17 -Xcompiler -fPIC \
      -gencode arch=compute_100,code=sm_100 -O3 $nvflags -Xcudafe --diag_suppress=221 -w &
    pids+=($!)
    if [ ${#pids[@]} -ge $JOBS ]; then wait "${pids[0]}"; pids=("${pids[@]:1}"); fi
  done
  for s in $CPP_SOURCES; do
    g++ -c "$SRC/$s.cpp" -o "$dir/obj/$s.o" $COMMON_DEFS $INCS -std=c++17 -fPIC -O3 -w &
    pids+=($!)
  done
  for p in "${pids[@]}"; do wait "$p"; done
  g++ -shared -o "$stamp" "$dir"/obj/*.o -L"$TORCH_LIB" -L"$CUDA_HOME/lib64" \
    -lc10 -lc10_cuda -ltorch -ltorch_cpu -ltorch_cuda -ltorch_python -lcudart \
    -Wl,-rpath,"$TORCH_LIB"
  rm -rf "$dir/obj"
  echo "[build_ref] $name: built $stamp"
}

build_variant fastmath --use_fast_math
build_variant precise
