#!/usr/bin/env bash
# Build the reference cudaSAXS, unmodified, from its own sources into oracle/_ref/.
#
# Test infrastructure only: the outputs are the reference's own pybind module
# (pycusaxs_cuda*.so) and a small kernel harness (libref_kernels.so, built from
# oracle/csrc/ref_harness.cu, which #includes the reference's device-kernel
# sources where they lie).  Nothing here is shipped or called by the product.
#
# The reference's CMake cannot be used as is (it runs nvidia-smi at configure
# time and forces arch 75;80;86;89), so this recipe compiles its 13 translation
# units directly with nvcc for sm_100a, mirroring its CMake options
# (cpp-src/Saxs/CMakeLists.txt:73-79, Exec/CMakeLists.txt:75-80): separable
# compilation, --expt-relaxed-constexpr, --expt-extended-lambda, C++17; fmt is
# the header-only copy that ships with torch.
#
# usage: oracle/build_ref.sh <reference-root>
set -euo pipefail

if [ $# -lt 1 ]; then
  echo "usage: oracle/build_ref.sh <reference-root>" >&2
  exit 2
fi
REF=$1
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
SRC="$REF/cpp-src"
if [ ! -d "$SRC" ]; then
  echo "build_ref: reference sources not found under $REF" >&2
  exit 2
fi
PY=${PYTHON:-python}
mkdir -p "$OUT/obj" "$OUT/inc"

PYINC=$($PY -c "import sysconfig;print(sysconfig.get_paths()['include'])")
PBINC=$($PY -c "import pybind11;print(pybind11.get_include())")
TORCHINC=$($PY -c "import torch,os;print(os.path.join(os.path.dirname(torch.__file__),'include'))")
EXT=$($PY -c "import sysconfig;print(sysconfig.get_config_var('EXT_SUFFIX'))")
# expose only fmt from torch's include tree (torch also ships its own pybind11)
ln -sfn "$TORCHINC/fmt" "$OUT/inc/fmt"

INCS=(-I"$SRC/include" -I"$SRC/Saxs" -I"$SRC/Exec" -I"$SRC/Utilities" -I"$SRC/System"
      -I"$PBINC" -I"$PYINC" -I"$OUT/inc")
ARCH=(-gencode arch=compute_100a,code=sm_100a)
NVFLAGS=(-O3 -std=c++17 -rdc=true -Xcompiler -fPIC "${ARCH[@]}" --expt-relaxed-constexpr
         --expt-extended-lambda -diag-suppress=2417,128 -DFMT_HEADER_ONLY=1 -w)

SOURCES=(
  Utilities/BSpmod.cpp Utilities/BSpline.cpp Utilities/Scattering.cpp
  System/Cell.cpp System/AtomCounter.cpp
  Saxs/saxsDeviceKernels.cu Saxs/Splines.cu Saxs/opsfact.cu Saxs/saxsKernel.cu
  Exec/RunSaxs.cu Exec/Options.cpp
  cudaSAXS.cu pybind/cuda_bindings.cpp
)

OBJS=()
for s in "${SOURCES[@]}"; do
  o="$OUT/obj/$(echo "$s" | tr '/' '_').o"
  if [[ "$s" == *.cu ]]; then
    nvcc "${NVFLAGS[@]}" "${INCS[@]}" -x cu -c "$SRC/$s" -o "$o"
  else
    nvcc "${NVFLAGS[@]}" "${INCS[@]}" -x c++ -c "$SRC/$s" -o "$o"
  fi
  OBJS+=("$o")
done

nvcc "${ARCH[@]}" -Xcompiler -fPIC -dlink "${OBJS[@]}" -o "$OUT/obj/dlink.o" -lcudadevrt
g++ -shared -o "$OUT/pycusaxs_cuda$EXT" "${OBJS[@]}" "$OUT/obj/dlink.o" \
    -L/usr/local/cuda/lib64 -lcufft -lcudadevrt -lcudart -Wl,-rpath,/usr/local/cuda/lib64

# kernel harness: the reference's calculate_histogram / rhoCartKernel behind a C entry point
nvcc -O3 -std=c++17 -Xcompiler -fPIC "${ARCH[@]}" --expt-relaxed-constexpr -w \
     -I"$SRC/include" -I"$SRC/Saxs" -DREF_SRC_DIR="\"$SRC\"" \
     -shared "$HERE/csrc/ref_harness.cu" -o "$OUT/libref_kernels.so"

echo "build_ref: wrote $OUT/pycusaxs_cuda$EXT and $OUT/libref_kernels.so"
