#!/usr/bin/env bash
# Builds the pin libraries (test infrastructure) from the reference's own
# sources, compiled in place (never copied):
#   oracle/_ref/libref_host.so  serial CPU routines of test_application.cu and
#                               spmspv.h, plus the GPU comparator (ref_pin.cu)
#   oracle/_ref/libref_csc.so   SpmSpvCSCHost of test_sort_spmspv.cu
#                               (ref_pin_csc.cu)
# The reference tree is $SPMX_REFERENCE, or else a checkout of
# hpc-research-2020/spmspv-adaptive named `reference` beside this repository's
# directory.  Without either, the recipe does nothing (the tests that need the
# libraries skip).  The reference's build system is not used; the few headers
# it takes from outside its tree get stubs here:
#   helper_cuda.h / helper_functions.h (CUDA samples), moderngpu.cuh (used only
#   under an off-by-default macro), and cusparseScsr2csc, which CUDA 12
#   removed (ToCSC calls it; the pins never do).
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${SPMX_REFERENCE:-$HERE/../../reference}
OUT="$HERE/_ref"
LA="$REF/hice-spmspv/hice/la"
if [ ! -d "$LA" ]; then echo "build_ref.sh: no reference tree at $REF (set SPMX_REFERENCE)" >&2; exit 0; fi
mkdir -p "$OUT/shim"
printf '#pragma once\n#include <cstdio>\n#define checkCudaErrors(x) (x)\n' > "$OUT/shim/helper_cuda.h"
printf '#pragma once\n' > "$OUT/shim/helper_functions.h"
printf '#pragma once\n' > "$OUT/shim/moderngpu.cuh"
cat > "$OUT/shim/cusparse_compat.h" <<'EOS'
#pragma once
#include <cusparse.h>
static inline cusparseStatus_t cusparseScsr2csc(cusparseHandle_t, int, int, int, const float*,
    const int*, const int*, float*, int*, int*, cusparseAction_t, cusparseIndexBase_t) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}
static inline cusparseStatus_t cusparseDcsr2csc(cusparseHandle_t, int, int, int, const double*,
    const int*, const int*, double*, int*, int*, cusparseAction_t, cusparseIndexBase_t) {
  return CUSPARSE_STATUS_NOT_SUPPORTED;
}
EOS
FLAGS=(-O2 -std=c++14 -gencode arch=compute_100a,code=sm_100a -shared -Xcompiler -fPIC,-fopenmp,-fpermissive
       -Xcudafe --diag_suppress=2361 -w -include sstream -include "$OUT/shim/cusparse_compat.h"
       -I"$OUT/shim" -I"$LA/include" -I"$LA/include/spmspv/csc-spmspv" -DVALUE_TYPE=float -DNUM_RUN=10)

# build <output> <pin source> <-D define naming the reference file>
build() {
  local so="$1" src="$2" def="$3"
  if [ -f "$so" ] && [ "$so" -nt "$src" ] && [ "$so" -nt "$0" ]; then return 0; fi
  nvcc "${FLAGS[@]}" "$def" -o "$so" "$src" -lcusparse -lgomp
  echo "built $so"
}
build "$OUT/libref_host.so" "$HERE/ref_pin.cu" "-DREF_TEST_APPLICATION=\"$LA/test/test_application.cu\""
build "$OUT/libref_csc.so" "$HERE/ref_pin_csc.cu" "-DREF_TEST_SORT_SPMSPV=\"$LA/test/test_sort_spmspv.cu\""
