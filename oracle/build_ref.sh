#!/usr/bin/env bash
# Builds oracle/_ref/libref_host.so: the reference's own serial CPU routines,
# compiled from its sources in place (never copied) with ref_pin.cu as the
# entry layer.  Test infrastructure only.  The reference's build system is not
# used; the few headers it takes from outside its tree get stubs here:
#   helper_cuda.h / helper_functions.h (CUDA samples), moderngpu.cuh (used only
#   under an off-by-default macro), and cusparseScsr2csc, which CUDA 12
#   removed (ToCSC calls it; the pin never does).
set -euo pipefail
REF=${SPMX_REFERENCE:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
LA="$REF/hice-spmspv/hice/la"
if [ ! -d "$LA" ]; then echo "build_ref.sh: no reference at $REF" >&2; exit 0; fi
SO="$OUT/libref_host.so"
if [ -f "$SO" ] && [ "$SO" -nt "$HERE/ref_pin.cu" ] && [ "$SO" -nt "$0" ]; then exit 0; fi
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
nvcc -O2 -std=c++14 -gencode arch=compute_100a,code=sm_100a -shared -Xcompiler -fPIC,-fopenmp,-fpermissive \
  -Xcudafe --diag_suppress=2361 -w -include sstream -include "$OUT/shim/cusparse_compat.h" \
  -I"$OUT/shim" -I"$LA/include" -I"$LA/include/spmspv/csc-spmspv" \
  -DVALUE_TYPE=float -DNUM_RUN=10 \
  "-DREF_TEST_APPLICATION=\"$LA/test/test_application.cu\"" \
  -o "$SO" "$HERE/ref_pin.cu" -lcusparse -lgomp
echo "built $SO"
