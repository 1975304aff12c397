// Pin harness (test infrastructure): exposes the reference's OWN host CSC
// SpMSpV, SpmSpvCSCHost (hice-spmspv/hice/la/test/test_sort_spmspv.cu:330-375),
// compiled from its source file where it lies (oracle/build_ref.sh passes the
// path), so that the oracle's restatement can be checked against it bit for
// bit.  Nothing here is a copy of reference code; the reference file is
// #included at build time.
//
// That test file no longer compiles against the reference's own handle: its
// TestCscSortSpmspv (test_sort_spmspv.cu:480-513) constructs the handle with
// two arguments and calls InputCsr / ToCsc / CscBasedSortSpmspv, which the
// handle (spmspv.h:88-344) no longer has.  The file is therefore compiled with
// the handle's name mapped to SpmxStaleDriverHandle below, a class that
// accepts those calls and does nothing.  TestCscSortSpmspv is never called;
// SpmSpvCSCHost does not use the handle at all.
#include "spmspv/csc-spmspv/spmspv.h"  // the real handle first; its guard keeps the file's own include a no-op

template <class I, class U, class V>
struct SpmxStaleDriverHandle {
  SpmxStaleDriverHandle(I, I) {}
  template <class... T> int InputCsr(T...) { return -1; }
  template <class... T> int set_sparse_x(T...) { return -1; }
  int ToCsc() { return -1; }
  template <class... T> int CscBasedSortSpmspv(T...) { return -1; }
  int Destroy() { return -1; }
};

#define SpmspvHandle SpmxStaleDriverHandle
#define main spmx_reference_test_sort_spmspv_main
#include REF_TEST_SORT_SPMSPV
#undef main
#undef SpmspvHandle

// y = A * x for a sparse x over a CSC (csc_col = column pointer, csc_row = row
// indices), written as the sparse (key, value) list of y's entries that are
// not IS_FLOAT_ZERO, in row order; *y_nnz receives their count.  y_key and
// y_val need room for m entries.
extern "C" void ref_spmspv_csc_host(int m, int n, int nnz, int* csc_row, int* csc_col,
                                    float* csc_val, int x_nnz, int* x_key, float* x_val,
                                    int* y_nnz, int* y_key, float* y_val) {
  SpmSpvCSCHost(m, n, nnz, csc_row, csc_col, csc_val, x_nnz, x_key, x_val, y_nnz, y_key, y_val);
}
