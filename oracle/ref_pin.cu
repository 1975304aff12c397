// Pin harness (test infrastructure): exposes the reference's OWN serial CPU
// routines, compiled from its sources where they lie (oracle/build_ref.sh
// passes the path), so the oracle's restatements can be checked against
// them.  Nothing here is a copy of reference code; the reference file is
// #included at build time.
//   serialspmv              hice-spmspv/hice/la/test/test_application.cu:107-116
//   computeMatFeture_serial include/spmspv/csc-spmspv/spmspv.h:2275-2335
//   extractMatFeature       include/spmspv/csc-spmspv/spmspv.h:423-447
#define main spmx_reference_test_application_main
#include REF_TEST_APPLICATION
#undef main

extern "C" void ref_serialspmv(int m, int n, int nnz, int* rowptr, int* col, float* val,
                               float* x, float* y, float alpha) {
  serialspmv(m, n, nnz, rowptr, col, val, x, y, alpha);
}

extern "C" void ref_mat_features(int m, int n, int nnz, int* rowptr, float* out7) {
  SpmspvHandle<int, unsigned, float> A(m, n, nnz);
  int mx = 0, mn = 0;
  float avg = 0, rng = 0, sd = 0, eq = 0, gini = 0;
  A.computeMatFeture_serial(m, n, nnz, rowptr, &mx, &mn, &avg, &rng, &sd, &eq, &gini);
  out7[0] = (float)mx; out7[1] = (float)mn; out7[2] = avg; out7[3] = rng;
  out7[4] = sd; out7[5] = eq; out7[6] = gini;
}

extern "C" float ref_std_row(int m, int n, int nnz, int* rowptr) {
  SpmspvHandle<int, unsigned, float> A(m, n, nnz);
  return A.extractMatFeature(rowptr);
}
