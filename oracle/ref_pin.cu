// Pin harness (test infrastructure): exposes the reference's OWN serial CPU
// routines, compiled from its sources where they lie (oracle/build_ref.sh
// passes the path), so the oracle's restatements can be checked against
// them.  Nothing here is a copy of reference code; the reference file is
// #included at build time.
//   serialspmv              hice-spmspv/hice/la/test/test_application.cu:107-116
//   computeMatFeture_serial include/spmspv/csc-spmspv/spmspv.h:2275-2335
//   extractMatFeature       include/spmspv/csc-spmspv/spmspv.h:423-447
//   ReadMTX (+ its sort)    include/spmspv/mtx.hpp:218-361
//   storeCSR / loadCSR_header / loadCSR   include/spmspv/mtx.hpp:750-808
//   COO2Hybrid              include/spmspv/mtx.hpp:436-701
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

// ReadMTX exits the process on a file it cannot open: pass readable files only.
extern "C" void ref_read_mtx(const char* path, int* m, int* n, int* nnz, int** row, int** col,
                             float** val) {
  MTX<float> mtx;
  ReadMTX<float>(path, &mtx, true);
  *m = mtx.rows; *n = mtx.cols; *nnz = mtx.nnz;
  *row = mtx.row; *col = mtx.col; *val = mtx.data;
}

extern "C" void ref_free(void* p) { free(p); }

extern "C" void ref_store_csr(const char* path, int m, int n, int nnz, int* rowptr, int* col,
                              float* val) {
  storeCSR<float>(m, n, nnz, rowptr, col, val, path);
}

extern "C" int ref_load_csr(const char* path, int* m, int* n, int* nnz, int* rowptr, int* col,
                            float* val, int cap_m, int cap_nnz) {
  try {
    loadCSR_header(path, m, n, nnz);
    if (*m > cap_m || *nnz > cap_nnz) return -2;
    return loadCSR<float>(path, *m, *n, *nnz, rowptr, col, val);
  } catch (...) {
    return -1;
  }
}

// COO2Hybrid sizes its count arrays by nnz: pass nnz >= max(rows, cols).
// On return the first *csr_nnz entries are the CSR part, sorted by (row,
// column), the rest the CSC part, sorted by (column, row).
extern "C" void ref_coo2hybrid(int m, int n, int nnz, int* row, int* col, float* val, int* csr_nnz) {
  COO2Hybrid<float>(1, m, n, nnz, row, col, val, csr_nnz);
}
