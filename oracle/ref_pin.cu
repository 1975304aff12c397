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

// The reference's serialspmv on all OpenMP threads: rows are independent, so
// each slice [r0, r1) of `nslices` nnz-balanced slices (bounds[0..nslices])
// runs the reference routine on its own rows (bit-identical y).
extern "C" void ref_serialspmv_slices(int nslices, const int* bounds, int m, int n, int nnz, int* rowptr,
                                      int* col, float* val, float* x, float* y, float alpha) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int q = 0; q < nslices; ++q) {
    const int r0 = bounds[q], r1 = bounds[q + 1];
    if (r1 > r0) serialspmv(r1 - r0, n, nnz, rowptr + r0, col, val, x, y + r0, alpha);
  }
  (void)m;
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

// GPU comparator (test infrastructure): the reference's own SpMV / SpMSpV
// kernels, compiled for sm_100a from its sources, timed with CUDA events on
// the default stream, with a 256 MiB memset before each call to flush L2.
// Only kernels without waits between thread blocks and without a known
// out-of-bounds access run here: Hola SpMV (holaspmv.h), the naive CSR SpMV
// (naivespmv.h) and the atomic naive CSC SpMSpV (CscBasedNoSortNaiveSpmspv,
// csc_sort_spmspv.cuh:98-119).  The merge-path and sort CSC variants use a
// chained scan whose blocks spin without a bound on the previous block's sum
// (scan_kernel.cuh:99, :232), so they are not run.  CSR5 is not built into
// this comparator at all: its descriptor kernel
// (generate_partition_descriptor_s1_kernel, format_conversion.h:147-163)
// maps a row that starts at offset nnz (an empty last row) to tile
// nnz / (omega * sigma), which is one past the last tile when nnz is a
// multiple of omega * sigma, and its atomicOr then writes one word past the
// descriptor array (spmspv.h:1464).
//   which: 0 Hola SpMV, 2 naive SpMV, 3 CSC naive atomic SpMSpV; any other
//   value returns -1 without touching the device.
// All arrays are host arrays; the function makes its own device copies.
// ms_out[reps] receives each call's time, y_out[m] the last result.
// Returns 0, or -1 after a CUDA error or for an unknown `which`.
namespace {
template <class T>
T* dcopy(const T* h, size_t count) {
  T* d = nullptr;
  if (cudaMalloc((void**)&d, sizeof(T) * (count ? count : 1)) != cudaSuccess) return nullptr;
  if (count && h) cudaMemcpy(d, h, sizeof(T) * count, cudaMemcpyHostToDevice);
  return d;
}
}  // namespace

// Number of CUDA devices this process can use (0 without a GPU or driver).
extern "C" int ref_gpu_count() {
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return c;
}

extern "C" int ref_gpu_time(int which, int m, int n, int nnz, const int* rowptr, const int* col,
                            const float* val, const int* colptr, const int* crow, const float* cval,
                            const float* x, int x_nnz, const int* xkey, const float* xval, int reps,
                            float* ms_out, float* y_out) {
  if (which != 0 && which != 2 && which != 3) return -1;
  int* d_rp = dcopy(rowptr, (size_t)m + 1);
  int* d_col = dcopy(col, (size_t)nnz);
  float* d_val = dcopy(val, (size_t)nnz);
  int* d_cp = which == 3 ? dcopy(colptr, (size_t)n + 1) : nullptr;
  int* d_crow = which == 3 ? dcopy(crow, (size_t)nnz) : nullptr;
  float* d_cval = which == 3 ? dcopy(cval, (size_t)nnz) : nullptr;
  float* d_x = dcopy(x, (size_t)n);
  int* d_xkey = which == 3 ? dcopy(xkey, (size_t)x_nnz) : nullptr;
  float* d_xval = which == 3 ? dcopy(xval, (size_t)x_nnz) : nullptr;
  float* d_y = dcopy<float>(nullptr, (size_t)m);
  char* flush = dcopy<char>(nullptr, (size_t)256 << 20);
  const bool csc = which == 3;
  if (!d_rp || !d_col || !d_val || !d_x || !d_y || !flush ||
      (csc && (!d_cp || !d_crow || !d_cval || !d_xkey || !d_xval))) {
    cudaFree(d_rp); cudaFree(d_col); cudaFree(d_val); cudaFree(d_cp); cudaFree(d_crow);
    cudaFree(d_cval); cudaFree(d_x); cudaFree(d_xkey); cudaFree(d_xval); cudaFree(d_y);
    cudaFree(flush);
    cudaGetLastError();
    return -1;
  }
  SpmspvHandle<int, unsigned int, float> A(m, n, nnz);
  if (which == 3) {
    A.InputCSC(nnz, d_crow, d_cp, d_cval);
    A.set_sparse_x(d_xkey, d_xval, x_nnz);
    A.allocPreBuffer();
  } else {
    A.InputCSR(nnz, d_rp, d_col, d_val);
    A.set_x(d_x);
    if (which == 0) A.holaPreprocess();
  }
  auto call = [&]() {
    int ynnz = 0;
    if (which == 0) A.holaspmv(1.0f, d_y);
    else if (which == 2) A.naivespmv(1.0f, d_y);
    else A.CscBasedNoSortNaiveSpmspv(1.0f, &ynnz, d_y);
  };
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int w = 0; w < 2; ++w) call();
  for (int r = 0; r < reps; ++r) {
    cudaMemset(flush, r & 0xff, (size_t)256 << 20);
    cudaEventRecord(e0, 0);
    call();
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms_out[r], e0, e1);
  }
  if (y_out) cudaMemcpy(y_out, d_y, sizeof(float) * (size_t)m, cudaMemcpyDeviceToHost);
  const cudaError_t err = cudaDeviceSynchronize();
  if (which == 0) A.holaPostprocess();
  if (which == 3) A.deallocPreBuffer();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_rp); cudaFree(d_col); cudaFree(d_val); cudaFree(d_cp); cudaFree(d_crow); cudaFree(d_cval);
  cudaFree(d_x); cudaFree(d_xkey); cudaFree(d_xval); cudaFree(d_y); cudaFree(flush);
  return err == cudaSuccess ? 0 : -1;
}
