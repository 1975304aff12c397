/*
 * spmx_oracle.c — CPU oracle for the adaptive SpMV / SpMSpV path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the tests, the smoke
 * check and the CPU-baseline leg of the benchmark load it; the product (the
 * CUDA library) never does.
 *
 * Each function restates a CPU routine of hpc-research-2020/spmspv-adaptive
 * (paths relative to hice-spmspv/hice/la/):
 *   - serialspmv                 test/test_application.cu:107-116
 *   - SpmSpvCSCHost              test/test_sort_spmspv.cu:330-375 (FP64 and
 *                                faithful forms)
 *   - computeMatFeture_serial    include/spmspv/csc-spmspv/spmspv.h:2275-2335
 *   - extractMatFeature (stdRow) include/spmspv/csc-spmspv/spmspv.h:423-447
 *   - computeVecFeture_serial    include/spmspv/csc-spmspv/spmspv.h:2338-2361
 *   - computeGM1/2/3             include/spmspv/csc-spmspv/spmspv.h:2727-2752
 *   - setSigma (auto rule)       include/spmspv/csc-spmspv/spmspv.h:1396-1416
 *   - updateFlag/streamCompact   include/spmspv/csc-spmspv/spmspv.h:1122-1175
 *   - scatter / bitvector        spmspv.h:1226-1308, detail/device/bitvector.h
 *   - ReadMTX + its sort         include/spmspv/mtx.hpp:218-361
 *   - COO2Hybrid (row priority)  include/spmspv/mtx.hpp:436-701
 * The reference has no BFS and no adjoint; those oracles are restated from
 * their definitions (level-synchronous Boolean SpMSpV with a visited mask, in
 * the loop structure of SpmSpvCSCHost; dx = A^T dy, dvals = dy[row]*x[col]).
 *
 * Parity status: the reference ships no golden vectors or fixtures for this
 * path; the restatements are pinned against the reference's own host code
 * compiled from its sources (oracle/build_ref.sh -> oracle/_ref) where that
 * builds, as recorded by tests/test_oracle_pin.py.
 *
 * It also holds a CSR -> CSC transpose and a restatement of the benchmark's
 * synthetic input generators (end of file), so the CPU legs of the benchmark
 * need nothing from the product library.
 *
 * Deliberate departures from the reference, each noted at its function:
 *   - SpmSpvCSCHost reads x_val into an int (test_sort_spmspv.cu:340); the
 *     FP64 oracle keeps the value (the faithful form truncates).
 *   - accumulation is FP64 unless the function is marked "faithful".
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <limits.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EXPORT __attribute__((visibility("default")))

/* ---- SpMV ---------------------------------------------------------------- */

/* serialspmv, faithful: FP32 accumulation, product order x*val*alpha
 * (test_application.cu:107-116). */
EXPORT void oracle_serialspmv_f32(int m, const int* rowptr, const int* col,
                                  const float* val, const float* x, float* y,
                                  float alpha) {
  for (int i = 0; i < m; i++) {
    float sum = 0;
    for (int j = rowptr[i]; j < rowptr[i + 1]; j++) sum += x[col[j]] * val[j] * alpha;
    y[i] = sum;
  }
}

/* serialspmv in FP64; also returns sum_j |a_ij x_j| per row (the magnitude
 * that scales the FP32 tolerance).  `bits` (may be NULL) gates x like
 * naive_spmspv_ker (detail/device/naivespmv.h:13-31). */
EXPORT void oracle_spmv_f64(int m, const int* rowptr, const int* col,
                            const float* val, const float* x, const int* bits,
                            double alpha, double* y, double* absy) {
#pragma omp parallel for schedule(dynamic, 1024)
  for (int i = 0; i < m; i++) {
    double s = 0, a = 0;
    for (int j = rowptr[i]; j < rowptr[i + 1]; j++) {
      const int c = col[j];
      if (bits && !((((const unsigned*)bits)[c >> 5] >> (c & 31)) & 1u)) continue;
      const double p = (double)val[j] * (double)x[c];
      s += p;
      a += fabs(p);
    }
    y[i] = alpha * s;
    if (absy) absy[i] = fabs(alpha) * a;
  }
}

/* ---- CSC SpMSpV ------------------------------------------------------------ */

/* SpmSpvCSCHost (test_sort_spmspv.cu:330-375) in FP64 with the x value kept
 * as a float (the reference truncates it to int).  Writes the dense result
 * y[m], its magnitude absy[m] and touched[m] (1 if row i appears in any
 * selected column: the structural output of the sort write-back). */
EXPORT void oracle_spmspv_csc_f64(int m, const int* colptr, const int* row,
                                  const float* val, int x_nnz, const int* x_key,
                                  const float* x_val, double alpha, double* y,
                                  double* absy, unsigned char* touched) {
  memset(y, 0, sizeof(double) * (size_t)m);
  if (absy) memset(absy, 0, sizeof(double) * (size_t)m);
  if (touched) memset(touched, 0, (size_t)m);
  for (int i = 0; i < x_nnz; i++) {
    const int c = x_key[i];
    const double xv = (double)x_val[i];
    for (int j = colptr[c]; j < colptr[c + 1]; j++) {
      const double p = (double)val[j] * xv;
      y[row[j]] += p;
      if (absy) absy[row[j]] += fabs(p);
      if (touched) touched[row[j]] = 1;
    }
  }
  for (int r = 0; r < m; r++) {
    y[r] *= alpha;
    if (absy) absy[r] *= fabs(alpha);
  }
}

/* The reference's CPU sparse output of SpmSpvCSCHost: entries whose |y| is
 * not below FLT_EPSILON (IS_FLOAT_ZERO in the test drivers), in row order.  Returns
 * the count. */
EXPORT int oracle_sparse_output_flt_eps(int m, const double* y, int* key, float* v) {
  int k = 0;
  for (int r = 0; r < m; r++)
    if (!(fabs(y[r]) < FLT_EPSILON)) { key[k] = r; v[k] = (float)y[r]; k++; }
  return k;
}

/* SpmSpvCSCHost, faithful (test_sort_spmspv.cu:330-375): each x value is
 * read into an int (`int col_index, x_val;`, :340), i.e. truncated toward
 * zero; y is a dense FP32 vector accumulated as y[row] += val * x in x order,
 * then column order; alpha is not applied (the routine takes none); the
 * output lists, in row order, the entries that are not IS_FLOAT_ZERO
 * (fabs(y) < FLT_EPSILON; the float overload of abs, as the reference build
 * resolves it).  y_key / y_val need room for m entries.  Returns y_nnz. */
EXPORT int oracle_spmspv_csc_host_faithful(int m, const int* colptr, const int* row,
                                           const float* val, int x_nnz, const int* x_key,
                                           const float* x_val, int* y_key, float* y_val) {
  float* y = (float*)calloc((size_t)(m > 0 ? m : 1), sizeof(float));
  for (int i = 0; i < x_nnz; i++) {
    const int c = x_key[i];
    const int xv = (int)x_val[i];
    for (int j = colptr[c]; j < colptr[c + 1]; j++) y[row[j]] += val[j] * (float)xv;
  }
  int k = 0;
  for (int r = 0; r < m; r++)
    if (!(fabsf(y[r]) < FLT_EPSILON)) { y_key[k] = r; y_val[k] = y[r]; k++; }
  free(y);
  return k;
}

/* Stable CSR -> CSC transpose (rows ascending within each column), the
 * layout the reference's ToCSC produces (cusparse csr2csc, spmspv.h:384-419).
 * colptr[n+1], row[nnz], cval[nnz] (cval may be NULL).  Returns 0, or -1 for
 * a column index out of range. */
EXPORT int oracle_csr2csc(int m, int n, const int* rowptr, const int* col, const float* val,
                          int* colptr, int* row, float* cval) {
  const int nnz = rowptr[m];
  memset(colptr, 0, sizeof(int) * (size_t)(n + 1));
  for (int k = 0; k < nnz; k++) {
    if ((unsigned)col[k] >= (unsigned)n) return -1;
    colptr[col[k] + 1]++;
  }
  for (int c = 0; c < n; c++) colptr[c + 1] += colptr[c];
  int* cur = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  memcpy(cur, colptr, sizeof(int) * (size_t)n);
  for (int r = 0; r < m; r++)
    for (int k = rowptr[r]; k < rowptr[r + 1]; k++) {
      const int p = cur[col[k]]++;
      row[p] = r;
      if (val && cval) cval[p] = val[k];
    }
  free(cur);
  return 0;
}

/* ---- vector format conversions --------------------------------------------- */

/* scatter (spmspv.h:1226-1236) into a zeroed dense vector; sets the bits of
 * the keys like set_sparse_x_bitvector (bitvector.h).  Either output may be
 * NULL. */
EXPORT void oracle_sparse2dense_bits(int n, int x_nnz, const int* key, const float* val,
                                     float* dense, unsigned* bits) {
  if (dense) memset(dense, 0, sizeof(float) * (size_t)n);
  if (bits) memset(bits, 0, sizeof(unsigned) * (size_t)((n + 31) / 32));
  for (int i = 0; i < x_nnz; i++) {
    if (dense) dense[key[i]] = val ? val[i] : 1.0f;
    if (bits) bits[key[i] >> 5] |= 1u << (key[i] & 31);
  }
}

/* updateFlagKernel + scan + streamCompactKeyValKernel (spmspv.h:1122-1175):
 * the entries != 0 in index order.  Returns the count. */
EXPORT int oracle_dense2sparse(int n, const float* dense, int* key, float* val) {
  int k = 0;
  for (int i = 0; i < n; i++)
    if (dense[i] != 0.0f) { key[k] = i; val[k] = dense[i]; k++; }
  return k;
}

/* dense2bitarray with the bit of every NONZERO entry set (the reference's
 * dense2bitarray_ker tests `!val` and so marks the zeros, spmspv.h:1362). */
EXPORT void oracle_dense2bitarray(int n, const float* dense, unsigned* bits) {
  memset(bits, 0, sizeof(unsigned) * (size_t)((n + 31) / 32));
  for (int i = 0; i < n; i++)
    if (dense[i] != 0.0f) bits[i >> 5] |= 1u << (i & 31);
}

/* ---- features ------------------------------------------------------------------- */

/* computeMatFeture_serial (spmspv.h:2275-2335) with exact (FP64 / int64)
 * accumulation.  out = {m, n, nnz, max, min, avg, range, stdRow,
 * edge_equlity, gini}.  avg keeps the reference's float division
 * mat_nnz/(float)m. */
EXPORT void oracle_mat_features(int m, int n, int nnz, const int* rowptr, double* out) {
  int mx = 0, mn = INT_MAX;
  const double avg = m ? (double)((float)nnz / (float)m) : 0.0;
  double sq = 0, ent = 0;
  int64_t* hist = NULL;
  for (int i = 0; i < m; i++) {
    const int d = rowptr[i + 1] - rowptr[i];
    sq += (d - avg) * (d - avg);
    if (d != 0) ent += -((double)d / nnz) * log((double)d / nnz);
    if (d > mx) mx = d;
    if (d < mn) mn = d;
  }
  /* Gini over sorted degrees: S1 = sum_{j>=1} j*d_(j), S2 = sum_{i<m-1} d_(i)
   * (spmspv.h:2314-2320), via a counting sort */
  double gini = 0;
  if (m > 0) {
    hist = (int64_t*)calloc((size_t)mx + 1, sizeof(int64_t));
    for (int i = 0; i < m; i++) hist[rowptr[i + 1] - rowptr[i]]++;
    int64_t pos = 0;
    unsigned long long s1 = 0;
    for (int v = 0; v <= mx; v++) {
      const int64_t h = hist[v];
      if (h) s1 += (unsigned long long)v * (unsigned long long)(h * pos + h * (h - 1) / 2);
      pos += h;
    }
    free(hist);
    const double S2 = (double)nnz - (double)mx;
    gini = (2.0 * (double)s1) / ((double)m * S2) - (double)(m + 1) / (double)m;
    if (gini < 0) gini = -gini;
    if (!isfinite(gini)) gini = 0;
  }
  out[0] = m; out[1] = n; out[2] = nnz; out[3] = mx; out[4] = mn; out[5] = avg;
  out[6] = n ? (double)(mx - mn) / (double)n : 0.0;
  out[7] = m ? sqrt(sq / m) : 0.0;
  out[8] = m > 1 ? ent / log((double)m) : 0.0;
  out[9] = gini;
}

/* computeMatFeture_serial, faithful: float accumulators exactly as written
 * (float sum, float sum_gini_1/2, std::sort of degrees).  Kept to document
 * how far the reference's float sums drift from the exact values. */
static int cmp_int(const void* a, const void* b) {
  const int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}
EXPORT void oracle_mat_features_faithful(int m, int n, int nnz, const int* rowptr,
                                         float* out) {
  int max = 0, min = INT_MAX;
  float sum = 0.0f, sum_gini_1 = 0.0f, sum_gini_2 = 0.0f;
  double sum_edge = 0.0;
  const double avg = nnz / (float)m;
  int* deg = (int*)malloc(sizeof(int) * (size_t)m);
  for (int i = 0; i < m; i++) {
    const int num = rowptr[i + 1] - rowptr[i];
    deg[i] = num;
    sum += (num - avg) * (num - avg);
    if (num != 0) sum_edge += -(num / (1.0 * nnz)) * log(num / (1.0 * nnz));
    if (num > max) max = num;
    if (num < min) min = num;
  }
  const float stdv = sqrtf(sum / m);
  const float edge = (float)sum_edge * (1.0 / log(m * 1.0));
  qsort(deg, (size_t)m, sizeof(int), cmp_int);
  int j = 1;
  for (int i = 0; i + 1 < m; i++) {
    sum_gini_1 += 1.0 * j * deg[i + 1];
    sum_gini_2 += 1.0 * deg[i];
    j++;
  }
  float gini = (2.0 * sum_gini_1) / (m * sum_gini_2) - (m + 1) / (float)m;
  if (gini < 0) gini *= -1;
  free(deg);
  out[0] = (float)max; out[1] = (float)min; out[2] = (float)avg;
  out[3] = (float)((max - min) / (1.0 * n)); out[4] = stdv; out[5] = edge; out[6] = gini;
}

/* extractMatFeature (spmspv.h:423-447): stdRow with the mean truncated to
 * int, accumulated in FP64 here. */
EXPORT double oracle_std_row_intmean(int m, int nnz, const int* rowptr) {
  const int avg = (int)(nnz / (float)m);
  double s = 0;
  for (int i = 0; i < m; i++) {
    const int d = rowptr[i + 1] - rowptr[i];
    s += (double)(d - avg) * (double)(d - avg);
  }
  return sqrt(s / m);
}

/* extractMatFeature, faithful: int-truncated mean, int differences squared
 * and added into a float, float square root (spmspv.h:423-447). */
EXPORT float oracle_std_row_intmean_faithful(int m, int nnz, const int* rowptr) {
  const int avg_nnz = (int)(nnz / (float)m);
  float sum = 0.0f;
  for (int i = 0; i < m; i++) {
    const int num = rowptr[i + 1] - rowptr[i];
    sum += (num - avg_nnz) * (num - avg_nnz);
  }
  return sqrtf(sum / m);
}

/* computeVecFeture_serial (spmspv.h:2338-2361): out = {bin_len, max, min} */
EXPORT void oracle_vec_features(const int* colptr, int x_nnz, const int* x_key,
                                long long* out) {
  long long sum = 0;
  int mx = 0, mn = INT_MAX;
  for (int i = 0; i < x_nnz; i++) {
    const int c = x_key[i];
    const int num = colptr[c + 1] - colptr[c];
    sum += num;
    if (num > mx) mx = num;
    if (num < mn) mn = num;
  }
  out[0] = sum; out[1] = mx; out[2] = mn;
}

/* computeGM1/2/3 (spmspv.h:2727-2752) with 4-byte indices and values */
EXPORT void oracle_gm(int m, int nnz, int x_nnz, long long bin_len, double* gm) {
  const double x = x_nnz, b = (double)bin_len;
  gm[0] = x * 4 + b * 4 + b * 4 + x * 4 + x * 4 + b * 4;
  gm[1] = ((double)m + 1) * 4 + b * 4 + (double)nnz * 4 + b * 4 + (double)m * 4;
  gm[2] = ((double)m + 1) * 4 + (double)nnz * 4 * 3 + (double)m * 4;
}

/* setSigma auto rule (spmspv.h:1396-1416) */
EXPORT int oracle_csr5_sigma(int m, int nnz) {
  const int r = 4, s = 32, t = 256, u = 6;
  const int nnz_per_row = nnz / m;
  if (nnz_per_row <= r) return r;
  if (nnz_per_row <= s) return nnz_per_row;
  if (nnz_per_row <= t) return s;
  return u;
}

/* ---- BFS ------------------------------------------------------------------------ */

/* Level-synchronous BFS as repeated Boolean SpMSpV y = A^T f masked by the
 * visited set, written in the loop structure of SpmSpvCSCHost (a CSC pass
 * over the frontier's columns).  levels[n] = hop count, -1 if unreachable.
 * Returns the number of levels. */
EXPORT int oracle_bfs_spmspv(int n, const int* colptr, const int* row, int src, int* levels) {
  int* qbuf = (int*)malloc(sizeof(int) * 2 * (size_t)(n > 0 ? n : 1));
  int* front = qbuf;
  int* next = qbuf + (n > 0 ? n : 1);
  unsigned char* y = (unsigned char*)calloc((size_t)(n > 0 ? n : 1), 1);
  for (int i = 0; i < n; i++) levels[i] = -1;
  levels[src] = 0;
  int nf = 1, level = 0;
  front[0] = src;
  while (nf > 0) {
    /* y = OR over frontier columns (Boolean SpMSpV) */
    for (int i = 0; i < nf; i++) {
      const int c = front[i];
      for (int j = colptr[c]; j < colptr[c + 1]; j++) y[row[j]] = 1;
    }
    /* mask by visited, emit the next frontier in row order */
    int nn = 0;
    for (int r = 0; r < n; r++) {
      if (y[r] && levels[r] < 0) { levels[r] = level + 1; next[nn++] = r; }
      y[r] = 0;
    }
    int* t = front; front = next; next = t;
    nf = nn;
    if (nf > 0) level++;
  }
  free(qbuf); free(y);
  return level + 1;
}

/* Plain FIFO-queue BFS, the cross-check of the SpMSpV formulation. */
EXPORT int oracle_bfs_queue(int n, const int* rowptr, const int* col, int src, int* levels) {
  int* q = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) levels[i] = -1;
  int head = 0, tail = 0, depth = 0;
  levels[src] = 0;
  q[tail++] = src;
  while (head < tail) {
    const int u = q[head++];
    if (levels[u] + 1 > depth) depth = levels[u] + 1;
    for (int j = rowptr[u]; j < rowptr[u + 1]; j++) {
      const int v = col[j];
      if (levels[v] < 0) { levels[v] = levels[u] + 1; q[tail++] = v; }
    }
  }
  free(q);
  return depth;
}

/* ---- adjoint of y = A x ------------------------------------------------------ */

/* dx = A^T dy (dense dy) in FP64, with per-entry magnitudes */
EXPORT void oracle_spmv_t_f64(int m, int n, const int* rowptr, const int* col,
                              const float* val, const float* dy, double* dx, double* absdx) {
  memset(dx, 0, sizeof(double) * (size_t)n);
  if (absdx) memset(absdx, 0, sizeof(double) * (size_t)n);
  for (int i = 0; i < m; i++)
    for (int j = rowptr[i]; j < rowptr[i + 1]; j++) {
      const double p = (double)val[j] * (double)dy[i];
      dx[col[j]] += p;
      if (absdx) absdx[col[j]] += fabs(p);
    }
}

/* dvals[k] = dy[row_k] * x[col_k] in FP64 */
EXPORT void oracle_dvals_f64(int m, const int* rowptr, const int* col, const float* dy,
                             const float* x, double* dvals) {
  for (int i = 0; i < m; i++)
    for (int j = rowptr[i]; j < rowptr[i + 1]; j++)
      dvals[j] = (double)dy[i] * (double)x[col[j]];
}

/* ---- timed CPU baselines ------------------------------------------------------ */

/* serialspmv (FP32, one core) over the whole matrix */
EXPORT void cpu_spmv_serial(int m, const int* rowptr, const int* col, const float* val,
                            const float* x, float* y, float alpha) {
  oracle_serialspmv_f32(m, rowptr, col, val, x, y, alpha);
}

/* the same loop split over rows with OpenMP (all host threads) */
EXPORT void cpu_spmv_omp(int m, const int* rowptr, const int* col, const float* val,
                         const float* x, float* y, float alpha) {
#pragma omp parallel for schedule(dynamic, 2048)
  for (int i = 0; i < m; i++) {
    float sum = 0;
    for (int j = rowptr[i]; j < rowptr[i + 1]; j++) sum += x[col[j]] * val[j] * alpha;
    y[i] = sum;
  }
}

/* SpmSpvCSCHost with FP32 accumulation into a dense y (one core) */
EXPORT void cpu_spmspv_csc_serial(int m, const int* colptr, const int* row, const float* val,
                                  int x_nnz, const int* x_key, const float* x_val, float* y) {
  memset(y, 0, sizeof(float) * (size_t)m);
  for (int i = 0; i < x_nnz; i++) {
    const int c = x_key[i];
    const float xv = x_val[i];
    for (int j = colptr[c]; j < colptr[c + 1]; j++) y[row[j]] += val[j] * xv;
  }
}

/* CSC SpMSpV on all host threads: x entries split across threads, each with
 * atomic float adds into y */
EXPORT void cpu_spmspv_csc_omp(int m, const int* colptr, const int* row, const float* val,
                               int x_nnz, const int* x_key, const float* x_val, float* y) {
  memset(y, 0, sizeof(float) * (size_t)m);
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < x_nnz; i++) {
    const int c = x_key[i];
    const float xv = x_val[i];
    for (int j = colptr[c]; j < colptr[c + 1]; j++) {
#pragma omp atomic
      y[row[j]] += val[j] * xv;
    }
  }
}

EXPORT int cpu_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ---- matrix files --------------------------------------------------------
 * ReadMTX (include/spmspv/mtx.hpp:218-361) restated: the banner is read as
 * whitespace tokens, the 4th naming the field and the 5th the symmetry
 * (only "symmetric" expands; any field other than real / pattern / integer
 * reads as complex and stores 1); comment lines are skipped up to the size
 * line; entries are read with fscanf, "real" through double; each
 * off-diagonal entry of a symmetric file is followed by its mirror; then the
 * entries are sorted by (row, col).
 * Departure: the reference's std::sort is not stable, the oracle's sort is
 * (counting sort by column, then by row), so entries with equal (row, col)
 * keep file order here; only their order can differ from the reference.
 * Returns 0, or < 0 for an unreadable file.  Arrays are malloc'ed
 * (oracle_free). */
static void counting_sort_by(int keys_n, int nnz, const int* key, const int* a, const int* b,
                             const float* v, int* ka, int* kb, float* kv, int* out_key) {
  int* cnt = (int*)calloc((size_t)keys_n + 1, sizeof(int));
  for (int i = 0; i < nnz; i++) cnt[key[i] + 1]++;
  for (int k = 0; k < keys_n; k++) cnt[k + 1] += cnt[k];
  for (int i = 0; i < nnz; i++) {
    const int o = cnt[key[i]]++;
    ka[o] = a[i];
    kb[o] = b[i];
    kv[o] = v[i];
    out_key[o] = key[i];
  }
  free(cnt);
}

EXPORT void oracle_free(void* p) { free(p); }

EXPORT int oracle_mtx_read(const char* path, int* m_out, int* n_out, int* nnz_out, int** row_out,
                           int** col_out, float** val_out) {
  FILE* f = fopen(path, "r");
  if (!f) return -1;
  char tok[128], line[1030];
  for (int t = 0; t < 4; t++)
    if (fscanf(f, "%127s", tok) != 1) { fclose(f); return -2; }
  const int is_real = strcmp(tok, "real") == 0;
  const int is_pattern = strcmp(tok, "pattern") == 0;
  const int is_int = strcmp(tok, "integer") == 0;
  const int is_complex = !is_real && !is_pattern && !is_int;
  if (fscanf(f, "%127s", tok) != 1) { fclose(f); return -2; }
  const int sym = strcmp(tok, "symmetric") == 0;
  int height = 0, width = 0, L = 0;
  for (;;) {
    if (fscanf(f, "%127s", tok) != 1) { fclose(f); return -3; }
    if (tok[0] != '%') { height = atoi(tok); break; }
    /* rest of the comment line */
    while (fgets(line, sizeof line, f) && !strchr(line, '\n')) {}
  }
  if (fscanf(f, "%d %d", &width, &L) != 2 || L < 0) { fclose(f); return -3; }
  int* r = (int*)malloc(sizeof(int) * (size_t)(L > 0 ? L : 1));
  int* c = (int*)malloc(sizeof(int) * (size_t)(L > 0 ? L : 1));
  float* v = (float*)malloc(sizeof(float) * (size_t)(L > 0 ? L : 1));
  int diag = 0;
  for (int i = 0; i < L; i++) {
    int ri = 0, ci = 0;
    if (fscanf(f, "%d %d", &ri, &ci) != 2) { free(r); free(c); free(v); fclose(f); return -4; }
    r[i] = ri - 1;
    c[i] = ci - 1;
    v[i] = 1.0f;
    if (is_real) {
      double d = 0.0;
      if (fscanf(f, "%lf", &d) != 1) { free(r); free(c); free(v); fclose(f); return -4; }
      v[i] = (float)d;
    } else if (is_int) {
      int d = 0;
      if (fscanf(f, "%d", &d) != 1) { free(r); free(c); free(v); fclose(f); return -4; }
      v[i] = (float)d;
    } else if (is_complex) {
      double a = 0.0, b = 0.0;
      if (fscanf(f, "%lf %lf", &a, &b) != 2) { free(r); free(c); free(v); fclose(f); return -4; }
    }
    if (r[i] == c[i]) diag++;
    if (r[i] < 0 || r[i] >= height || c[i] < 0 || c[i] >= width) {
      free(r); free(c); free(v); fclose(f); return -5;
    }
  }
  fclose(f);
  int nnz = L;
  if (sym) {
    nnz = 2 * L - diag;
    int* r2 = (int*)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    int* c2 = (int*)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    float* v2 = (float*)malloc(sizeof(float) * (size_t)(nnz > 0 ? nnz : 1));
    int o = 0;
    for (int i = 0; i < L; i++) {
      r2[o] = r[i]; c2[o] = c[i]; v2[o] = v[i]; o++;
      if (r[i] != c[i]) { r2[o] = c[i]; c2[o] = r[i]; v2[o] = v[i]; o++; }
    }
    free(r); free(c); free(v);
    r = r2; c = c2; v = v2;
  }
  /* stable sort by (row, col): by column, then by row */
  const size_t sz = (size_t)(nnz > 0 ? nnz : 1);
  int* r1 = (int*)malloc(sizeof(int) * sz);
  int* c1 = (int*)malloc(sizeof(int) * sz);
  float* v1 = (float*)malloc(sizeof(float) * sz);
  int* kk = (int*)malloc(sizeof(int) * sz);
  counting_sort_by(width, nnz, c, r, c, v, r1, c1, v1, kk);
  counting_sort_by(height, nnz, r1, c1, r1, v1, c, r, v, kk);
  /* after the second pass: c holds columns, r holds rows (key copy in kk) */
  free(r1); free(c1); free(v1); free(kk);
  *m_out = height;
  *n_out = width;
  *nnz_out = nnz;
  *row_out = r;
  *col_out = c;
  *val_out = v;
  return 0;
}

/* COO2Hybrid with row priority (include/spmspv/mtx.hpp:436-701, the branch
 * test/test_coo2hybrid.cu:276 uses), restated over a CSR: nonzeros visited in
 * (row, column) order with running row and column counts; to_csr[k] = 1 when
 * count_row[r] >= count_col[c] (then count_col[c]--), else 0 (count_row[r]--).
 * Returns the number of CSR-part nonzeros.  The reference sizes its count
 * arrays by nnz; here they are sized by m and n. */
EXPORT int oracle_coo2hybrid(int m, int n, const int* rowptr, const int* col, unsigned char* to_csr) {
  int* cr = (int*)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
  int* cc = (int*)calloc((size_t)(n > 0 ? n : 1), sizeof(int));
  for (int r = 0; r < m; r++) cr[r] = rowptr[r + 1] - rowptr[r];
  for (int k = 0; k < rowptr[m]; k++) cc[col[k]]++;
  int csr = 0;
  for (int r = 0; r < m; r++)
    for (int k = rowptr[r]; k < rowptr[r + 1]; k++) {
      const int c = col[k];
      if (cr[r] >= cc[c]) {
        to_csr[k] = 1;
        csr++;
        cc[c]--;
      } else {
        to_csr[k] = 0;
        cr[r]--;
      }
    }
  free(cr);
  free(cc);
  return csr;
}

/* ---- synthetic inputs of the benchmark --------------------------------------
 * A second, independent statement of the benchmark's input generators, so
 * that the CPU reference arm of the benchmark builds its inputs without the
 * product library.  The scheme (stated here in full; the product's
 * generators follow the same one and a CPU test checks the outputs equal):
 *   rng(seed, stream, ctr) = mix(mix(seed*0x632be59bd9b4e019 + stream) ^
 *                                (ctr*0xd1b54a32d192ed03)), mix = splitmix64's
 *   finaliser; u01 = (rng >> 11) / 2^53; normal = Box-Muller on two u01.
 *   Streams: 2 Zipf length, 3 Zipf rounding, 4 Zipf total fix, 5 Zipf
 *   column, 6 Zipf value, 10 vector position, 11 vector value. */
static uint64_t gen_mix(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
static uint64_t gen_rng(uint64_t seed, uint64_t stream, uint64_t ctr) {
  return gen_mix(gen_mix(seed * 0x632be59bd9b4e019ULL + stream) ^ (ctr * 0xd1b54a32d192ed03ULL));
}
static double gen_u01(uint64_t seed, uint64_t stream, uint64_t ctr) {
  return (double)(gen_rng(seed, stream, ctr) >> 11) * (1.0 / 9007199254740992.0);
}
static double gen_normal(uint64_t seed, uint64_t stream, uint64_t ctr) {
  double u1 = gen_u01(seed, stream, 2 * ctr), u2 = gen_u01(seed, stream, 2 * ctr + 1);
  if (u1 < 1e-300) u1 = 1e-300;
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}
static int gen_cmp_int(const void* a, const void* b) {
  const int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}
static int gen_unique(int* c, int len) {
  int w = 0;
  for (int k = 0; k < len; k++)
    if (w == 0 || c[k] != c[w - 1]) c[w++] = c[k];
  return w;
}

/* m x m matrix whose row lengths are Zipf(s) on [1, maxlen], scaled by
 * mean / E[L] with stochastic rounding and clamped to [0, maxlen], the total
 * then fixed to exactly mean * m by +-1 on random rows; per row distinct
 * uniform columns (draw, sort, deduplicate, redraw the shortfall) and values
 * U(-1, 1).  rowptr[m+1], col / val [mean*m] are the caller's.  Returns 0, or
 * -1 for arguments out of range. */
EXPORT int oracle_gen_zipf_rows(int m, double s, int mean, int maxlen, uint64_t seed, int* rowptr,
                                int* col, float* val) {
  if (m < 1 || mean < 0 || maxlen < 1 || maxlen > m) return -1;
  const long long target = (long long)mean * m;
  if (target > 2147483647LL || target > (long long)maxlen * m) return -1;
  double* cdf = (double*)malloc(sizeof(double) * (size_t)maxlen);
  double z = 0, ez = 0;
  for (int k = 1; k <= maxlen; k++) {
    const double p = pow((double)k, -s);
    z += p;
    ez += k * p;
    cdf[k - 1] = z;
  }
  for (int k = 0; k < maxlen; k++) cdf[k] /= z;
  ez /= z;
  const double f = ez > 0 ? (double)mean / ez : 0.0;
  int* len = (int*)malloc(sizeof(int) * (size_t)m);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < m; i++) {
    const double r = gen_u01(seed, 2, (uint64_t)i);
    int lo = 0, hi = maxlen; /* first index with cdf >= r */
    while (lo < hi) {
      const int mid = lo + (hi - lo) / 2;
      if (cdf[mid] < r) lo = mid + 1; else hi = mid;
    }
    const double scaled = (lo + 1) * f;
    int L = (int)floor(scaled);
    if (gen_u01(seed, 3, (uint64_t)i) < scaled - L) ++L;
    len[i] = L < 0 ? 0 : (L > maxlen ? maxlen : L);
  }
  long long tot = 0;
  for (int i = 0; i < m; i++) tot += len[i];
  uint64_t ctr = 0;
  while (tot != target) {
    const int i = (int)(gen_rng(seed, 4, ctr++) % (uint64_t)m);
    if (tot < target && len[i] < maxlen) { ++len[i]; ++tot; }
    else if (tot > target && len[i] > 0) { --len[i]; --tot; }
  }
  rowptr[0] = 0;
  for (int i = 0; i < m; i++) rowptr[i + 1] = rowptr[i] + len[i];
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < m; i++) {
    const int L = len[i];
    int* c = col + rowptr[i];
    int have = 0;
    uint64_t t = 0;
    while (have < L) {
      for (int k = have; k < L; k++)
        c[k] = (int)(gen_rng(seed, 5, ((uint64_t)i << 24) + t++) % (uint64_t)m);
      qsort(c, (size_t)L, sizeof(int), gen_cmp_int);
      have = gen_unique(c, L);
    }
    for (int k = 0; k < L; k++)
      val[rowptr[i] + k] = (float)(2.0 * gen_u01(seed, 6, (uint64_t)rowptr[i] + k) - 1.0);
  }
  free(len);
  free(cdf);
  return 0;
}

/* k distinct positions in [0, n), sorted, with U(-1,1) (dist 0) or N(0,1)
 * values: a partial Fisher-Yates over [0, n) when 3k >= n, else draws in
 * order keeping first occurrences.  Returns 0, or -1 for k outside [0, n]. */
EXPORT int oracle_gen_sparse_vector(int n, int k, int dist, uint64_t seed, int* key, float* val) {
  if (n < 0 || k < 0 || k > n) return -1;
  if (k == 0) return 0;
  if ((long long)k * 3 >= n) {
    int* p = (int*)malloc(sizeof(int) * (size_t)n);
    for (int i = 0; i < n; i++) p[i] = i;
    for (int i = 0; i < k; i++) {
      const int j = i + (int)(gen_rng(seed, 10, (uint64_t)i) % (uint64_t)(n - i));
      const int t = p[i];
      p[i] = p[j];
      p[j] = t;
    }
    memcpy(key, p, sizeof(int) * (size_t)k);
    free(p);
  } else {
    unsigned char* seen = (unsigned char*)calloc((size_t)n / 8 + 1, 1);
    uint64_t t = 0;
    int have = 0;
    while (have < k) {
      const int c = (int)(gen_rng(seed, 10, t++) % (uint64_t)n);
      if (!(seen[c >> 3] & (1u << (c & 7)))) {
        seen[c >> 3] |= (unsigned char)(1u << (c & 7));
        key[have++] = c;
      }
    }
    free(seen);
  }
  qsort(key, (size_t)k, sizeof(int), gen_cmp_int);
  for (int i = 0; i < k; i++)
    val[i] = dist == 0 ? (float)(2.0 * gen_u01(seed, 11, (uint64_t)i) - 1.0)
                       : (float)gen_normal(seed, 11, (uint64_t)i);
  return 0;
}
