// C ABI of the engine, part 2: feature extraction, the kernel selector, the
// adaptive iteration and the BFS driver.
//
// The reference's run-time selector is three stubs returning 0
// (TEST/new_test_app.cu:121-131) and its dispatch tree is compiled out
// (:404-465); the trees are trained offline (model/[123]-test_dtree.py).  The
// selector here evaluates a tree over the reference's feature schema using
// only features known on the host without a device round trip: matrix
// features (computed once per matrix) and x_nnz, with bin_len estimated as
// x_nnz * nnz / n unless it has been measured.
#include <algorithm>
#include <cmath>
#include <climits>
#include <cstring>
#include <string>

#include "bfs.h"
#include "engine.h"
#include "feat.h"
#include "kernels.h"
#include "selector.h"
#include "sort.h"

using namespace spmx;


// ---------------------------------------------------------------------------
// matrix features
// ---------------------------------------------------------------------------
static int compute_mat_features(spmx_handle_t h) {
  if (h->mat_feat_ready) return SPMX_SUCCESS;
  if (!h->has_csr) return set_error(SPMX_ERR_NOT_READY, "matrix features need the CSR input");
  cudaStream_t st = h->stream;
  const int m = h->m, n = h->n, nnz = h->nnz;
  // computeMatFeture_serial divides in float: mat_nnz/(float)m (H:2292)
  const double avg = m ? (double)((float)nnz / (float)m) : 0.0;
  // extractMatFeature(Parallel) truncates the mean to int (H:429, H:929)
  const double avg_int = m ? (double)(int)((float)nnz / (float)m) : 0.0;
  SPMX_CUDA(cudaMemsetAsync(h->d_facc, 0, sizeof(double) * 4, st));
  SPMX_CUDA(cudaMemsetAsync(h->d_iacc, 0, sizeof(int) * 4, st));
  SPMX_CUDA(cudaMemsetAsync(h->d_u64, 0, sizeof(unsigned long long) * 4, st));
  launch_mat_features(m, h->rowptr, nnz, avg, avg_int, h->d_facc, h->d_iacc, st);
  double facc[4];
  int iacc[4];
  SPMX_CUDA(cudaMemcpyAsync(facc, h->d_facc, sizeof(facc), cudaMemcpyDeviceToHost, st));
  SPMX_CUDA(cudaMemcpyAsync(iacc, h->d_iacc, sizeof(iacc), cudaMemcpyDeviceToHost, st));
  SPMX_CUDA(cudaStreamSynchronize(st));
  SPMX_TRY(launch_ok("matrix features"));
  const int maxd = m ? iacc[0] : 0;
  const int mind = m ? INT_MAX - iacc[1] : INT_MAX;
  // Gini from the row-length histogram: S1 = sum_j j*d_(j) over sorted
  // lengths; S2 = sum of all lengths but the largest (H:2314-2320)
  double gini = 0.0;
  if (m > 0) {
    int *hist = nullptr, *pref = nullptr;
    SPMX_TRY(dalloc((void**)&hist, 4 * (size_t)(maxd + 1), "degree hist"));
    SPMX_TRY(dalloc((void**)&pref, 4 * (size_t)(maxd + 1), "degree prefix"));
    cudaMemsetAsync(hist, 0, 4 * (size_t)(maxd + 1), st);
    launch_degree_hist(m, h->rowptr, hist, st);
    int rc = launch_scan_exclusive(hist, pref, maxd + 1, nullptr, h->ls, h->d_err, st);
    if (rc) {
      dfree(hist); dfree(pref);
      return set_error(SPMX_ERR_INVALID_VALUE, "degree histogram exceeds the scan capacity");
    }
    launch_gini_sum(maxd, hist, pref, h->d_u64, st);
    unsigned long long s1 = 0;
    cudaMemcpyAsync(&s1, h->d_u64, sizeof(s1), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    dfree(hist); dfree(pref);
    if (e != cudaSuccess) return set_error(SPMX_ERR_CUDA, cudaGetErrorString(e));
    const double S1 = (double)s1;
    const double S2 = (double)nnz - (double)maxd;
    gini = (2.0 * S1) / ((double)m * S2) - (double)(m + 1) / (double)m;
    if (gini < 0) gini = -gini;
    if (!std::isfinite(gini)) gini = 0.0;
  }
  double* f = h->mat_feat;
  f[0] = m;
  f[1] = n;
  f[2] = nnz;
  f[3] = maxd;
  f[4] = mind;
  f[5] = avg;
  f[6] = n ? (double)(maxd - mind) / (double)n : 0.0;
  f[7] = m ? std::sqrt(facc[0] / m) : 0.0;
  f[8] = (m > 1) ? facc[2] / std::log((double)m) : 0.0;
  f[9] = gini;
  h->std_row = m ? (float)std::sqrt(facc[1] / m) : 0.f;
  h->std_row_ready = true;
  h->mat_feat_ready = true;
  return SPMX_SUCCESS;
}

extern "C" int spmx_mat_features(spmx_handle_t h, double out[10]) {
  SPMX_CHECK_HANDLE(h);
  if (!out) return set_error(SPMX_ERR_INVALID_VALUE, "out is NULL");
  SPMX_TRY(compute_mat_features(h));
  std::memcpy(out, h->mat_feat, sizeof(double) * 10);
  return SPMX_SUCCESS;
}

extern "C" int spmx_std_row(spmx_handle_t h, float* std_row) {
  SPMX_CHECK_HANDLE(h);
  if (!std_row) return set_error(SPMX_ERR_INVALID_VALUE, "out is NULL");
  SPMX_TRY(compute_mat_features(h));
  *std_row = h->std_row;
  return SPMX_SUCCESS;
}

// ---------------------------------------------------------------------------
// vector features
// ---------------------------------------------------------------------------
extern "C" int spmx_vec_features(spmx_handle_t h, long long out[3]) {
  SPMX_CHECK_HANDLE(h);
  if (!out) return set_error(SPMX_ERR_INVALID_VALUE, "out is NULL");
  if (!h->has_csc) return set_error(SPMX_ERR_NOT_READY, "vector features need the CSC");
  cudaStream_t st = h->stream;
  SPMX_CUDA(cudaMemsetAsync(h->d_u64, 0, sizeof(unsigned long long) * 4, st));
  SPMX_CUDA(cudaMemsetAsync(h->d_iacc, 0, sizeof(int) * 4, st));
  launch_vec_features(h->x_nnz, h->n, h->x_key, h->csc_colptr, h->d_u64, h->d_iacc, h->d_err, st);
  unsigned long long s = 0;
  int iacc[4];
  SPMX_CUDA(cudaMemcpyAsync(&s, h->d_u64, sizeof(s), cudaMemcpyDeviceToHost, st));
  SPMX_CUDA(cudaMemcpyAsync(iacc, h->d_iacc, sizeof(iacc), cudaMemcpyDeviceToHost, st));
  SPMX_CUDA(cudaStreamSynchronize(st));
  SPMX_TRY(launch_ok("vector features"));
  h->bin_len = (long long)s;
  h->vec_max = h->x_nnz ? iacc[0] : 0;
  h->vec_min = h->x_nnz ? (long long)(INT_MAX - iacc[1]) : (long long)INT_MAX;
  out[0] = h->bin_len;
  out[1] = h->vec_max;
  out[2] = h->vec_min;
  return SPMX_SUCCESS;
}

extern "C" int spmx_compute_binlen(spmx_handle_t h, long long* bin_len) {
  long long v[3];
  SPMX_TRY(spmx_vec_features(h, v));
  if (bin_len) *bin_len = v[0];
  return SPMX_SUCCESS;
}

static void gm_models(spmx_handle_t h, double bin_len, double gm[3]) {
  // computeGM1/2/3 (H:2727-2752): bytes of the CSC SpMSpV, the CSR SpMSpV and
  // the SpMV under 4-byte indices and values
  const double x = h->x_nnz, m = h->m, nnz = h->nnz;
  gm[0] = x * 4 + bin_len * 4 + bin_len * 4 + x * 4 + x * 4 + bin_len * 4;
  gm[1] = (m + 1) * 4 + bin_len * 4 + nnz * 4 + bin_len * 4 + m * 4;
  gm[2] = (m + 1) * 4 + nnz * 4 + nnz * 4 + nnz * 4 + m * 4;
}

extern "C" int spmx_compute_gm(spmx_handle_t h, double gm[3]) {
  SPMX_CHECK_HANDLE(h);
  if (!gm) return set_error(SPMX_ERR_INVALID_VALUE, "gm is NULL");
  if (h->bin_len < 0) {
    long long b;
    SPMX_TRY(spmx_compute_binlen(h, &b));
  }
  gm_models(h, (double)h->bin_len, h->gm);
  std::memcpy(gm, h->gm, sizeof(h->gm));
  return SPMX_SUCCESS;
}

static void fill_features(spmx_handle_t h, double bin_len, long long vmax, long long vmin,
                          double out[SPMX_NUM_FEATURES]) {
  std::memcpy(out, h->mat_feat, sizeof(double) * 10);
  const double n = h->n ? h->n : 1, nnz = h->nnz ? h->nnz : 1;
  double gm[3];
  gm_models(h, bin_len, gm);
  out[10] = h->x_nnz;
  out[11] = bin_len;
  out[12] = (double)vmax;
  out[13] = (double)vmin;
  out[14] = h->x_nnz / n;
  out[15] = bin_len / nnz;
  out[16] = (double)(vmax - vmin) / n;
  out[17] = gm[0];
  out[18] = gm[1];
  out[19] = gm[2];
  out[20] = gm[1] ? gm[0] / gm[1] : 0;
  out[21] = gm[2] ? gm[1] / gm[2] : 0;
  out[22] = gm[2] ? gm[0] / gm[2] : 0;
}

extern "C" int spmx_features(spmx_handle_t h, double out[SPMX_NUM_FEATURES]) {
  SPMX_CHECK_HANDLE(h);
  if (!out) return set_error(SPMX_ERR_INVALID_VALUE, "out is NULL");
  SPMX_TRY(compute_mat_features(h));
  long long v[3];
  SPMX_TRY(spmx_vec_features(h, v));
  fill_features(h, (double)v[0], v[1], v[2], out);
  return SPMX_SUCCESS;
}

// ---------------------------------------------------------------------------
// selector and the adaptive iteration
// ---------------------------------------------------------------------------
// longest column of the CSC (once per matrix): an upper bound of the longest
// column any x selects
static int compute_col_max(spmx_handle_t h) {
  if (h->col_max >= 0) return SPMX_SUCCESS;
  if (!h->has_csc) { h->col_max = 0; return SPMX_SUCCESS; }
  cudaStream_t st = h->stream;
  SPMX_CUDA(cudaMemsetAsync(h->d_facc, 0, sizeof(double) * 4, st));
  SPMX_CUDA(cudaMemsetAsync(h->d_iacc, 0, sizeof(int) * 4, st));
  launch_mat_features(h->n, h->csc_colptr, h->nnz, 0.0, 0.0, h->d_facc, h->d_iacc, st);
  int iacc[4];
  SPMX_CUDA(cudaMemcpyAsync(iacc, h->d_iacc, sizeof(iacc), cudaMemcpyDeviceToHost, st));
  SPMX_CUDA(cudaStreamSynchronize(st));
  h->col_max = h->n ? iacc[0] : 0;
  return launch_ok("column features");
}

extern "C" int spmx_selector_inputs(spmx_handle_t h, double out[SPMX_NUM_FEATURES]) {
  SPMX_CHECK_HANDLE(h);
  if (!out) return set_error(SPMX_ERR_INVALID_VALUE, "out is NULL");
  SPMX_TRY(compute_mat_features(h));
  SPMX_TRY(compute_col_max(h));
  const double est = h->bin_len >= 0 ? (double)h->bin_len
                                      : (h->n ? (double)h->x_nnz * h->nnz / h->n : 0.0);
  // x's own longest / shortest column need a device pass; the matrix's
  // longest column bounds the former, the latter is not used
  fill_features(h, est, h->col_max, 0, out);
  return SPMX_SUCCESS;
}

extern "C" int spmx_select(spmx_handle_t h, int* kernel_id) {
  SPMX_CHECK_HANDLE(h);
  if (!kernel_id) return set_error(SPMX_ERR_INVALID_VALUE, "kernel_id is NULL");
  double f[SPMX_NUM_FEATURES];
  SPMX_TRY(spmx_selector_inputs(h, f));
  *kernel_id = spmx_select_kernel(f);
  return SPMX_SUCCESS;
}

extern "C" int spmx_select_features(const double* f, int* kernel_id) {
  if (!f || !kernel_id) return set_error(SPMX_ERR_INVALID_VALUE, "NULL argument");
  *kernel_id = spmx_select_kernel(f);
  return SPMX_SUCCESS;
}

extern "C" int spmx_csc_bucket(spmx_handle_t h, float alpha, int* ynnz, float* y, int* ykey,
                               float* yval, int buckets);

extern "C" int spmx_run_kernel(spmx_handle_t h, int kid, float alpha, float* y) {
  SPMX_CHECK_HANDLE(h);
  switch (kid) {
    case SPMX_K_CSC_NAIVE_SORT:
      return spmx_spmspv_csc(h, SPMX_CSC_NAIVE, SPMX_WB_SORT, alpha, y, nullptr, nullptr, nullptr);
    case SPMX_K_CSC_NAIVE_ATOMIC:
      return spmx_spmspv_csc(h, SPMX_CSC_NAIVE, SPMX_WB_ATOMIC, alpha, y, nullptr, nullptr, nullptr);
    case SPMX_K_CSC_LB_SORT:
      return spmx_spmspv_csc(h, h->lb_variant, SPMX_WB_SORT, alpha, y, nullptr, nullptr, nullptr);
    case SPMX_K_CSC_LB_ATOMIC:
      return spmx_spmspv_csc(h, h->lb_variant, SPMX_WB_ATOMIC, alpha, y, nullptr, nullptr, nullptr);
    case SPMX_K_CSR_NAIVE_SPMSPV:
      SPMX_TRY(spmx_sparse2bitarray(h));
      return spmx_naivespmspv(h, alpha, y);
    case SPMX_K_CSR_LB_SPMSPV:
      SPMX_TRY(spmx_sparse2bitarray(h));
      if (h->spmv_type == SPMX_SPMV_HOLA && !h->hola_ready) SPMX_TRY(spmx_hola_preprocess(h));
      return spmx_spmspv(h, alpha, y);
    case SPMX_K_NAIVE_SPMV:
      SPMX_TRY(spmx_sparse2dense(h));
      return spmx_naivespmv(h, alpha, y);
    case SPMX_K_LB_SPMV:
      SPMX_TRY(spmx_sparse2dense(h));
      if (h->spmv_type == SPMX_SPMV_HOLA && !h->hola_ready) SPMX_TRY(spmx_hola_preprocess(h));
      return spmx_spmv(h, alpha, y);
    default:
      return set_error(SPMX_ERR_INVALID_VALUE, "kernel id must be in [0, 8)");
  }
}

extern "C" int spmx_run_adaptive(spmx_handle_t h, float alpha, float* y, int* kernel_used) {
  SPMX_CHECK_HANDLE(h);
  int kid = 0;
  SPMX_TRY(spmx_select(h, &kid));
  if (kernel_used) *kernel_used = kid;
  return spmx_run_kernel(h, kid, alpha, y);
}

// ---------------------------------------------------------------------------
// BFS: level-synchronous, direction-optimising (push = CSC SpMSpV, pull =
// bitmap-gated CSR SpMSpV).  For a symmetric pattern CSR and CSC coincide.
// ---------------------------------------------------------------------------
static int bfs_stepped(spmx_handle_t h, int source, int* levels, int* depth);

static int ensure_bfs(spmx_handle_t h) {
  if (h->bfs_n == h->n && h->bfs_visited) return SPMX_SUCCESS;
  dfree(h->bfs_visited); dfree(h->bfs_front); dfree(h->bfs_q[0]); dfree(h->bfs_q[1]);
  dfree(h->bfs_cnt); dfree(h->bfs_edges); dfree(h->bfs_fb1); dfree(h->bfs_fb2); dfree(h->bfs_ctrl);
  const size_t words = (size_t)std::max((h->n + 31) / 32, 1);
  SPMX_TRY(dalloc((void**)&h->bfs_visited, 4 * words, "bfs visited"));
  SPMX_TRY(dalloc((void**)&h->bfs_front, 4 * words, "bfs front"));
  SPMX_TRY(dalloc((void**)&h->bfs_fb1, 4 * words, "bfs front 1"));
  SPMX_TRY(dalloc((void**)&h->bfs_fb2, 4 * words, "bfs front 2"));
  SPMX_TRY(dalloc((void**)&h->bfs_q[0], 4 * (size_t)std::max(h->n, 1), "bfs queue 0"));
  SPMX_TRY(dalloc((void**)&h->bfs_q[1], 4 * (size_t)std::max(h->n, 1), "bfs queue 1"));
  SPMX_TRY(dalloc((void**)&h->bfs_cnt, 4 * 4, "bfs counts"));
  SPMX_TRY(dalloc((void**)&h->bfs_edges, 8 * 4, "bfs edges"));
  SPMX_TRY(dalloc((void**)&h->bfs_ctrl, sizeof(BfsCtrl), "bfs ctrl"));
  h->bfs_n = h->n;
  return SPMX_SUCCESS;
}

static int bfs_check(spmx_handle_t h) {
  if (!h->has_csr) return set_error(SPMX_ERR_NOT_READY, "BFS needs the (symmetric) CSR pattern");
  if (h->m != h->n) return set_error(SPMX_ERR_INVALID_VALUE, "BFS needs a square matrix");
  return SPMX_SUCCESS;
}

extern "C" int spmx_set_bfs_mode(spmx_handle_t h, int mode) {
  SPMX_CHECK_HANDLE(h);
  if (mode != 0 && mode != 1) return set_error(SPMX_ERR_INVALID_VALUE, "BFS mode must be 0 or 1");
  h->bfs_mode = mode;
  return SPMX_SUCCESS;
}

static int bfs_persistent(spmx_handle_t h, int source, int* levels, int* depth) {
  cudaStream_t st = h->stream;
  const int n = h->n;
  // the kernel initialises levels, the visited set and the frontier bitmaps
  BfsPersistentArgs a{n, source, h->num_sms, (long long)h->nnz, h->rowptr, h->col, levels,
                      h->bfs_visited, h->bfs_front, h->bfs_fb1, h->bfs_fb2, h->bfs_q[0], h->bfs_q[1],
                      (BfsCtrl*)h->bfs_ctrl, h->bfs_alpha, h->bfs_beta, h->d_err};
  const int rc = launch_bfs_persistent(a, st);
  if (rc) return set_error(SPMX_ERR_CUDA, std::string("cooperative BFS launch: ") +
                                              cudaGetErrorString(cudaGetLastError()));
  if (depth) {  // through the handle's pinned word: a pageable copy costs ~15 us
    SPMX_CUDA(cudaMemcpyAsync(h->h_pinned + 1, &((BfsCtrl*)h->bfs_ctrl)->depth, sizeof(int),
                              cudaMemcpyDeviceToHost, st));
    SPMX_CUDA(cudaStreamSynchronize(st));
    *depth = h->h_pinned[1];
  }
  return SPMX_SUCCESS;
}

extern "C" int spmx_bfs(spmx_handle_t h, int source, int* levels, int* depth) {
  SPMX_CHECK_HANDLE(h);
  SPMX_TRY(bfs_check(h));
  if (source < 0 || source >= h->n) return set_error(SPMX_ERR_INVALID_VALUE, "source out of range");
  if (!levels) return set_error(SPMX_ERR_INVALID_VALUE, "levels is NULL");
  SPMX_TRY(ensure_bfs(h));
  if (h->bfs_mode == 0) return bfs_persistent(h, source, levels, depth);
  return bfs_stepped(h, source, levels, depth);
}

static int ensure_msbfs(spmx_handle_t h) {
  if (h->ms_n == h->n && h->ms_visit) return SPMX_SUCCESS;
  dfree(h->ms_visit); dfree(h->ms_front0); dfree(h->ms_front1); dfree(h->ms_next);
  dfree(h->ms_q0); dfree(h->ms_q1); dfree(h->ms_srcs); dfree(h->ms_ctrl);
  const size_t n = (size_t)std::max(h->n, 1);
  SPMX_TRY(dalloc((void**)&h->ms_visit, 8 * n, "msbfs visit"));
  SPMX_TRY(dalloc((void**)&h->ms_front0, 8 * n, "msbfs front 0"));
  SPMX_TRY(dalloc((void**)&h->ms_front1, 8 * n, "msbfs front 1"));
  SPMX_TRY(dalloc((void**)&h->ms_next, 8 * n, "msbfs next"));
  SPMX_TRY(dalloc((void**)&h->ms_q0, 4 * n, "msbfs queue 0"));
  SPMX_TRY(dalloc((void**)&h->ms_q1, 4 * n, "msbfs queue 1"));
  SPMX_TRY(dalloc((void**)&h->ms_srcs, 4 * 64, "msbfs sources"));
  SPMX_TRY(dalloc((void**)&h->ms_ctrl, sizeof(BfsCtrl), "msbfs ctrl"));
  h->ms_n = h->n;
  return SPMX_SUCCESS;
}

// vertices of degree above this are pulled in chunks of this many edges
constexpr int kHubDegree = 1024;

// hub chunk list of the multi-source pull, built once per matrix
static int ensure_hubs(spmx_handle_t h) {
  if (h->ms_hub_rowptr == h->rowptr && h->ms_hub_nnz == h->nnz && h->ms_hcounters) return SPMX_SUCCESS;
  cudaStream_t st = h->stream;
  SPMX_CUDA(cudaStreamSynchronize(st));
  dfree(h->ms_hchunk); dfree(h->ms_hcnt); dfree(h->ms_hacc); dfree(h->ms_hleft); dfree(h->ms_hcounters);
  h->ms_hchunk = nullptr; h->ms_hcnt = nullptr; h->ms_hacc = nullptr; h->ms_hleft = nullptr;
  h->ms_hcounters = nullptr;
  const long long nnz = std::max(h->nnz, 0);
  const int max_hubs = (int)(nnz / (kHubDegree + 1) + 1);
  const long long max_chunks = nnz / kHubDegree + max_hubs + 1;
  SPMX_TRY(dalloc((void**)&h->ms_hchunk, sizeof(int4) * (size_t)max_chunks, "msbfs hub chunks"));
  SPMX_TRY(dalloc((void**)&h->ms_hcnt, 4 * (size_t)max_hubs, "msbfs hub chunk counts"));
  SPMX_TRY(dalloc((void**)&h->ms_hacc, 8 * (size_t)max_hubs, "msbfs hub accumulators"));
  SPMX_TRY(dalloc((void**)&h->ms_hleft, 4 * (size_t)max_hubs, "msbfs hub counters"));
  SPMX_TRY(dalloc((void**)&h->ms_hcounters, 8, "msbfs hub totals"));
  SPMX_CUDA(cudaMemsetAsync(h->ms_hcounters, 0, 8, st));
  launch_hub_chunks(h->n, h->rowptr, kHubDegree, h->ms_hchunk, h->ms_hcnt, h->ms_hcounters, max_hubs,
                    (int)max_chunks, st);
  int cnt[2] = {0, 0};
  SPMX_CUDA(cudaMemcpyAsync(cnt, h->ms_hcounters, 8, cudaMemcpyDeviceToHost, st));
  SPMX_CUDA(cudaStreamSynchronize(st));
  if (cnt[0] > max_hubs || cnt[1] > max_chunks) return set_error(SPMX_ERR_OOB, "hub chunk capacity");
  h->ms_nhubs = cnt[0];
  h->ms_nhchunks = cnt[1];
  h->ms_hub_rowptr = h->rowptr;
  h->ms_hub_nnz = h->nnz;
  return SPMX_SUCCESS;
}

extern "C" int spmx_bfs_batched(spmx_handle_t h, const int* srcs, int nsrc, int* levels,
                                int layout, int* depth) {
  SPMX_CHECK_HANDLE(h);
  SPMX_TRY(bfs_check(h));
  if (nsrc < 1 || nsrc > 64) return set_error(SPMX_ERR_INVALID_VALUE, "nsrc must be in [1, 64]");
  if (!srcs || !levels) return set_error(SPMX_ERR_INVALID_VALUE, "NULL argument");
  if (layout != 0 && layout != 1) return set_error(SPMX_ERR_INVALID_VALUE, "layout must be 0 or 1");
  for (int s = 0; s < nsrc; ++s)
    if (srcs[s] < 0 || srcs[s] >= h->n) return set_error(SPMX_ERR_INVALID_VALUE, "source out of range");
  SPMX_TRY(ensure_msbfs(h));
  SPMX_TRY(ensure_hubs(h));
  cudaStream_t st = h->stream;
  const size_t n = (size_t)h->n;
  const size_t total = n * (size_t)nsrc;
  int* vmajor = levels;
  if (layout == 1) {
    if (h->ms_tmp_len < total) {
      SPMX_CUDA(cudaStreamSynchronize(st));
      dfree(h->ms_tmp);
      h->ms_tmp = nullptr;
      h->ms_tmp_len = 0;
      SPMX_TRY(dalloc((void**)&h->ms_tmp, 4 * total, "msbfs levels"));
      h->ms_tmp_len = total;
    }
    vmajor = h->ms_tmp;
  }
  SPMX_CUDA(cudaMemcpyAsync(h->ms_srcs, srcs, 4 * (size_t)nsrc, cudaMemcpyHostToDevice, st));
  SPMX_CUDA(cudaMemsetAsync(vmajor, 0xff, 4 * total, st));
  SPMX_CUDA(cudaMemsetAsync(h->ms_visit, 0, 8 * n, st));
  SPMX_CUDA(cudaMemsetAsync(h->ms_front0, 0, 8 * n, st));
  SPMX_CUDA(cudaMemsetAsync(h->ms_front1, 0, 8 * n, st));
  SPMX_CUDA(cudaMemsetAsync(h->ms_next, 0, 8 * n, st));
  if (h->ms_nhubs > 0) {
    SPMX_CUDA(cudaMemsetAsync(h->ms_hacc, 0, 8 * (size_t)h->ms_nhubs, st));
    SPMX_CUDA(cudaMemcpyAsync(h->ms_hleft, h->ms_hcnt, 4 * (size_t)h->ms_nhubs, cudaMemcpyDeviceToDevice, st));
  }
  HubChunks hub{h->ms_hchunk, h->ms_nhchunks, h->ms_hcnt, h->ms_hacc, h->ms_hleft, h->ms_nhubs, kHubDegree};
  MsBfsArgs a{h->n, nsrc, h->num_sms, (long long)h->nnz, h->msbfs_alpha, h->ms_srcs, h->rowptr,
              h->col, vmajor, h->ms_visit, h->ms_front0, h->ms_front1, h->ms_next, h->ms_q0,
              h->ms_q1, (BfsCtrl*)h->ms_ctrl, hub, h->d_err};
  if (launch_msbfs_persistent(a, st))
    return set_error(SPMX_ERR_CUDA, std::string("cooperative multi-source BFS launch: ") +
                                        cudaGetErrorString(cudaGetLastError()));
  if (layout == 1) launch_levels_transpose(h->n, nsrc, vmajor, levels, st);
  SPMX_TRY(launch_ok("batched bfs"));
  if (depth) {
    SPMX_CUDA(cudaMemcpyAsync(h->h_pinned + 1, &((BfsCtrl*)h->ms_ctrl)->depth, sizeof(int),
                              cudaMemcpyDeviceToHost, st));
    SPMX_CUDA(cudaStreamSynchronize(st));
    *depth = h->h_pinned[1];
  }
  return SPMX_SUCCESS;
}

static int bfs_stepped(spmx_handle_t h, int source, int* levels, int* depth) {
  cudaStream_t st = h->stream;
  const int n = h->n;
  const size_t words = (size_t)((n + 31) / 32);
  SPMX_CUDA(cudaMemsetAsync(levels, 0xff, 4 * (size_t)n, st));
  SPMX_CUDA(cudaMemsetAsync(h->bfs_visited, 0, 4 * words, st));
  launch_bfs_init(source, levels, h->bfs_visited, h->bfs_q[0], h->bfs_cnt, st);
  // degree of the source
  int rp[2];
  SPMX_CUDA(cudaMemcpyAsync(rp, h->rowptr + source, 8, cudaMemcpyDeviceToHost, st));
  SPMX_CUDA(cudaStreamSynchronize(st));
  long long nf = 1, mf = rp[1] - rp[0];
  long long mu = (long long)h->nnz - mf;
  const double alpha_b = 14.0, beta_b = 24.0;
  bool pull = false;
  int cur = 0, level = 0;
  const int max_grid = h->num_sms * 8;
  while (nf > 0) {
    if (!pull && (double)mf > (double)mu / alpha_b) pull = true;
    else if (pull && (double)nf < (double)n / beta_b) pull = false;
    const int nxt = cur ^ 1;
    SPMX_CUDA(cudaMemsetAsync(h->bfs_cnt + nxt, 0, sizeof(int), st));
    SPMX_CUDA(cudaMemsetAsync(h->bfs_edges + nxt, 0, sizeof(unsigned long long), st));
    if (pull) {
      SPMX_CUDA(cudaMemsetAsync(h->bfs_front, 0, 4 * words, st));
      launch_scatter((int)nf, n, h->bfs_q[cur], nullptr, nullptr, (int*)h->bfs_front, h->d_err, st);
      launch_bfs_pull(n, h->rowptr, h->col, h->bfs_visited, h->bfs_front, levels, level + 1,
                      h->bfs_q[nxt], h->bfs_cnt + nxt, h->bfs_edges + nxt, h->d_err, max_grid, st);
    } else {
      launch_bfs_push((int)nf, h->bfs_q[cur], n, h->rowptr, h->col, h->bfs_visited, levels,
                      level + 1, h->bfs_q[nxt], h->bfs_cnt + nxt, h->bfs_edges + nxt, h->d_err,
                      max_grid, st);
    }
    SPMX_TRY(launch_ok("bfs level"));
    int cnt = 0;
    unsigned long long edges = 0;
    SPMX_CUDA(cudaMemcpyAsync(&cnt, h->bfs_cnt + nxt, sizeof(int), cudaMemcpyDeviceToHost, st));
    SPMX_CUDA(cudaMemcpyAsync(&edges, h->bfs_edges + nxt, 8, cudaMemcpyDeviceToHost, st));
    SPMX_CUDA(cudaStreamSynchronize(st));
    nf = cnt;
    mf = (long long)edges;
    mu -= mf;
    cur = nxt;
    if (nf > 0) ++level;
  }
  if (depth) *depth = level + 1;
  return SPMX_SUCCESS;
}
