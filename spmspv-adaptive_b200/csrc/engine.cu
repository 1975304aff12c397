// C ABI of the engine, part 1: lifecycle, matrix input, CSR->CSC, vectors and
// their format conversions, scratch, SpMV / CSR SpMSpV and CSC SpMSpV.
// Reference: SpmspvHandle (H = hice-spmspv/hice/la/include/spmspv/csc-spmspv/
// spmspv.h); line numbers are given per entry point in spmx.h.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <mutex>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "feat.h"
#include "kernels.h"
#include "sort.h"
#include "bucket.h"

namespace spmx {

static thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int dalloc(void** p, size_t bytes, const char* what) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return set_error(SPMX_ERR_ALLOC, std::string("cudaMalloc(") + what + ", " +
                                         std::to_string(bytes) + " B): " +
                                         cudaGetErrorString(e));
  }
  return SPMX_SUCCESS;
}

void dfree(void* p) {
  if (p) cudaFree(p);
}

cudaError_t kernel_smem_limit(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::vector<std::pair<std::pair<const void*, int>, size_t>> set;  // (kernel, device) -> bytes
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  for (auto& s : set) {
    if (s.first.first == kernel && s.first.second == dev) {
      if (s.second == bytes) return cudaSuccess;
      e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
      if (e == cudaSuccess) s.second = bytes;
      return e;
    }
  }
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) set.push_back({{kernel, dev}, bytes});
  return e;
}

static std::atomic<unsigned long long> g_launches{0};

// L2 persistence for gathered operands: on by default, SPMX_L2_WINDOW=0 turns
// it off.  The first use on a device raises the CUDA context's persisting-L2
// set-aside (a property of this process's context, released with it) to at
// most 32 MiB.
static std::mutex g_l2_mu;
static int g_l2_state[64] = {0};       // 0 unknown, 1 ready, -1 unavailable
static size_t g_l2_maxwin[64] = {0};

size_t l2_window_bytes(const void* base, size_t bytes) {
  // off unless SPMX_L2_WINDOW is set to a non-zero value: x stays in L2
  // without it, and the first window raises the context's persisting-L2
  // set-aside (32 MB) for the rest of the process, which slows the kernels
  // that use no window (the round SpMV by about 9 %)
  static const bool enabled = [] {
    const char* e = getenv("SPMX_L2_WINDOW");
    return e && e[0] && e[0] != '0';
  }();
  if (!enabled || !base || bytes == 0) return 0;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { cudaGetLastError(); return 0; }
  std::lock_guard<std::mutex> lock(g_l2_mu);
  if (g_l2_state[dev] == 0) {
    int maxwin = 0, maxpersist = 0;
    cudaDeviceGetAttribute(&maxwin, cudaDevAttrMaxAccessPolicyWindowSize, dev);
    cudaDeviceGetAttribute(&maxpersist, cudaDevAttrMaxPersistingL2CacheSize, dev);
    size_t cur = 0;
    cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize);
    const size_t want = std::min<size_t>((size_t)maxpersist, (size_t)32 << 20);
    bool ok = maxwin > 0 && maxpersist > 0;
    if (ok && cur < want) ok = cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) == cudaSuccess;
    cudaGetLastError();
    g_l2_maxwin[dev] = ok ? (size_t)maxwin : 0;
    g_l2_state[dev] = ok ? 1 : -1;
  }
  if (g_l2_state[dev] != 1) return 0;
  return std::min(bytes, g_l2_maxwin[dev]);
}
void note_launch(int k) { g_launches.fetch_add((unsigned long long)k, std::memory_order_relaxed); }

int csc_lb_blocks_per_sm();

}  // namespace spmx

using namespace spmx;


static int pow2_group(double mean) {
  int g = 1;
  while (g < 32 && g < mean) g <<= 1;
  return g;
}

// lanes per row for short-row streaming passes: about 4 nonzeros per lane
static int stream_group(double mean) {
  int g = 1;
  while (g < 32 && 8.0 * g <= mean) g <<= 1;
  return g;
}

static int ceil_log2(long long v) {
  int b = 0;
  while ((1LL << b) < v) ++b;
  return b < 1 ? 1 : b;
}

// ---------------------------------------------------------------------------
// lifecycle
// ---------------------------------------------------------------------------
extern "C" const char* spmx_last_error_string(void) { return g_last_error.c_str(); }

extern "C" unsigned long long spmx_launch_count(void) { return g_launches.load(); }

extern "C" int spmx_create(int m, int n, int nnz, spmx_handle_t* out) {
  if (!out) return set_error(SPMX_ERR_INVALID_VALUE, "out is NULL");
  *out = nullptr;
  if (m < 0 || n < 0 || nnz < 0)
    return set_error(SPMX_ERR_INVALID_VALUE, "negative m, n or nnz");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(SPMX_ERR_NO_DEVICE, "no CUDA device visible");
  }
  spmx_handle_s* h = new spmx_handle_s();
  h->m = m;
  h->n = n;
  h->nnz = nnz;
  h->num_ints = (n + 31) / 32;
  cudaGetDevice(&h->device);
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
  int rc = SPMX_SUCCESS;
  rc = rc ? rc : dalloc((void**)&h->d_counts, sizeof(int) * kCntTotal, "counts");
  rc = rc ? rc : dalloc((void**)&h->d_err, sizeof(int), "err");
  rc = rc ? rc : dalloc((void**)&h->d_facc, sizeof(double) * 4, "facc");
  rc = rc ? rc : dalloc((void**)&h->d_iacc, sizeof(int) * 4, "iacc");
  rc = rc ? rc : dalloc((void**)&h->d_u64, sizeof(unsigned long long) * 4, "u64");
  const long long big = std::max<long long>(std::max<long long>(m, n), nnz);
  h->ls.status_len = (int)(big / 2048 + 4);
  rc = rc ? rc : dalloc((void**)&h->ls.status, sizeof(unsigned long long) * h->ls.status_len,
                        "lookback status");
  rc = rc ? rc : dalloc((void**)&h->ls.ticket, sizeof(unsigned) * 4, "ticket");
  rc = rc ? rc : dalloc((void**)&h->ls.counts, sizeof(unsigned) * h->ls.status_len, "range counts");
  if (!rc && cudaMallocHost((void**)&h->h_pinned, sizeof(int) * 16) != cudaSuccess) {
    cudaGetLastError();
    rc = set_error(SPMX_ERR_ALLOC, "cudaMallocHost(pinned counters)");
  }
  if (!rc) {
    cudaMemset(h->d_counts, 0, sizeof(int) * kCntTotal);
    cudaMemset(h->d_err, 0, sizeof(int));
    cudaMemset(h->ls.status, 0, sizeof(unsigned long long) * h->ls.status_len);
    cudaMemset(h->ls.ticket, 0, sizeof(unsigned) * 4);
    if (cudaDeviceSynchronize() != cudaSuccess) {
      rc = set_error(SPMX_ERR_CUDA, std::string("init: ") + cudaGetErrorString(cudaGetLastError()));
    }
  }
  if (rc) {
    spmx_destroy(h);
    return rc;
  }
  *out = h;
  return SPMX_SUCCESS;
}

static void free_sort_scratch(spmx_handle_t h) {
  dfree(h->sk); dfree(h->sk_alt); dfree(h->sv); dfree(h->sv_alt);
  dfree(h->shist); dfree(h->shist_off); dfree(h->sslot);
  dfree(h->sy_key); dfree(h->sy_val);
  dfree(h->bk_gcount); dfree(h->bk_boff); dfree(h->bk_cursor);
  h->bk_gcount = h->bk_boff = h->bk_cursor = nullptr;
  h->sk = h->sk_alt = h->sv = h->sv_alt = nullptr;
  h->shist = h->shist_off = h->sslot = nullptr;
  h->sy_key = nullptr;
  h->sy_val = nullptr;
  h->sort_ready = false;
}

static void free_csc_scratch(spmx_handle_t h) {
  dfree(h->cs.off); dfree(h->cs.colstart); dfree(h->cs.bstart_tl); dfree(h->cs.bstart_mg);
  h->cs = CscScratch{};
  h->cs_ready = false;
}

extern "C" int spmx_hola_postprocess(spmx_handle_t h);
extern "C" int spmx_csr5_postprocess(spmx_handle_t h);
extern "C" int spmx_tiled_postprocess(spmx_handle_t h);
int tiled_spmv_impl(spmx_handle_t h, float alpha, float* y, bool gated);
extern "C" int spmx_round_postprocess(spmx_handle_t h);
int round_spmv_impl(spmx_handle_t h, float alpha, float* y, bool gated);

extern "C" int spmx_destroy(spmx_handle_t h) {
  if (!h) return SPMX_SUCCESS;
  if (h->stream) cudaStreamSynchronize(h->stream); else cudaDeviceSynchronize();
  cudaGetLastError();
  dfree(h->d_counts); dfree(h->d_err); dfree(h->d_facc); dfree(h->d_iacc); dfree(h->d_u64);
  dfree(h->ls.status); dfree(h->ls.ticket); dfree(h->ls.counts);
  if (h->h_pinned) cudaFreeHost(h->h_pinned);
  dfree(h->own_colptr); dfree(h->own_row); dfree(h->own_cval);
  dfree(h->own_csr_rowptr); dfree(h->own_csr_col); dfree(h->own_csr_val);
  dfree(h->own_xdense); dfree(h->own_bits);
  free_csc_scratch(h);
  free_sort_scratch(h);
  spmx_hola_postprocess(h);
  spmx_csr5_postprocess(h);
  spmx_tiled_postprocess(h);
  spmx_round_postprocess(h);
  spmx_hybrid_postprocess(h);
  dfree(h->bfs_visited); dfree(h->bfs_front); dfree(h->bfs_q[0]); dfree(h->bfs_q[1]);
  dfree(h->bfs_cnt); dfree(h->bfs_edges); dfree(h->bfs_fb1); dfree(h->bfs_fb2); dfree(h->bfs_ctrl);
  dfree(h->ms_visit); dfree(h->ms_front0); dfree(h->ms_front1); dfree(h->ms_next);
  dfree(h->ms_q0); dfree(h->ms_q1); dfree(h->ms_srcs); dfree(h->ms_tmp); dfree(h->ms_ctrl);
  dfree(h->ms_hchunk); dfree(h->ms_hcnt); dfree(h->ms_hacc); dfree(h->ms_hleft); dfree(h->ms_hcounters);
  for (void* p : h->batch_buf) dfree(p);
  dfree(h->batch_hist); dfree(h->batch_hoff); dfree(h->batch_invptr); dfree(h->batch_rec);
  dfree(h->batch_chunk); dfree(h->batch_ctr);
  delete h;
  return SPMX_SUCCESS;
}

extern "C" int spmx_set_stream(spmx_handle_t h, void* stream) {
  SPMX_CHECK_HANDLE(h);
  h->stream = (cudaStream_t)stream;
  return SPMX_SUCCESS;
}

extern "C" int spmx_warmup(spmx_handle_t h) {
  SPMX_CHECK_HANDLE(h);
  SPMX_CUDA(cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream));
  SPMX_CUDA(cudaStreamSynchronize(h->stream));
  return SPMX_SUCCESS;
}

extern "C" int spmx_check_device_error(spmx_handle_t h) {
  SPMX_CHECK_HANDLE(h);
  SPMX_CUDA(cudaStreamSynchronize(h->stream));
  int e = 0;
  SPMX_CUDA(cudaMemcpy(&e, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  SPMX_CUDA(cudaMemset(h->d_err, 0, sizeof(int)));
  if (e & kDevErrTimeout) return set_error(SPMX_ERR_TIMEOUT, "a bounded device wait timed out");
  if (e & kDevErrOob) return set_error(SPMX_ERR_OOB, "an index was out of range (bad input)");
  if (e & kDevErrCapacity) return set_error(SPMX_ERR_OOB, "an internal capacity was exceeded");
  return SPMX_SUCCESS;
}

// read the device counter `slot` to the host (synchronises the stream)
static int read_counter(spmx_handle_t h, int slot, int* out) {
  SPMX_CUDA(cudaMemcpyAsync(h->h_pinned, h->d_counts + slot, sizeof(int),
                            cudaMemcpyDeviceToHost, h->stream));
  SPMX_CUDA(cudaStreamSynchronize(h->stream));
  *out = h->h_pinned[0];
  return SPMX_SUCCESS;
}

extern "C" int spmx_get_device_counts(spmx_handle_t h, const int** d_counts) {
  SPMX_CHECK_HANDLE(h);
  if (!d_counts) return set_error(SPMX_ERR_INVALID_VALUE, "d_counts is NULL");
  *d_counts = h->d_counts;
  return SPMX_SUCCESS;
}

// ---------------------------------------------------------------------------
// matrix input
// ---------------------------------------------------------------------------
extern "C" int spmx_input_csr(spmx_handle_t h, int nnz, const int* rowptr,
                              const int* col, const float* val) {
  SPMX_CHECK_HANDLE(h);
  if (nnz != h->nnz) return set_error(SPMX_ERR_INVALID_VALUE, "nnz differs from the handle's nnz");
  if (!rowptr || (!col && nnz > 0))
    return set_error(SPMX_ERR_INVALID_VALUE, "NULL CSR array");
  h->rowptr = rowptr;
  h->col = col;
  h->val = val;
  h->has_csr = true;
  h->mat_feat_ready = false;
  h->std_row_ready = false;
  h->batch_chunk_ready = false;
  return SPMX_SUCCESS;
}

extern "C" int spmx_input_csc(spmx_handle_t h, int nnz, const int* csc_row,
                              const int* csc_col, const float* csc_val) {
  SPMX_CHECK_HANDLE(h);
  if (nnz != h->nnz) return set_error(SPMX_ERR_INVALID_VALUE, "nnz differs from the handle's nnz");
  if (!csc_col || (!csc_row && nnz > 0))
    return set_error(SPMX_ERR_INVALID_VALUE, "NULL CSC array");
  h->csc_row = csc_row;
  h->csc_colptr = csc_col;
  h->csc_val = csc_val;
  h->has_csc = true;
  return SPMX_SUCCESS;
}

static int ensure_sort_scratch(spmx_handle_t h) {
  if (h->sort_ready) return SPMX_SUCCESS;
  const size_t cap = (size_t)std::max(h->nnz, 1);
  SPMX_TRY(dalloc((void**)&h->sk, 4 * cap, "sort keys"));
  SPMX_TRY(dalloc((void**)&h->sk_alt, 4 * cap, "sort keys alt"));
  SPMX_TRY(dalloc((void**)&h->sv, 4 * cap, "sort vals"));
  SPMX_TRY(dalloc((void**)&h->sv_alt, 4 * cap, "sort vals alt"));
  SPMX_TRY(dalloc((void**)&h->sslot, 4 * cap, "sort slots"));
  const size_t hn = radix_hist_ints((int)cap);
  SPMX_TRY(dalloc((void**)&h->shist, 4 * hn, "radix hist"));
  SPMX_TRY(dalloc((void**)&h->shist_off, 4 * hn, "radix hist off"));
  const size_t ycap = (size_t)std::max(h->m, 1);
  SPMX_TRY(dalloc((void**)&h->sy_key, 4 * ycap, "sparse y keys"));
  SPMX_TRY(dalloc((void**)&h->sy_val, 4 * ycap, "sparse y vals"));
  SPMX_TRY(dalloc((void**)&h->bk_gcount, 4 * (size_t)kBucketMax, "bucket counts"));
  SPMX_TRY(dalloc((void**)&h->bk_boff, 4 * (size_t)(kBucketMax + 1), "bucket offsets"));
  SPMX_TRY(dalloc((void**)&h->bk_cursor, 4 * (size_t)kBucketMax, "bucket cursors"));
  h->sort_ready = true;
  return SPMX_SUCCESS;
}

extern "C" int spmx_to_csc(spmx_handle_t h) {
  SPMX_CHECK_HANDLE(h);
  if (!h->has_csr) return set_error(SPMX_ERR_NOT_READY, "ToCSC needs the CSR input");
  const int m = h->m, n = h->n, nnz = h->nnz;
  dfree(h->own_colptr); dfree(h->own_row); dfree(h->own_cval);
  h->own_colptr = nullptr; h->own_row = nullptr; h->own_cval = nullptr;
  SPMX_TRY(dalloc((void**)&h->own_colptr, 4 * (size_t)(n + 1), "csc colptr"));
  SPMX_TRY(dalloc((void**)&h->own_row, 4 * (size_t)std::max(nnz, 1), "csc row"));
  if (h->val) SPMX_TRY(dalloc((void**)&h->own_cval, 4 * (size_t)std::max(nnz, 1), "csc val"));
  cudaStream_t st = h->stream;
  // column counts -> colptr
  int* cnt = nullptr;
  SPMX_TRY(dalloc((void**)&cnt, 4 * (size_t)std::max(n, 1), "col counts"));
  SPMX_CUDA(cudaMemsetAsync(cnt, 0, 4 * (size_t)std::max(n, 1), st));
  launch_count_keys(nnz, n, h->col, cnt, h->d_err, st);
  if (n > 0) {
    if (launch_scan_exclusive(cnt, h->own_colptr, n, h->own_colptr + n, h->ls, h->d_err, st)) {
      dfree(cnt);
      return set_error(SPMX_ERR_INVALID_VALUE, "scan capacity");
    }
  } else {
    SPMX_CUDA(cudaMemsetAsync(h->own_colptr, 0, 4, st));
  }
  if (nnz > 0) {
    // stable sort of the row-major COO by column
    unsigned *k0 = nullptr, *k1 = nullptr, *r0 = nullptr, *r1 = nullptr, *v0 = nullptr, *v1 = nullptr;
    int *hist = nullptr, *hoff = nullptr;
    const size_t b = 4 * (size_t)nnz;
    const size_t hn = radix_hist_ints(nnz);
    int rc = SPMX_SUCCESS;
    rc = rc ? rc : dalloc((void**)&k0, b, "t keys");
    rc = rc ? rc : dalloc((void**)&k1, b, "t keys alt");
    rc = rc ? rc : dalloc((void**)&r0, b, "t rows");
    rc = rc ? rc : dalloc((void**)&r1, b, "t rows alt");
    if (h->val) {
      rc = rc ? rc : dalloc((void**)&v0, b, "t vals");
      rc = rc ? rc : dalloc((void**)&v1, b, "t vals alt");
    }
    rc = rc ? rc : dalloc((void**)&hist, 4 * hn, "t hist");
    rc = rc ? rc : dalloc((void**)&hoff, 4 * hn, "t hist off");
    if (!rc) {
      cudaMemcpyAsync(k0, h->col, b, cudaMemcpyDeviceToDevice, st);
      if (h->val) cudaMemcpyAsync(v0, h->val, b, cudaMemcpyDeviceToDevice, st);
      launch_expand_rows(m, h->rowptr, r0, st);
      RadixBuffers rb{k0, k1, r0, r1, v0, v1, hist, hoff, false};
      if (radix_sort_pairs(rb, nnz, ceil_log2(std::max(n, 2)), h->ls, h->d_err, st))
        rc = set_error(SPMX_ERR_INVALID_VALUE, "radix capacity");
      if (!rc) {
        unsigned* rr = rb.result_in_alt ? r1 : r0;
        unsigned* vv = rb.result_in_alt ? v1 : v0;
        cudaMemcpyAsync(h->own_row, rr, b, cudaMemcpyDeviceToDevice, st);
        if (h->val) cudaMemcpyAsync(h->own_cval, vv, b, cudaMemcpyDeviceToDevice, st);
      }
    }
    cudaError_t se = cudaStreamSynchronize(st);
    dfree(k0); dfree(k1); dfree(r0); dfree(r1); dfree(v0); dfree(v1); dfree(hist); dfree(hoff);
    if (rc) { dfree(cnt); return rc; }
    if (se != cudaSuccess) { dfree(cnt); return set_error(SPMX_ERR_CUDA, cudaGetErrorString(se)); }
  }
  SPMX_CUDA(cudaStreamSynchronize(st));
  dfree(cnt);
  h->csc_colptr = h->own_colptr;
  h->csc_row = h->own_row;
  h->csc_val = h->own_cval;
  h->has_csc = true;
  return launch_ok("ToCSC");
}

extern "C" int spmx_copy_csc(spmx_handle_t h, int* row, int* colptr, float* val) {
  SPMX_CHECK_HANDLE(h);
  if (!h->has_csc) return set_error(SPMX_ERR_NOT_READY, "no CSC (call spmx_to_csc)");
  cudaStream_t st = h->stream;
  if (row && h->nnz)
    SPMX_CUDA(cudaMemcpyAsync(row, h->csc_row, 4 * (size_t)h->nnz, cudaMemcpyDeviceToDevice, st));
  if (colptr)
    SPMX_CUDA(cudaMemcpyAsync(colptr, h->csc_colptr, 4 * (size_t)(h->n + 1), cudaMemcpyDeviceToDevice, st));
  if (val && h->csc_val && h->nnz)
    SPMX_CUDA(cudaMemcpyAsync(val, h->csc_val, 4 * (size_t)h->nnz, cudaMemcpyDeviceToDevice, st));
  return SPMX_SUCCESS;
}

extern "C" int spmx_get_csc(spmx_handle_t h, const int** row, const int** colptr,
                            const float** val) {
  SPMX_CHECK_HANDLE(h);
  if (!h->has_csc) return set_error(SPMX_ERR_NOT_READY, "no CSC (call spmx_to_csc)");
  if (row) *row = h->csc_row;
  if (colptr) *colptr = h->csc_colptr;
  if (val) *val = h->csc_val;
  return SPMX_SUCCESS;
}

// ---------------------------------------------------------------------------
// vectors
// ---------------------------------------------------------------------------
extern "C" int spmx_set_x(spmx_handle_t h, float* x) {
  SPMX_CHECK_HANDLE(h);
  h->x_dense = x;
  return SPMX_SUCCESS;
}

extern "C" int spmx_set_sparse_x(spmx_handle_t h, int* key, float* val, int xnnz) {
  SPMX_CHECK_HANDLE(h);
  if (xnnz < 0 || xnnz > h->n)
    return set_error(SPMX_ERR_INVALID_VALUE, "xnnz must be in [0, n]");
  if (xnnz > 0 && (!key || !val)) return set_error(SPMX_ERR_INVALID_VALUE, "NULL x key/val");
  h->x_key = key;
  h->x_val = val;
  h->x_nnz = xnnz;
  h->bin_len = -1;
  return SPMX_SUCCESS;
}

extern "C" int spmx_set_bitvector(spmx_handle_t h, int* bits, int num_ints) {
  SPMX_CHECK_HANDLE(h);
  if (num_ints < (h->n + 31) / 32) return set_error(SPMX_ERR_INVALID_VALUE, "num_ints < ceil(n/32)");
  h->bitvec = bits;
  return SPMX_SUCCESS;
}

extern "C" int spmx_set_sparse_x_dense_x(spmx_handle_t h, int* key, float* val,
                                         float* dense, int xnnz) {
  SPMX_TRY(spmx_set_sparse_x(h, key, val, xnnz));
  h->x_dense = dense;
  return SPMX_SUCCESS;
}

extern "C" int spmx_set_vector_type(spmx_handle_t h, int code) {
  SPMX_CHECK_HANDLE(h);
  if (code < 0 || code > 2) return set_error(SPMX_ERR_INVALID_VALUE, "vector type must be 0, 1 or 2");
  h->vec_type = code;
  return SPMX_SUCCESS;
}

static int ensure_dense_x(spmx_handle_t h) {
  if (h->x_dense) return SPMX_SUCCESS;
  SPMX_TRY(dalloc((void**)&h->own_xdense, 4 * (size_t)std::max(h->n, 1), "dense x"));
  h->x_dense = h->own_xdense;
  return SPMX_SUCCESS;
}

static int ensure_bits(spmx_handle_t h) {
  if (h->bitvec) return SPMX_SUCCESS;
  SPMX_TRY(dalloc((void**)&h->own_bits, 4 * (size_t)std::max(h->num_ints, 1), "bitvector"));
  h->bitvec = h->own_bits;
  return SPMX_SUCCESS;
}

extern "C" int spmx_sparse2dense(spmx_handle_t h) {
  SPMX_CHECK_HANDLE(h);
  SPMX_TRY(ensure_dense_x(h));
  if (launch_dense_from_sparse(h->x_nnz, h->n, h->x_key, h->x_val, h->x_dense, h->d_err, h->num_sms,
                               h->stream))
    return set_error(SPMX_ERR_CUDA, "sparse2dense launch");
  h->vec_type = SPMX_VEC_DENSE;
  return launch_ok("sparse2dense");
}

extern "C" int spmx_sparse2bitarray(spmx_handle_t h) {
  SPMX_CHECK_HANDLE(h);
  SPMX_TRY(ensure_dense_x(h));
  SPMX_TRY(ensure_bits(h));
  SPMX_CUDA(cudaMemsetAsync(h->x_dense, 0, 4 * (size_t)h->n, h->stream));
  SPMX_CUDA(cudaMemsetAsync(h->bitvec, 0, 4 * (size_t)h->num_ints, h->stream));
  launch_scatter(h->x_nnz, h->n, h->x_key, h->x_val, h->x_dense, h->bitvec, h->d_err, h->stream);
  h->vec_type = SPMX_VEC_BITARRAY;
  return launch_ok("sparse2bitarray");
}

static int dense_to_sparse(spmx_handle_t h, int len, const float* dense, int* key,
                           float* val, int slot, int* host_count) {
  if (launch_compact_nonzero(len, dense, key, val, h->d_counts + slot, h->ls, h->d_err, h->stream))
    return set_error(SPMX_ERR_INVALID_VALUE, "compaction capacity");
  SPMX_TRY(launch_ok("dense2sparse"));
  if (host_count) SPMX_TRY(read_counter(h, slot, host_count));
  return SPMX_SUCCESS;
}

extern "C" int spmx_dense2sparse(spmx_handle_t h, int* xnnz) {
  SPMX_CHECK_HANDLE(h);
  if (!h->x_dense || !h->x_key || !h->x_val)
    return set_error(SPMX_ERR_NOT_READY, "dense2sparse needs dense x and x key/val buffers");
  int cnt = 0;
  SPMX_TRY(dense_to_sparse(h, h->n, h->x_dense, h->x_key, h->x_val, kCntXnnz, &cnt));
  h->x_nnz = cnt;
  h->bin_len = -1;
  if (xnnz) *xnnz = cnt;
  h->vec_type = SPMX_VEC_SPARSE;
  return SPMX_SUCCESS;
}

extern "C" int spmx_bitarray2sparse(spmx_handle_t h, int* xnnz) {
  return spmx_dense2sparse(h, xnnz);
}

extern "C" int spmx_dense2bitarray(spmx_handle_t h) {
  SPMX_CHECK_HANDLE(h);
  if (!h->x_dense) return set_error(SPMX_ERR_NOT_READY, "dense2bitarray needs dense x");
  SPMX_TRY(ensure_bits(h));
  launch_dense2bits(h->n, h->x_dense, h->bitvec, h->stream);
  h->vec_type = SPMX_VEC_BITARRAY;
  return launch_ok("dense2bitarray");
}

// grow the look-back status array (synchronises; not for use under capture)
static int ensure_scan_tiles(spmx_handle_t h, long long tiles) {
  if (tiles <= h->ls.status_len) return SPMX_SUCCESS;
  SPMX_CUDA(cudaStreamSynchronize(h->stream));
  dfree(h->ls.status);
  dfree(h->ls.counts);
  h->ls.status = nullptr;
  h->ls.counts = nullptr;
  h->ls.status_len = 0;
  const int len = (int)(tiles + 4);
  SPMX_TRY(dalloc((void**)&h->ls.status, sizeof(unsigned long long) * len, "lookback status"));
  SPMX_TRY(dalloc((void**)&h->ls.counts, sizeof(unsigned) * len, "range counts"));
  SPMX_CUDA(cudaMemset(h->ls.status, 0, sizeof(unsigned long long) * len));
  h->ls.status_len = len;
  return SPMX_SUCCESS;
}

extern "C" int spmx_dense2sparse_outer(spmx_handle_t h, int m, const float* dense,
                                       int* ynnz, int* key, float* val) {
  SPMX_CHECK_HANDLE(h);
  if (m < 0 || (m > 0 && (!dense || !key || !val)))
    return set_error(SPMX_ERR_INVALID_VALUE, "bad dense2sparse_outer arguments");
  SPMX_TRY(ensure_scan_tiles(h, ((long long)m + 2047) / 2048));
  return dense_to_sparse(h, m, dense, key, val, kCntYnnz, ynnz);
}

// a page-locked host buffer the device can address (UVA-mapped)
static int host_mapped(const void* p, const char* what) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return set_error(SPMX_ERR_INVALID_VALUE, std::string(what) + " is not a pointer CUDA knows");
  }
  if (at.type != cudaMemoryTypeHost || at.devicePointer != p)
    return set_error(SPMX_ERR_INVALID_VALUE,
                     std::string(what) + " must be page-locked host memory mapped into the device's "
                                         "address space (cudaHostAlloc / cudaMallocHost)");
  return SPMX_SUCCESS;
}

extern "C" int spmx_dense2sparse_to_host(spmx_handle_t h, int m, const float* dense, int* h_key,
                                         float* h_val, int* h_count) {
  SPMX_CHECK_HANDLE(h);
  if (m < 0 || !h_count || (m > 0 && (!dense || !h_key || !h_val)))
    return set_error(SPMX_ERR_INVALID_VALUE, "bad dense2sparse_to_host arguments");
  SPMX_TRY(host_mapped(h_count, "h_count"));
  if (m > 0) {
    SPMX_TRY(host_mapped(h_key, "h_key"));
    SPMX_TRY(host_mapped(h_val, "h_val"));
  }
  SPMX_TRY(ensure_scan_tiles(h, ((long long)m + 2047) / 2048));
  if (launch_compact_nonzero(m, dense, h_key, h_val, h_count, h->ls, h->d_err, h->stream))
    return set_error(SPMX_ERR_INVALID_VALUE, "compaction capacity");
  return launch_ok("dense2sparse_to_host");
}

extern "C" int spmx_sparse2dense_outer(spmx_handle_t h, int ynnz, const int* key,
                                       const float* val, int m, float* dense) {
  SPMX_CHECK_HANDLE(h);
  if (m < 0 || ynnz < 0 || (m > 0 && !dense)) return set_error(SPMX_ERR_INVALID_VALUE, "bad arguments");
  if (m > 0) SPMX_CUDA(cudaMemsetAsync(dense, 0, 4 * (size_t)m, h->stream));
  launch_scatter(ynnz, m, key, val, dense, nullptr, h->d_err, h->stream);
  return launch_ok("sparse2dense_outer");
}

// ---------------------------------------------------------------------------
// scratch / preprocess
// ---------------------------------------------------------------------------
static int ensure_csc_scratch(spmx_handle_t h) {
  if (h->cs_ready) return SPMX_SUCCESS;
  const int n = std::max(h->n, 1);
  const long long K = kCscLbNT * kCscLbVT;
  h->cs.tl_cap = (int)(h->nnz / K + 2);
  h->cs.mg_cap = (int)(((long long)h->nnz + h->n) / K + 2);
  SPMX_TRY(dalloc((void**)&h->cs.off, 4 * (size_t)(n + 1), "csc off"));
  SPMX_TRY(dalloc((void**)&h->cs.colstart, 4 * (size_t)n, "csc colstart"));
  SPMX_TRY(dalloc((void**)&h->cs.bstart_tl, 4 * (size_t)h->cs.tl_cap, "bstart tl"));
  SPMX_TRY(dalloc((void**)&h->cs.bstart_mg, 4 * (size_t)h->cs.mg_cap, "bstart mg"));
  if (h->lb_grid <= 0) h->lb_grid = h->num_sms * std::max(1, csc_lb_blocks_per_sm());
  h->cs_ready = true;
  return SPMX_SUCCESS;
}

extern "C" int spmx_alloc_pre_buffer(spmx_handle_t h) {
  SPMX_CHECK_HANDLE(h);
  SPMX_TRY(ensure_csc_scratch(h));
  SPMX_TRY(ensure_sort_scratch(h));
  SPMX_TRY(ensure_dense_x(h));
  SPMX_TRY(ensure_bits(h));
  return SPMX_SUCCESS;
}

extern "C" int spmx_dealloc_pre_buffer(spmx_handle_t h) {
  SPMX_CHECK_HANDLE(h);
  cudaStreamSynchronize(h->stream);
  free_csc_scratch(h);
  free_sort_scratch(h);
  return SPMX_SUCCESS;
}

extern "C" int spmx_hola_preprocess(spmx_handle_t h) {
  SPMX_CHECK_HANDLE(h);
  if (!h->has_csr) return set_error(SPMX_FORMAT_ERR_HOLA_SPMV, "Hola needs the CSR input");
  spmx_hola_postprocess(h);
  HolaTables t{};
  t.vt = h->hola_vt;
  t.K = hola_chunk_nnz(t.vt);
  t.nchunks = (h->nnz + t.K - 1) / t.K;
  SPMX_TRY(dalloc((void**)&t.chunk_row, 4 * (size_t)(t.nchunks + 1), "hola chunk rows"));
  SPMX_TRY(dalloc((void**)&t.carry, 8 * (size_t)std::max(2 * t.nchunks, 1), "hola carry"));
  SPMX_TRY(dalloc((void**)&t.arrive, 4 * (size_t)std::max(t.nchunks, 1), "hola arrive"));
  SPMX_CUDA(cudaMemsetAsync(t.arrive, 0, 4 * (size_t)std::max(t.nchunks, 1), h->stream));
  launch_chunk_rows(h->m, h->rowptr, t.K, t.nchunks, t.chunk_row, h->stream);
  h->hola = t;
  h->hola_ready = true;
  return launch_ok("holaPreprocess");
}

extern "C" int spmx_hola_postprocess(spmx_handle_t h) {
  SPMX_CHECK_HANDLE(h);
  if (h->hola_ready) {
    cudaStreamSynchronize(h->stream);
    dfree(h->hola.chunk_row); dfree(h->hola.carry); dfree(h->hola.arrive);
  }
  h->hola = HolaTables{};
  h->hola_ready = false;
  return SPMX_SUCCESS;
}

extern "C" int spmx_set_spmv_type(spmx_handle_t h, int code) {
  SPMX_CHECK_HANDLE(h);
  if (code != SPMX_SPMV_HOLA && code != SPMX_SPMV_CSR5 && code != SPMX_SPMV_TILED && code != SPMX_SPMV_ROUND)
    return set_error(SPMX_ERR_INVALID_VALUE, "spmv type must be 0 (Hola), 1 (CSR5), 2 (tiled) or 3 (round)");
  h->spmv_type = code;
  return SPMX_SUCCESS;
}

// ---------------------------------------------------------------------------
// SpMV / CSR SpMSpV
// ---------------------------------------------------------------------------
static int spmv_common(spmx_handle_t h, float alpha, float* y, bool gated, SpmvArgs* a) {
  if (!h->has_csr || (!h->val && h->nnz > 0))
    return set_error(SPMX_ERR_NOT_READY, "SpMV needs the CSR input with values");
  if (!h->x_dense) return set_error(SPMX_VEC_FORMAT_ERR, "SpMV needs the dense x (set_x / sparse2dense)");
  if (gated && !h->bitvec) return set_error(SPMX_VEC_FORMAT_ERR, "SpMSpV needs the bitarray (sparse2bitarray)");
  if (!y && h->m > 0) return set_error(SPMX_ERR_INVALID_VALUE, "y is NULL");
  *a = SpmvArgs{h->m, h->n, h->nnz, h->rowptr, h->col, h->val, h->x_dense,
                gated ? h->bitvec : nullptr, (double)alpha, y, h->d_err};
  return SPMX_SUCCESS;
}

static int naive_spmv_impl(spmx_handle_t h, float alpha, float* y, bool gated) {
  SpmvArgs a;
  SPMX_TRY(spmv_common(h, alpha, y, gated, &a));
  const int g = h->naive_row_group > 0 ? h->naive_row_group
                                       : pow2_group(h->m ? (double)h->nnz / h->m : 1.0);
  if (launch_spmv_naive(a, g, h->stream)) return set_error(SPMX_ERR_INVALID_VALUE, "bad row group");
  return launch_ok("naive spmv");
}

static int hola_spmv_impl(spmx_handle_t h, float alpha, float* y, bool gated) {
  SpmvArgs a;
  SPMX_TRY(spmv_common(h, alpha, y, gated, &a));
  if (!h->hola_ready) return set_error(SPMX_ERR_NOT_READY, "call spmx_hola_preprocess first");
  if (launch_spmv_hola(a, h->hola, h->stream)) return set_error(SPMX_ERR_INVALID_VALUE, "bad Hola tile");
  return launch_ok("hola spmv");
}

extern "C" int spmx_naivespmv(spmx_handle_t h, float alpha, float* y) {
  SPMX_CHECK_HANDLE(h);
  return naive_spmv_impl(h, alpha, y, false);
}
extern "C" int spmx_naivespmspv(spmx_handle_t h, float alpha, float* y) {
  SPMX_CHECK_HANDLE(h);
  return naive_spmv_impl(h, alpha, y, true);
}
extern "C" int spmx_holaspmv(spmx_handle_t h, float alpha, float* y) {
  SPMX_CHECK_HANDLE(h);
  return hola_spmv_impl(h, alpha, y, false);
}
extern "C" int spmx_holaspmspv(spmx_handle_t h, float alpha, float* y) {
  SPMX_CHECK_HANDLE(h);
  return hola_spmv_impl(h, alpha, y, true);
}

int csr5_spmv_impl(spmx_handle_t h, float alpha, float* y, bool gated);

extern "C" int spmx_csr5spmv(spmx_handle_t h, float alpha, float* y) {
  SPMX_CHECK_HANDLE(h);
  return csr5_spmv_impl(h, alpha, y, false);
}
extern "C" int spmx_csr5spmspv(spmx_handle_t h, float alpha, float* y) {
  SPMX_CHECK_HANDLE(h);
  return csr5_spmv_impl(h, alpha, y, true);
}

extern "C" int spmx_spmv(spmx_handle_t h, float alpha, float* y) {
  SPMX_CHECK_HANDLE(h);
  if (h->spmv_type == SPMX_SPMV_TILED) return tiled_spmv_impl(h, alpha, y, false);
  if (h->spmv_type == SPMX_SPMV_ROUND) return round_spmv_impl(h, alpha, y, false);
  return h->spmv_type == SPMX_SPMV_HOLA ? spmx_holaspmv(h, alpha, y) : spmx_csr5spmv(h, alpha, y);
}
extern "C" int spmx_spmspv(spmx_handle_t h, float alpha, float* y) {
  SPMX_CHECK_HANDLE(h);
  if (h->spmv_type == SPMX_SPMV_TILED) return tiled_spmv_impl(h, alpha, y, true);
  if (h->spmv_type == SPMX_SPMV_ROUND) return round_spmv_impl(h, alpha, y, true);
  return h->spmv_type == SPMX_SPMV_HOLA ? spmx_holaspmspv(h, alpha, y) : spmx_csr5spmspv(h, alpha, y);
}

// ---------------------------------------------------------------------------
// adjoint of y = alpha*A*x: dx = alpha*A^T dy, dvals = alpha*dy[row]*x[col]
// (alpha folded into dy by the caller's choice of dy; here alpha = 1)
// ---------------------------------------------------------------------------
extern "C" int spmx_spmv_backward(spmx_handle_t h, const float* x, const float* dy, float* dx,
                                  float* dvals) {
  SPMX_CHECK_HANDLE(h);
  if (!h->has_csr || (!h->val && h->nnz > 0))
    return set_error(SPMX_ERR_NOT_READY, "backward needs the CSR input with values");
  if (!dy || (dvals && !x)) return set_error(SPMX_ERR_INVALID_VALUE, "NULL x / dy");
  if (h->has_csc && (h->csc_val || h->nnz == 0)) {
    // dx = A^T dy as a gather over the CSC and dvals over the CSR, one launch
    const int g1 = h->naive_row_group > 0 ? h->naive_row_group
                                          : stream_group(h->n ? (double)h->nnz / h->n : 1.0);
    const int g2 = std::min(8, stream_group(h->m ? (double)h->nnz / h->m : 1.0));
    launch_spmv_backward_csc(h->m, h->n, h->rowptr, h->col, h->csc_colptr, h->csc_row, h->csc_val, x, dy, g1,
                             g2, dx, h->nnz > 0 ? dvals : nullptr, h->d_err, h->stream);
    return launch_ok("spmv backward");
  }
  if (!h->hola_ready || h->hola.K != 2048) {
    const int vt = h->hola_vt;
    h->hola_vt = 8;
    const int rc = spmx_hola_preprocess(h);
    h->hola_vt = vt;
    SPMX_TRY(rc);
  }
  cudaStream_t st = h->stream;
  if (dx) SPMX_CUDA(cudaMemsetAsync(dx, 0, 4 * (size_t)h->n, st));
  if (launch_spmv_backward(h->m, h->n, h->nnz, h->rowptr, h->col, h->val, x, dy, h->hola, dx,
                           dvals, h->d_err, st))
    return set_error(SPMX_ERR_INVALID_VALUE, "backward chunk geometry");
  return launch_ok("spmv backward");
}

extern "C" int spmx_spmv_backward_sparse(spmx_handle_t h, const float* x, const int* dy_key,
                                         const float* dy_val, int dy_nnz, float* dx,
                                         float* dvals) {
  SPMX_CHECK_HANDLE(h);
  if (!h->has_csr || (!h->val && h->nnz > 0))
    return set_error(SPMX_ERR_NOT_READY, "backward needs the CSR input with values");
  if (dy_nnz < 0 || dy_nnz > h->m) return set_error(SPMX_ERR_INVALID_VALUE, "dy_nnz must be in [0, m]");
  if (dy_nnz > 0 && (!dy_key || !dy_val)) return set_error(SPMX_ERR_INVALID_VALUE, "NULL dy");
  if (dvals && !x) return set_error(SPMX_ERR_INVALID_VALUE, "NULL x");
  cudaStream_t st = h->stream;
  if (dx) SPMX_CUDA(cudaMemsetAsync(dx, 0, 4 * (size_t)h->n, st));
  if (dvals && h->nnz) SPMX_CUDA(cudaMemsetAsync(dvals, 0, 4 * (size_t)h->nnz, st));
  const int g = pow2_group(h->m ? (double)h->nnz / h->m : 1.0);
  launch_spmv_backward_sparse(h->m, h->n, h->rowptr, h->col, h->val, x, dy_nnz, dy_key, dy_val,
                              g, dx, dvals, h->d_err, st);
  return launch_ok("spmv backward (sparse dy)");
}

// ---------------------------------------------------------------------------
// CSC SpMSpV
// ---------------------------------------------------------------------------
int csc_bucket_impl(spmx_handle_t h, float alpha, float* y, int* ykey, float* yval,
                    int* ynnz, int buckets);
static int ensure_csc_scratch(spmx_handle_t h);
static int read_counter(spmx_handle_t h, int slot, int* out);
static int ensure_scan_tiles(spmx_handle_t h, long long tiles);

static CscArgs csc_args(spmx_handle_t h, float alpha) {
  return CscArgs{h->m, h->n, h->csc_colptr, h->csc_row, h->csc_val, h->x_nnz,
                 h->x_key, h->x_val, (double)alpha, h->d_err, h->d_counts};
}

static int col_group(spmx_handle_t h) {
  if (h->naive_col_group > 0) return h->naive_col_group;
  return pow2_group(h->n ? (double)h->nnz / h->n : 1.0);
}

static int csc_atomic(spmx_handle_t h, int variant, float alpha, float* y, int* ykey,
                      float* yval, int* ynnz) {
  cudaStream_t st = h->stream;
  const CscArgs a = csc_args(h, alpha);
  if (variant == SPMX_CSC_NAIVE) {
    // zero-fill and SpMSpV overlap through a programmatic dependent launch
    if (launch_csc_naive_zeroed(a, col_group(h), y, h->num_sms, st))
      return set_error(SPMX_ERR_INVALID_VALUE, "bad column group");
  } else {
    SPMX_CUDA(cudaMemsetAsync(y, 0, 4 * (size_t)h->m, st));
    SPMX_TRY(ensure_csc_scratch(h));
    if (launch_csc_scan(a, h->cs, h->ls, kCscLbNT * kCscLbVT, st))
      return set_error(SPMX_ERR_INVALID_VALUE, "scan capacity");
    launch_csc_lb(a, h->cs, variant == SPMX_CSC_LB_MERGE ? 1 : 2, y, nullptr, nullptr, h->lb_grid, st);
  }
  SPMX_TRY(launch_ok("csc spmspv"));
  if (ykey && yval) return dense_to_sparse(h, h->m, y, ykey, yval, kCntYnnz, ynnz);
  if (ynnz) *ynnz = 0;
  return SPMX_SUCCESS;
}

static int csc_sort(spmx_handle_t h, int variant, float alpha, float* y, int* ykey,
                    float* yval, int* ynnz) {
  cudaStream_t st = h->stream;
  const CscArgs a = csc_args(h, alpha);
  SPMX_TRY(ensure_csc_scratch(h));
  SPMX_TRY(ensure_sort_scratch(h));
  if (launch_csc_scan(a, h->cs, h->ls, kCscLbNT * kCscLbVT, st))
    return set_error(SPMX_ERR_INVALID_VALUE, "scan capacity");
  // the pair count sizes the sort launches (the reference reads it back too,
  // DEV/csc_sort_spmspv.cuh:266)
  int bin_len = 0;
  SPMX_TRY(read_counter(h, kCntBinlen, &bin_len));
  h->bin_len = bin_len;
  if (bin_len > h->nnz) return set_error(SPMX_ERR_INVALID_VALUE, "bin_len exceeds nnz: duplicate x keys");
  if (variant == SPMX_CSC_NAIVE) {
    launch_csc_naive_pairs(a, h->cs, col_group(h), (int*)h->sk, (float*)h->sv, st);
  } else {
    launch_csc_lb(a, h->cs, variant == SPMX_CSC_LB_MERGE ? 1 : 2, nullptr, (int*)h->sk,
                  (float*)h->sv, h->lb_grid, st);
  }
  RadixBuffers rb{h->sk, h->sk_alt, h->sv, h->sv_alt, nullptr, nullptr, h->shist, h->shist_off, false};
  if (radix_sort_pairs(rb, bin_len, ceil_log2(std::max(h->m, 2)), h->ls, h->d_err, st))
    return set_error(SPMX_ERR_INVALID_VALUE, "radix capacity");
  const unsigned* keys = rb.result_in_alt ? h->sk_alt : h->sk;
  const float* vals = (const float*)(rb.result_in_alt ? h->sv_alt : h->sv);
  int* ok = ykey ? ykey : h->sy_key;
  float* ov = yval ? yval : h->sy_val;
  if (reduce_by_key_sorted(keys, vals, bin_len, h->sslot, ok, ov, h->d_counts + kCntYnnz, h->ls,
                           h->d_err, st))
    return set_error(SPMX_ERR_INVALID_VALUE, "reduce capacity");
  SPMX_TRY(launch_ok("csc sort spmspv"));
  int cnt = 0;
  if (ynnz || y) SPMX_TRY(read_counter(h, kCntYnnz, &cnt));
  if (ynnz) *ynnz = cnt;
  if (y) {
    SPMX_CUDA(cudaMemsetAsync(y, 0, 4 * (size_t)h->m, st));
    launch_scatter(cnt, h->m, ok, ov, y, nullptr, h->d_err, st);
    SPMX_TRY(launch_ok("csc sort scatter"));
  }
  return SPMX_SUCCESS;
}

extern "C" int spmx_spmspv_csc(spmx_handle_t h, int variant, int writeback, float alpha,
                               float* y, int* ykey, float* yval, int* ynnz) {
  SPMX_CHECK_HANDLE(h);
  if (!h->has_csc || !h->csc_val)
    return set_error(SPMX_ERR_NOT_READY, "CSC SpMSpV needs the CSC with values (ToCSC / InputCSC)");
  if (variant < SPMX_CSC_NAIVE || variant > SPMX_CSC_BUCKET)
    return set_error(SPMX_ERR_INVALID_VALUE, "bad CSC variant");
  if (writeback != SPMX_WB_ATOMIC && writeback != SPMX_WB_SORT)
    return set_error(SPMX_ERR_INVALID_VALUE, "bad write-back");
  if (h->x_nnz > 0 && (!h->x_key || !h->x_val)) return set_error(SPMX_VEC_FORMAT_ERR, "no sparse x");
  const bool sparse_out = ykey && yval;
  if (writeback == SPMX_WB_ATOMIC && !y && h->m > 0 && variant != SPMX_CSC_BUCKET)
    return set_error(SPMX_ERR_INVALID_VALUE, "atomic write-back needs the dense y");
  if (writeback == SPMX_WB_SORT && !sparse_out && !y)
    return set_error(SPMX_ERR_INVALID_VALUE, "sort write-back needs y_key/y_val or y");
  if (h->x_nnz == 0) {
    if (y && h->m > 0) SPMX_CUDA(cudaMemsetAsync(y, 0, 4 * (size_t)h->m, h->stream));
    SPMX_CUDA(cudaMemsetAsync(h->d_counts + kCntYnnz, 0, sizeof(int), h->stream));
    SPMX_CUDA(cudaMemsetAsync(h->d_counts + kCntBinlen, 0, sizeof(int), h->stream));
    if (ynnz) *ynnz = 0;
    return SPMX_SUCCESS;
  }
  if (variant == SPMX_CSC_BUCKET) return csc_bucket_impl(h, alpha, y, ykey, yval, ynnz, 0);
  if (writeback == SPMX_WB_ATOMIC) return csc_atomic(h, variant, alpha, y, ykey, yval, ynnz);
  return csc_sort(h, variant, alpha, y, ykey, yval, ynnz);
}

extern "C" int spmx_csc_naive_atomic(spmx_handle_t h, float alpha, int* ynnz, float* y) {
  return spmx_spmspv_csc(h, SPMX_CSC_NAIVE, SPMX_WB_ATOMIC, alpha, y, nullptr, nullptr, ynnz);
}
extern "C" int spmx_csc_naive_atomic_keyval(spmx_handle_t h, float alpha, int* ynnz, float* y,
                                            int* ykey, float* yval) {
  return spmx_spmspv_csc(h, SPMX_CSC_NAIVE, SPMX_WB_ATOMIC, alpha, y, ykey, yval, ynnz);
}
extern "C" int spmx_csc_naive_sort(spmx_handle_t h, float alpha, int* ynnz, int* ykey,
                                   float* yval) {
  return spmx_spmspv_csc(h, SPMX_CSC_NAIVE, SPMX_WB_SORT, alpha, nullptr, ykey, yval, ynnz);
}
extern "C" int spmx_csc_merge_atomic(spmx_handle_t h, int, float alpha, int* ynnz, float* y,
                                     int*, float*) {
  return spmx_spmspv_csc(h, SPMX_CSC_LB_MERGE, SPMX_WB_ATOMIC, alpha, y, nullptr, nullptr, ynnz);
}
extern "C" int spmx_csc_merge_atomic_keyval(spmx_handle_t h, int, float alpha, int* ynnz,
                                            float* y, int* ykey, float* yval) {
  return spmx_spmspv_csc(h, SPMX_CSC_LB_MERGE, SPMX_WB_ATOMIC, alpha, y, ykey, yval, ynnz);
}
extern "C" int spmx_csc_merge_sort(spmx_handle_t h, int, float alpha, int* ynnz, float* y,
                                   int* ykey, float* yval) {
  return spmx_spmspv_csc(h, SPMX_CSC_LB_MERGE, SPMX_WB_SORT, alpha, y, ykey, yval, ynnz);
}
extern "C" int spmx_csc_twolayer_atomic(spmx_handle_t h, int, float alpha, int* ynnz, float* y,
                                        int*, float*) {
  return spmx_spmspv_csc(h, SPMX_CSC_LB_TWOLAYER, SPMX_WB_ATOMIC, alpha, y, nullptr, nullptr, ynnz);
}
extern "C" int spmx_csc_twolayer_atomic_keyval(spmx_handle_t h, int, float alpha, int* ynnz,
                                               float* y, int* ykey, float* yval) {
  return spmx_spmspv_csc(h, SPMX_CSC_LB_TWOLAYER, SPMX_WB_ATOMIC, alpha, y, ykey, yval, ynnz);
}
extern "C" int spmx_csc_twolayer_sort(spmx_handle_t h, int, float alpha, int* ynnz, float* y,
                                      int* ykey, float* yval) {
  return spmx_spmspv_csc(h, SPMX_CSC_LB_TWOLAYER, SPMX_WB_SORT, alpha, y, ykey, yval, ynnz);
}
extern "C" int spmx_csc_bucket(spmx_handle_t h, float alpha, int* ynnz, float* y, int* ykey,
                               float* yval, int buckets) {
  SPMX_CHECK_HANDLE(h);
  if (!h->has_csc || !h->csc_val)
    return set_error(SPMX_ERR_NOT_READY, "CSC SpMSpV needs the CSC with values");
  if (h->x_nnz == 0) return spmx_spmspv_csc(h, SPMX_CSC_BUCKET, SPMX_WB_SORT, alpha, y, ykey, yval, ynnz);
  return csc_bucket_impl(h, alpha, y, ykey, yval, ynnz, buckets);
}

// ---------------------------------------------------------------------------
// bucket-based CSC SpMSpV
// ---------------------------------------------------------------------------
int csc_bucket_impl(spmx_handle_t h, float alpha, float* y, int* ykey, float* yval,
                    int* ynnz, int buckets) {
  SPMX_TRY(ensure_csc_scratch(h));
  SPMX_TRY(ensure_sort_scratch(h));
  int rshift = 0, nb = 0;
  if (bucket_geometry(h->m, buckets > 0 ? buckets : h->buckets, &rshift, &nb))
    return set_error(SPMX_ERR_INVALID_VALUE, "too many rows for the bucket method");
  SPMX_TRY(ensure_scan_tiles(h, nb));
  cudaStream_t st = h->stream;
  const CscArgs a = csc_args(h, alpha);
  if (launch_csc_scan(a, h->cs, h->ls, kCscLbNT * kCscLbVT, st))
    return set_error(SPMX_ERR_INVALID_VALUE, "scan capacity");
  BucketScratch bs{h->bk_gcount, h->bk_boff, h->bk_cursor, (int*)h->sk, (float*)h->sv, h->nnz};
  if (launch_bucket_spmspv(a, h->cs, bs, SPMX_CSC_LB_MERGE, rshift, nb, y, ykey, yval,
                           h->d_counts + kCntYnnz, h->ls, h->lb_grid, st))
    return set_error(SPMX_ERR_INVALID_VALUE, "bucket launch capacity");
  SPMX_TRY(launch_ok("bucket spmspv"));
  if (ynnz) SPMX_TRY(read_counter(h, kCntYnnz, ynnz));
  return SPMX_SUCCESS;
}
