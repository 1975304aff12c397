// Per-matrix autotuner (no reference counterpart; the reference picks between
// Hola and CSR5 SpMV by timing both in its data generator,
// TEST/generate_model_data.cu:487-516).  spmx_autotune times the candidates
// of every tunable choice on the handle's matrix with CUDA events and keeps
// the fastest:
//   - the load-balanced SpMV back-end: Hola (4, 8 or 16 nonzeros per thread),
//     CSR5 (sigma: the reference's rule or 4, 8, 16, 32 nonzeros per lane),
//     tiled (x window width) or round;
//   - the lanes per row of the naive CSR kernel and per column of the naive
//     CSC kernel;
//   - merge-path vs fixed-nonzero blocks for the load-balanced CSC kernel;
//   - the bucket count of the bucket kernel.
// Results can be cached in a small text file keyed by a fingerprint of the
// matrix (m, n, nnz and a sample of the row pointer), so a second process
// applies them without timing.
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "kernels.h"

using namespace spmx;

namespace {

__global__ void fill_kernel(float* x, int n, float v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = v;
}

// k distinct sorted keys, one at a hashed offset inside each of k equal
// buckets of [0, n): irregular like a random sparse x (evenly strided keys made
// the column-bound loads regular and the lanes-per-column choice flip between
// 16 and 32 from one GPU to the next, while random keys favour 32 clearly)
__global__ void stride_keys_kernel(int* key, float* val, int k, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < k) {
    const long long b0 = ((long long)i * n) / k, b1 = ((long long)(i + 1) * n) / k;
    unsigned hsh = (unsigned)i * 2654435761u;
    hsh ^= hsh >> 15;
    hsh *= 2246822519u;
    hsh ^= hsh >> 13;
    key[i] = (int)(b0 + (b1 > b0 ? hsh % (unsigned)(b1 - b0) : 0u));
    val[i] = 1.0f;
  }
}

struct Params {
  int spmv_type = SPMX_SPMV_HOLA, hola_vt = 8, tiled_rb = 0, tiled_win = 8192;
  int row_group = 0, col_group = 0, lb_variant = SPMX_CSC_LB_MERGE, buckets = 256;
  int csr5_sigma = -1;  // -1: the reference's rule
};

unsigned long long fingerprint(spmx_handle_t h) {
  // m, n, nnz and 64 row-pointer samples, FNV-1a
  unsigned long long f = 1469598103934665603ULL;
  auto mix = [&](unsigned long long v) { f = (f ^ v) * 1099511628211ULL; };
  mix((unsigned long long)h->m);
  mix((unsigned long long)h->n);
  mix((unsigned long long)h->nnz);
  if (h->has_csr && h->m > 0) {
    std::vector<int> s(64);
    for (int i = 0; i < 64; ++i) {
      const long long r = ((long long)i * h->m) / 63;
      cudaMemcpy(&s[i], h->rowptr + r, sizeof(int), cudaMemcpyDeviceToHost);
      mix((unsigned long long)(unsigned)s[i]);
    }
  }
  return f;
}

bool cache_lookup(const char* path, unsigned long long fp, Params* p) {
  if (!path) return false;
  FILE* f = fopen(path, "r");
  if (!f) return false;
  char line[512];
  bool found = false;
  while (fgets(line, sizeof(line), f)) {
    unsigned long long k = 0;
    Params q;
    // 10 fields; lines written before CSR5 sigma was tuned have 9
    const int got = sscanf(line, "%llx %d %d %d %d %d %d %d %d %d", &k, &q.spmv_type, &q.hola_vt,
                           &q.tiled_rb, &q.tiled_win, &q.row_group, &q.col_group, &q.lb_variant,
                           &q.buckets, &q.csr5_sigma);
    if (got == 9) q.csr5_sigma = -1;
    if (got >= 9 && k == fp) {
      *p = q;
      found = true;
    }
  }
  fclose(f);
  return found;
}

void cache_store(const char* path, unsigned long long fp, const Params& q) {
  if (!path) return;
  FILE* f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "%llx %d %d %d %d %d %d %d %d %d\n", fp, q.spmv_type, q.hola_vt, q.tiled_rb, q.tiled_win,
          q.row_group, q.col_group, q.lb_variant, q.buckets, q.csr5_sigma);
  fclose(f);
}

}  // namespace

extern "C" int spmx_csc_bucket(spmx_handle_t h, float alpha, int* ynnz, float* y, int* ykey,
                               float* yval, int buckets);

static int apply_params(spmx_handle_t h, const Params& p) {
  h->naive_row_group = p.row_group;
  h->naive_col_group = p.col_group;
  h->lb_variant = p.lb_variant;
  h->buckets = p.buckets;
  h->spmv_type = p.spmv_type;
  int rc = SPMX_SUCCESS;
  if (p.spmv_type == SPMX_SPMV_HOLA && h->has_csr) {
    if (!h->hola_ready || h->hola_vt != p.hola_vt) {
      h->hola_vt = p.hola_vt;
      rc = spmx_hola_preprocess(h);
    }
  } else if (p.spmv_type == SPMX_SPMV_CSR5) {
    if (!h->csr5 || h->sigma != p.csr5_sigma) {
      spmx_csr5_postprocess(h);
      h->sigma = p.csr5_sigma;
      rc = spmx_csr5_preprocess(h);
    }
  } else if (p.spmv_type == SPMX_SPMV_TILED) {
    rc = spmx_tiled_preprocess(h, p.tiled_rb, p.tiled_win, 0, 0);
  } else if (p.spmv_type == SPMX_SPMV_ROUND) {
    // for the round back-end the window field holds the CTAs per row block
    rc = spmx_round_preprocess_parts(h, p.tiled_rb, p.tiled_win == 1 || p.tiled_win == 4 ? p.tiled_win : 2);
  }
  return rc;
}

extern "C" int spmx_set_naive_lanes(spmx_handle_t h, int row_lanes, int col_lanes) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  auto ok = [](int g) { return g == 0 || g == 1 || g == 2 || g == 4 || g == 8 || g == 16 || g == 32; };
  if (!ok(row_lanes) || !ok(col_lanes))
    return set_error(SPMX_ERR_INVALID_VALUE, "lanes must be 0, 1, 2, 4, 8, 16 or 32");
  h->naive_row_group = row_lanes;
  h->naive_col_group = col_lanes;
  return SPMX_SUCCESS;
}

extern "C" int spmx_autotune(spmx_handle_t h, const char* cache_path, int* spmv_type_out) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  if (!h->has_csr || (!h->val && h->nnz > 0))
    return set_error(SPMX_ERR_NOT_READY, "autotune needs the CSR input with values");
  const unsigned long long fp = fingerprint(h);
  Params best;
  if (cache_lookup(cache_path, fp, &best)) {
    const int rc = apply_params(h, best);
    if (spmv_type_out) *spmv_type_out = best.spmv_type;
    return rc;
  }
  cudaStream_t st = h->stream;
  const int m = h->m, n = h->n;
  float *x = nullptr, *y = nullptr, *xval = nullptr;
  int* xkey = nullptr;
  int rc = SPMX_SUCCESS;
  rc = rc ? rc : dalloc((void**)&x, 4 * (size_t)std::max(n, 1), "tune x");
  rc = rc ? rc : dalloc((void**)&y, 4 * (size_t)std::max(m, 1), "tune y");
  const int k = std::max(1, n / 10);
  rc = rc ? rc : dalloc((void**)&xkey, 4 * (size_t)k, "tune x keys");
  rc = rc ? rc : dalloc((void**)&xval, 4 * (size_t)k, "tune x vals");
  // a buffer twice the size of L2, written before every timed run: timed
  // back to back, repeated calls found their inputs in L2, and the lanes per
  // column picked that way (16 on this 1M-column matrix) were 17 % slower on
  // the cold data a call normally meets than the lanes picked cold (32)
  int l2 = 0, dev = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev) != cudaSuccess) {
    cudaGetLastError();
    l2 = 0;
  }
  const long long flush_n = std::max<long long>(1, 2LL * l2 / 4);
  float* flush = nullptr;
  rc = rc ? rc : dalloc((void**)&flush, 4 * (size_t)flush_n, "tune L2 flush");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float* saved_x = h->x_dense;
  int* saved_key = h->x_key;
  float* saved_val = h->x_val;
  const int saved_xnnz = h->x_nnz;
  if (!rc) {
    note_launch(2);
    fill_kernel<<<(std::max(n, 1) + 255) / 256, 256, 0, st>>>(x, n, 0.5f);
    stride_keys_kernel<<<(k + 255) / 256, 256, 0, st>>>(xkey, xval, k, n);
    h->x_dense = x;
  }
  // median of 5 timed runs after 2 warm-ups
  auto time_us = [&](auto&& fn) -> float {
    std::vector<float> ts;
    for (int it = 0; it < 7; ++it) {
      note_launch();
      fill_kernel<<<(unsigned)std::min<long long>((flush_n + 255) / 256, 4096), 256, 0, st>>>(
          flush, (int)std::min<long long>(flush_n, INT_MAX), (float)it);
      cudaEventRecord(e0, st);
      const int r = fn();
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      if (r != SPMX_SUCCESS) return 1e30f;
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (it >= 2) ts.push_back(ms * 1e3f);
    }
    std::sort(ts.begin(), ts.end());
    return ts[ts.size() / 2];
  };
  float best_t = 1e30f;
  if (!rc && h->nnz > 0) {
    // load-balanced SpMV back-ends
    for (int vt : {4, 8, 16}) {
      h->hola_vt = vt;
      if (spmx_hola_preprocess(h) != SPMX_SUCCESS) continue;
      const float t = time_us([&] { return spmx_holaspmv(h, 1.0f, y); });
      if (t < best_t) { best_t = t; best.spmv_type = SPMX_SPMV_HOLA; best.hola_vt = vt; }
    }
    const int saved_sigma = h->sigma;
    for (int sg : {-1, 4, 8, 16, 32}) {
      spmx_csr5_postprocess(h);
      h->sigma = sg;
      if (spmx_csr5_preprocess(h) != SPMX_SUCCESS) continue;
      const float t = time_us([&] { return spmx_csr5spmv(h, 1.0f, y); });
      if (t < best_t) { best_t = t; best.spmv_type = SPMX_SPMV_CSR5; best.csr5_sigma = sg; }
    }
    spmx_csr5_postprocess(h);
    h->sigma = saved_sigma;
    for (int win : {4096, 8192}) {
      const int rb = 0;  // rows per block: as many as shared memory holds
      if (spmx_tiled_preprocess(h, rb, win, 0, 0) != SPMX_SUCCESS) continue;
      const float t = time_us([&] { return spmx_tiledspmv(h, 1.0f, y); });
      if (t < best_t) {
        best_t = t;
        best.spmv_type = SPMX_SPMV_TILED;
        best.tiled_rb = rb;
        best.tiled_win = win;
      }
      spmx_tiled_postprocess(h);
    }
    // round back-end with 1, 2 or 4 CTAs per row block (a build that does
    // not fit shared memory is skipped)
    for (int parts : {1, 2, 4}) {
      if (spmx_round_preprocess_parts(h, 0, parts) != SPMX_SUCCESS) continue;
      const float t = time_us([&] { return spmx_roundspmv(h, 1.0f, y); });
      if (t < best_t) {
        best_t = t;
        best.spmv_type = SPMX_SPMV_ROUND;
        best.tiled_rb = 0;
        best.tiled_win = parts;
      }
      spmx_round_postprocess(h);
    }
    // naive CSR lanes per row
    float bt = 1e30f;
    for (int g : {1, 2, 4, 8, 16, 32}) {
      h->naive_row_group = g;
      const float t = time_us([&] { return spmx_naivespmv(h, 1.0f, y); });
      if (t < bt) { bt = t; best.row_group = g; }
    }
    if (h->has_csc && h->csc_val) {
      h->x_key = xkey;
      h->x_val = xval;
      h->x_nnz = k;
      bt = 1e30f;
      for (int g : {1, 2, 4, 8, 16, 32}) {
        h->naive_col_group = g;
        const float t = time_us([&] {
          return spmx_spmspv_csc(h, SPMX_CSC_NAIVE, SPMX_WB_ATOMIC, 1.0f, y, nullptr, nullptr, nullptr);
        });
        if (t < bt) { bt = t; best.col_group = g; }
      }
      bt = 1e30f;
      for (int v : {SPMX_CSC_LB_MERGE, SPMX_CSC_LB_TWOLAYER}) {
        const float t = time_us([&] {
          return spmx_spmspv_csc(h, v, SPMX_WB_ATOMIC, 1.0f, y, nullptr, nullptr, nullptr);
        });
        if (t < bt) { bt = t; best.lb_variant = v; }
      }
      bt = 1e30f;
      for (int b : {64, 256, 1024}) {
        const float t = time_us([&] { return spmx_csc_bucket(h, 1.0f, nullptr, y, nullptr, nullptr, b); });
        if (t < bt) { bt = t; best.buckets = b; }
      }
    }
  }
  h->x_dense = saved_x;
  h->x_key = saved_key;
  h->x_val = saved_val;
  h->x_nnz = saved_xnnz;
  cudaStreamSynchronize(st);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dfree(x);
  dfree(y);
  dfree(xkey);
  dfree(xval);
  dfree(flush);
  if (rc) return rc;
  rc = apply_params(h, best);
  if (!rc) cache_store(cache_path, fp, best);
  if (spmv_type_out) *spmv_type_out = best.spmv_type;
  return rc;
}
