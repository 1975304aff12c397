// Tiled SpMV / bitmap-gated SpMSpV (y = alpha * A * x): a third load-balanced
// back-end beside Hola and CSR5 (spmv_type 2).
//
// Why: with uniformly random columns every nonzero of a row-ordered SpMV
// gathers x through L2 one 32-byte sector at a time; on B200 that caps a
// 1M-column, 16.8M-nonzero SpMV at about 68 us whatever the kernel does
// (measured with a bare gather loop).  Tiling the matrix into row blocks of
// RB rows x column windows of W columns makes every CTA's x accesses fall
// in one W-column window that stays in its SM's L1, so each x sector leaves
// L2 once per tile instead of once per nonzero.  y of the current row block
// accumulates in shared memory (shared atomics) and is added to the global y
// with coalesced atomics whenever the CTA moves to another row block.
//
// Format (built on the device by spmx_tiled_preprocess): nonzeros sorted by
// tile (row block major, window minor), stable inside a tile; per nonzero one
// packed word (local row in the low 16 bits, local column in the high 16
// bits) and the value; tiles cut into chunks of at most `chunk` nonzeros,
// and each CTA of a persistent grid owns a contiguous run of chunks with an
// (almost) equal nonzero count.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "feat.h"
#include "kernels.h"
#include "sort.h"

namespace spmx {

struct TiledChunk {
  int tile;   // row block * nwin + window
  int begin;  // first nonzero (in tiled order)
  int end;
};

template <int NT, bool GATED>
__global__ void __launch_bounds__(NT)
tiled_spmv_kernel(int m, int n, int rb_rows, int win, int nwin,
                  const unsigned* __restrict__ packed, const float* __restrict__ val,
                  const TiledChunk* __restrict__ chunks, const int* __restrict__ cta_first,
                  const float* __restrict__ x, const unsigned* __restrict__ xbits,
                  float alpha, float* __restrict__ y, int* err) {
  extern __shared__ float ys[];
  const int c0 = __ldg(cta_first + blockIdx.x), c1 = __ldg(cta_first + blockIdx.x + 1);
  for (int r = threadIdx.x; r < rb_rows; r += NT) ys[r] = 0.f;
  __syncthreads();
  int cur_rb = -1;
  for (int c = c0; c < c1; ++c) {
    const TiledChunk ch = chunks[c];
    const int rb = ch.tile / nwin, w = ch.tile - rb * nwin;
    if (rb != cur_rb) {
      if (cur_rb >= 0) {
        __syncthreads();
        const int base = cur_rb * rb_rows;
        const int rows = min(rb_rows, m - base);
        for (int r = threadIdx.x; r < rows; r += NT) {
          const float v = ys[r];
          if (v != 0.f) atomicAdd(y + base + r, alpha * v);
          ys[r] = 0.f;
        }
        __syncthreads();
      }
      cur_rb = rb;
    }
    const int cbase = w * win;
#pragma unroll 4
    for (int k = ch.begin + (int)threadIdx.x; k < ch.end; k += NT) {
      const unsigned p = __ldg(packed + k);
      const int lr = (int)(p & 0xffffu), lc = (int)(p >> 16);
      const int col = cbase + lc;
      if ((unsigned)col >= (unsigned)n || lr >= rb_rows) { flag_error(err, kDevErrOob); continue; }
      if (GATED && !((__ldg(xbits + (col >> 5)) >> (col & 31)) & 1u)) continue;
      atomicAdd(&ys[lr], __ldg(val + k) * __ldg(x + col));
    }
  }
  __syncthreads();
  if (cur_rb >= 0) {
    const int base = cur_rb * rb_rows;
    const int rows = min(rb_rows, m - base);
    for (int r = threadIdx.x; r < rows; r += NT) {
      const float v = ys[r];
      if (v != 0.f) atomicAdd(y + base + r, alpha * v);
    }
  }
}

// pack the tile key, local coordinates and value of every nonzero (CSR order)
__global__ void tiled_keys_kernel(int m, int nnz, const int* __restrict__ rowptr,
                                  const int* __restrict__ col, const float* __restrict__ val,
                                  int rb_shift, int win_shift, int nwin, unsigned* __restrict__ key,
                                  unsigned* __restrict__ packed, float* __restrict__ v_out) {
  // one warp per row
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= m) return;
  const int r = (int)gw;
  const int a = __ldg(rowptr + r), b = __ldg(rowptr + r + 1);
  const unsigned rb = (unsigned)(r >> rb_shift), lr = (unsigned)(r & ((1 << rb_shift) - 1));
  for (int k = a + lane; k < b; k += 32) {
    const int c = __ldg(col + k);
    const unsigned w = (unsigned)(c >> win_shift), lc = (unsigned)(c & ((1 << win_shift) - 1));
    key[k] = rb * (unsigned)nwin + w;
    packed[k] = lr | (lc << 16);
    v_out[k] = __ldg(val + k);
  }
}

}  // namespace spmx

using namespace spmx;

struct TiledTables {
  int rb_shift = 0, win_shift = 0, nwin = 0, nrb = 0, nchunks = 0, grid = 0, nt = 512;
  unsigned* packed = nullptr;
  float* val = nullptr;
  TiledChunk* chunks = nullptr;
  int* cta_first = nullptr;
};

static TiledTables* ttab(spmx_handle_t h) { return reinterpret_cast<TiledTables*>(h->tiled); }

extern "C" int spmx_tiled_postprocess(spmx_handle_t h) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  TiledTables* t = ttab(h);
  if (t) {
    cudaStreamSynchronize(h->stream);
    dfree(t->packed); dfree(t->val); dfree(t->chunks); dfree(t->cta_first);
    delete t;
    h->tiled = nullptr;
  }
  return SPMX_SUCCESS;
}

static int log2_ceil(long long v) {
  int b = 0;
  while ((1LL << b) < v) ++b;
  return b;
}

// rows per block (<= 32768, in shared memory) and columns per window
// (<= 65536, meant to stay in L1): rb_rows and win are powers of two
extern "C" int spmx_tiled_preprocess(spmx_handle_t h, int rb_rows, int win, int chunk) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  if (!h->has_csr || (!h->val && h->nnz > 0))
    return set_error(SPMX_ERR_NOT_READY, "tiled SpMV needs the CSR input with values");
  if (rb_rows <= 0) rb_rows = 16384;
  if (win <= 0) win = 16384;
  if (chunk <= 0) chunk = 8192;
  if ((rb_rows & (rb_rows - 1)) || rb_rows > 32768 || (win & (win - 1)) || win > 65536 ||
      chunk < 256)
    return set_error(SPMX_ERR_INVALID_VALUE,
                     "tiled SpMV: rb_rows (<= 32768) and win (<= 65536) must be powers of two");
  spmx_tiled_postprocess(h);
  TiledTables* t = new TiledTables();
  h->tiled = t;
  const int m = h->m, n = h->n, nnz = h->nnz;
  t->rb_shift = log2_ceil(rb_rows);
  t->win_shift = log2_ceil(win);
  t->nwin = std::max(1, (n + win - 1) / win);
  t->nrb = std::max(1, (m + rb_rows - 1) / rb_rows);
  const long long ntiles = (long long)t->nrb * t->nwin;
  if (ntiles > (1LL << 30)) {
    spmx_tiled_postprocess(h);
    return set_error(SPMX_ERR_INVALID_VALUE, "tiled SpMV: too many tiles");
  }
  cudaStream_t st = h->stream;
  const size_t b = 4 * (size_t)std::max(nnz, 1);
  unsigned *k0 = nullptr, *k1 = nullptr, *p0 = nullptr, *p1 = nullptr, *v0 = nullptr, *v1 = nullptr;
  int *hist = nullptr, *hoff = nullptr, *cnt = nullptr, *tptr = nullptr;
  const size_t hn = radix_hist_ints(std::max(nnz, 1));
  int rc = SPMX_SUCCESS;
  rc = rc ? rc : dalloc((void**)&k0, b, "tiled keys");
  rc = rc ? rc : dalloc((void**)&k1, b, "tiled keys alt");
  rc = rc ? rc : dalloc((void**)&p0, b, "tiled packed");
  rc = rc ? rc : dalloc((void**)&p1, b, "tiled packed alt");
  rc = rc ? rc : dalloc((void**)&v0, b, "tiled vals");
  rc = rc ? rc : dalloc((void**)&v1, b, "tiled vals alt");
  rc = rc ? rc : dalloc((void**)&hist, 4 * hn, "tiled hist");
  rc = rc ? rc : dalloc((void**)&hoff, 4 * hn, "tiled hist off");
  rc = rc ? rc : dalloc((void**)&cnt, 4 * (size_t)ntiles, "tiled counts");
  rc = rc ? rc : dalloc((void**)&tptr, 4 * (size_t)(ntiles + 1), "tiled pointers");
  std::vector<int> htp((size_t)ntiles + 1, 0);
  if (!rc && nnz > 0) {
    note_launch();
    tiled_keys_kernel<<<(unsigned)(((long long)m * 32 + 255) / 256), 256, 0, st>>>(
        m, nnz, h->rowptr, h->col, h->val, t->rb_shift, t->win_shift, t->nwin, k0, p0, (float*)v0);
    RadixBuffers rb{k0, k1, p0, p1, v0, v1, hist, hoff, false};
    if (radix_sort_pairs(rb, nnz, std::max(1, log2_ceil(ntiles)), h->ls, h->d_err, st))
      rc = set_error(SPMX_ERR_INVALID_VALUE, "tiled SpMV: sort capacity");
    if (!rc) {
      unsigned* ks = rb.result_in_alt ? k1 : k0;
      cudaMemsetAsync(cnt, 0, 4 * (size_t)ntiles, st);
      launch_count_keys(nnz, (int)ntiles, (const int*)ks, cnt, h->d_err, st);
      if (launch_scan_exclusive(cnt, tptr, (int)ntiles, tptr + ntiles, h->ls, h->d_err, st))
        rc = set_error(SPMX_ERR_INVALID_VALUE, "tiled SpMV: scan capacity");
      // keep the sorted payloads: swap them into the table
      t->packed = rb.result_in_alt ? p1 : p0;
      t->val = (float*)(rb.result_in_alt ? v1 : v0);
      if (rb.result_in_alt) { p1 = nullptr; v1 = nullptr; } else { p0 = nullptr; v0 = nullptr; }
      if (!rc && cudaMemcpyAsync(htp.data(), tptr, 4 * (size_t)(ntiles + 1), cudaMemcpyDeviceToHost,
                                 st) != cudaSuccess)
        rc = set_error(SPMX_ERR_CUDA, "tiled SpMV: tile pointers");
    }
  }
  const cudaError_t se = cudaStreamSynchronize(st);
  dfree(k0); dfree(k1); dfree(p0); dfree(p1); dfree(v0); dfree(v1);
  dfree(hist); dfree(hoff); dfree(cnt); dfree(tptr);
  if (!rc && se != cudaSuccess) rc = set_error(SPMX_ERR_CUDA, cudaGetErrorString(se));
  if (rc) { spmx_tiled_postprocess(h); return rc; }
  // chunks of at most `chunk` nonzeros inside a tile, then equal-nonzero runs
  std::vector<TiledChunk> ch;
  for (long long tt = 0; tt < ntiles; ++tt)
    for (int s0 = htp[tt]; s0 < htp[tt + 1]; s0 += chunk)
      ch.push_back(TiledChunk{(int)tt, s0, std::min(s0 + chunk, htp[tt + 1])});
  int occ = 2;
  t->nt = 512;
  {
    int bps = 0;
    const int smem = 4 << t->rb_shift;
    cudaFuncSetAttribute(tiled_spmv_kernel<512, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(tiled_spmv_kernel<512, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, tiled_spmv_kernel<512, false>, 512, smem) ==
            cudaSuccess && bps > 0)
      occ = bps;
    cudaGetLastError();
  }
  const int grid = std::max(1, std::min((int)ch.size(), h->num_sms * occ));
  std::vector<int> first(grid + 1, 0);
  // split the chunk list into `grid` runs of about nnz / grid nonzeros
  {
    long long acc = 0;
    int g = 1;
    const double per = (double)std::max(nnz, 1) / grid;
    for (size_t i = 0; i < ch.size() && g < grid; ++i) {
      acc += ch[i].end - ch[i].begin;
      while (g < grid && acc >= per * g) first[g++] = (int)i + 1;
    }
    while (g < grid) first[g++] = (int)ch.size();
    first[grid] = (int)ch.size();
  }
  t->nchunks = (int)ch.size();
  t->grid = grid;
  rc = dalloc((void**)&t->chunks, sizeof(TiledChunk) * std::max<size_t>(ch.size(), 1), "tiled chunks");
  rc = rc ? rc : dalloc((void**)&t->cta_first, 4 * (size_t)(grid + 1), "tiled cta runs");
  if (!rc && !ch.empty())
    if (cudaMemcpy(t->chunks, ch.data(), sizeof(TiledChunk) * ch.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      rc = set_error(SPMX_ERR_CUDA, "tiled chunks upload");
  if (!rc && cudaMemcpy(t->cta_first, first.data(), 4 * (size_t)(grid + 1), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = set_error(SPMX_ERR_CUDA, "tiled runs upload");
  if (rc) { spmx_tiled_postprocess(h); return rc; }
  return SPMX_SUCCESS;
}

int tiled_spmv_impl(spmx_handle_t h, float alpha, float* y, bool gated) {
  TiledTables* t = ttab(h);
  if (!t) return set_error(SPMX_ERR_NOT_READY, "call spmx_tiled_preprocess first");
  if (!h->x_dense) return set_error(SPMX_VEC_FORMAT_ERR, "tiled SpMV needs the dense x");
  if (gated && !h->bitvec) return set_error(SPMX_VEC_FORMAT_ERR, "tiled SpMSpV needs the bitarray");
  if (!y && h->m > 0) return set_error(SPMX_ERR_INVALID_VALUE, "y is NULL");
  cudaStream_t st = h->stream;
  if (h->m == 0) return SPMX_SUCCESS;
  cudaMemsetAsync(y, 0, 4 * (size_t)h->m, st);
  if (t->nchunks == 0) return SPMX_SUCCESS;
  const int smem = 4 << t->rb_shift;
  note_launch();
  if (gated)
    tiled_spmv_kernel<512, true><<<t->grid, 512, smem, st>>>(
        h->m, h->n, 1 << t->rb_shift, 1 << t->win_shift, t->nwin, t->packed, t->val, t->chunks,
        t->cta_first, h->x_dense, (const unsigned*)h->bitvec, alpha, y, h->d_err);
  else
    tiled_spmv_kernel<512, false><<<t->grid, 512, smem, st>>>(
        h->m, h->n, 1 << t->rb_shift, 1 << t->win_shift, t->nwin, t->packed, t->val, t->chunks,
        t->cta_first, h->x_dense, nullptr, alpha, y, h->d_err);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(SPMX_ERR_CUDA, std::string("tiled spmv: ") + cudaGetErrorString(e));
  return SPMX_SUCCESS;
}

extern "C" int spmx_tiledspmv(spmx_handle_t h, float alpha, float* y) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  return tiled_spmv_impl(h, alpha, y, false);
}

extern "C" int spmx_tiledspmspv(spmx_handle_t h, float alpha, float* y) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  return tiled_spmv_impl(h, alpha, y, true);
}
