// CSR5-style SpMV / bitmap-gated SpMSpV (y = alpha * A * x).
//
// Replaces csr5_spmv / csr5_spmspv (DEV/csr5_spmv_cuda.h:440-582,
// DEV/csr5_spmspv.h:450-611) and the CSR->CSR5 conversion
// (DEV/format_conversion.h:112-718, CSR5Preprocess H:1426-1582).  Kept from
// CSR5: tiles of omega x sigma nonzeros (omega = 32 lanes, sigma from the
// reference's auto rule, H:1396-1416), column-major ("transposed") storage
// inside a tile so that a warp's loads are coalesced, one row-start bit flag
// per nonzero, and a warp-level segmented sum.  Our own choices:
//   - the user's CSR is not permuted in place (the reference transposes the
//     caller's arrays and transposes them back in CSR5Postprocess); the tile
//     copies belong to the handle;
//   - rows are addressed through the list of non-empty rows and a per-lane
//     rank, so empty rows need no per-tile offset table; the lane that opens
//     a row also zeroes the empty rows just before it;
//   - the last tile is zero-padded, so there is no separate tail kernel;
//   - sums are FP64 (exact products, prefix differences across lanes) and a
//     row crossing tiles is finished by the last tile to arrive, which adds
//     the per-tile partials in tile order (deterministic, no zero-fill of y,
//     no calibrate kernel).
#include <algorithm>

#include "common.cuh"
#include "engine.h"
#include "kernels.h"
#include "sort.h"

namespace spmx {

// ---- preprocess -----------------------------------------------------------
__global__ void nonempty_flag_kernel(int m, const int* __restrict__ rowptr, int* flag) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < m) flag[r] = __ldg(rowptr + r + 1) > __ldg(rowptr + r);
}

__global__ void nonempty_list_kernel(int m, const int* __restrict__ rowptr,
                                     const int* __restrict__ rank, int* nz_rows) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < m && __ldg(rowptr + r + 1) > __ldg(rowptr + r)) nz_rows[__ldg(rank + r)] = r;
}

// one thread per (tile, lane): row-start bit flags, the rank of the row
// holding the lane's first element, and the transposed copies of col / val
__global__ void csr5_tiles_kernel(int m, int nnz, int sigma, int ntiles,
                                  const int* __restrict__ rowptr, const int* __restrict__ col,
                                  const float* __restrict__ val, const int* __restrict__ rank,
                                  int m_nz, unsigned* __restrict__ bits,
                                  int* __restrict__ lane_rank, int* __restrict__ col5,
                                  float* __restrict__ val5) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)ntiles * 32) return;
  const int t = (int)(gid >> 5), l = (int)(gid & 31);
  const long long K = 32LL * sigma;
  const long long e0 = t * K + (long long)l * sigma;
  unsigned word = 0;
  int rk = m_nz - 1;
  if (e0 < nnz) {
    // row of e0: last r with rowptr[r] <= e0 (it is non-empty)
    int lo = 0, hi = m - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(rowptr + mid) <= e0) lo = mid; else hi = mid - 1;
    }
    int r = lo;
    // the rank of the row open just before e0: one less when a row starts at
    // e0 itself (-1 before the first row)
    rk = __ldg(rank + r) - (__ldg(rowptr + r) == e0 ? 1 : 0);
    for (int j = 0; j < sigma; ++j) {
      const long long e = e0 + j;
      if (e >= nnz) break;
      while (r + 1 < m && __ldg(rowptr + r + 1) <= e) ++r;
      if (__ldg(rowptr + r) == e) word |= 1u << j;
    }
  }
  bits[gid] = word;
  lane_rank[gid] = rk;
  for (int j = 0; j < sigma; ++j) {
    const long long e = e0 + j;
    const long long dst = t * K + (long long)j * 32 + l;
    col5[dst] = e < nnz ? __ldg(col + e) : 0;
    val5[dst] = e < nnz ? __ldg(val + e) : 0.f;
  }
}

// ---- the SpMV kernel: one warp per tile ------------------------------------
__device__ __forceinline__ void csr5_contribute(int R, int t, int slot, double part, int K,
                                                const int* __restrict__ rowptr, double* carry,
                                                unsigned* arrive, double alpha, float* y) {
  const int rs = __ldg(rowptr + R), re = __ldg(rowptr + R + 1);
  const int c_first = rs / K, c_last = (re - 1) / K;
  carry[2 * t + slot] = part;
  __threadfence();
  const unsigned old = atomicAdd(&arrive[c_first], 1u);
  if ((int)old == c_last - c_first) {
    __threadfence();
    const volatile double* vc = carry;
    double sum = vc[2 * c_first + 1];
    for (int cc = c_first + 1; cc <= c_last; ++cc) sum += vc[2 * cc];
    y[R] = (float)(alpha * sum);
    arrive[c_first] = 0u;
  }
}

__device__ __forceinline__ void zero_rows(float* y, int from, int to) {
  for (int r = from; r < to; ++r) y[r] = 0.f;
}

template <int SIGMA, bool GATED>
__global__ void __launch_bounds__(256)
csr5_spmv_kernel(int m, int n, int ntiles, const int* __restrict__ rowptr,
                 const int* __restrict__ col5, const float* __restrict__ val5,
                 const unsigned* __restrict__ bits, const int* __restrict__ lane_rank,
                 const int* __restrict__ nz_rows, int m_nz, const float* __restrict__ x,
                 const int* __restrict__ xbits, double alpha, float* __restrict__ y,
                 double* carry, unsigned* arrive, int* err) {
  constexpr int K = 32 * SIGMA;
  const int t = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int l = threadIdx.x & 31;
  if (t >= ntiles) return;  // whole warps exit together
  const unsigned flags = __ldg(bits + (size_t)t * 32 + l);
  int rk = __ldg(lane_rank + (size_t)t * 32 + l);
  const size_t base = (size_t)t * K + l;
  double run = 0.0, head = 0.0;
  bool seen = false;
#pragma unroll
  for (int j = 0; j < SIGMA; ++j) {
    const int c = __ldcs(col5 + base + (size_t)j * 32);
    double p = 0.0;
    if ((unsigned)c < (unsigned)n) {
      if (!GATED || ((__ldg((const unsigned*)xbits + (c >> 5)) >> (c & 31)) & 1u))
        p = (double)__ldcs(val5 + base + (size_t)j * 32) * (double)__ldg(x + c);
    } else {
      flag_error(err, kDevErrOob);
    }
    if ((flags >> j) & 1u) {
      if (!seen) {
        head = run;
        seen = true;
      } else if ((unsigned)rk < (unsigned)m_nz) {
        y[__ldg(nz_rows + rk)] = (float)(alpha * run);  // a row complete inside the lane
      } else {
        flag_error(err, kDevErrOob);
      }
      ++rk;
      if ((unsigned)rk < (unsigned)m_nz) {
        // empty rows between the previous non-empty row and this one
        if (rk >= 1) zero_rows(y, __ldg(nz_rows + rk - 1) + 1, __ldg(nz_rows + rk));
      } else {
        flag_error(err, kDevErrOob);
      }
      run = 0.0;
    }
    run += p;
  }
  if (!seen) head = run;  // the whole lane continues the open row
  const double tail = seen ? run : 0.0;
  // segmented suffix sum of head partials: V[l] = head[l] + ... + head[b],
  // b the first lane >= l that opens a row (or lane 31); only values of one
  // row are ever added together
  double V = head;
  int stop = seen;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double v2 = __shfl_down_sync(0xffffffffu, V, o);
    const int s2 = __shfl_down_sync(0xffffffffu, stop, o);
    if (l + o < 32 && !stop) {
      V += v2;
      stop |= s2;
    }
  }
  const double Vnext = __shfl_down_sync(0xffffffffu, V, 1);  // V[l+1]
  const double V0 = __shfl_sync(0xffffffffu, V, 0);
  const unsigned f0 = __shfl_sync(0xffffffffu, flags, 0);
  const int tile_end = (t + 1) * K;
  if (seen && (unsigned)rk < (unsigned)m_nz) {
    // the last row opened in this lane: its tail plus the heads of the lanes
    // up to the next lane that opens a row (or to the end of the tile)
    const int R = __ldg(nz_rows + rk);
    const double sum = tail + (l < 31 ? Vnext : 0.0);
    if (__ldg(rowptr + R + 1) <= tile_end) y[R] = (float)(alpha * sum);
    else csr5_contribute(R, t, 1, sum, K, rowptr, carry, arrive, alpha, y);
  }
  if (l == 0) {
    const int r0 = __ldg(lane_rank + (size_t)t * 32);
    if (!(f0 & 1u) && (unsigned)r0 < (unsigned)m_nz) {
      // the row open at the tile start began in an earlier tile: its part here
      // runs through the first lane that opens a row (or the whole tile)
      csr5_contribute(__ldg(nz_rows + r0), t, 0, V0, K, rowptr, carry, arrive, alpha, y);
    }
    if (t == 0) zero_rows(y, 0, __ldg(nz_rows + 0));
    if (t == ntiles - 1) zero_rows(y, __ldg(nz_rows + m_nz - 1) + 1, m);
  }
}

}  // namespace spmx

using namespace spmx;

// ---- handle glue -----------------------------------------------------------
struct Csr5Tables {
  int sigma = 0, K = 0, ntiles = 0, m_nz = 0;
  int* col5 = nullptr;
  float* val5 = nullptr;
  unsigned* bits = nullptr;
  int* lane_rank = nullptr;
  int* nz_rows = nullptr;
  double* carry = nullptr;
  unsigned* arrive = nullptr;
};

static Csr5Tables* tables(spmx_handle_t h) { return reinterpret_cast<Csr5Tables*>(h->csr5); }

static int csr5_auto_sigma(int m, int nnz) {
  // setSigma, ANONYMOUSLIB_AUTO_TUNED_SIGMA (H:1396-1416)
  const int r = 4, s = 32, t = 256, u = 6;
  const int per = m ? nnz / m : 0;
  if (per <= r) return r;
  if (per <= s) return per;
  if (per <= t) return s;
  return u;
}

extern "C" int spmx_set_sigma(spmx_handle_t h, int sigma) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  if (sigma != -1 && (sigma < 1 || sigma > 32))
    return set_error(SPMX_ERR_INVALID_VALUE, "sigma must be -1 (auto) or in [1, 32]");
  h->sigma = sigma;
  return SPMX_SUCCESS;
}

extern "C" int spmx_csr5_postprocess(spmx_handle_t h) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  Csr5Tables* t = tables(h);
  if (t) {
    cudaStreamSynchronize(h->stream);
    dfree(t->col5); dfree(t->val5); dfree(t->bits); dfree(t->lane_rank);
    dfree(t->nz_rows); dfree(t->carry); dfree(t->arrive);
    delete t;
    h->csr5 = nullptr;
  }
  return SPMX_SUCCESS;
}

#define CSR5_TRY(expr)                                                          \
  do {                                                                          \
    int r_ = (expr);                                                            \
    if (r_ != SPMX_SUCCESS) { spmx_csr5_postprocess(h); return r_; }            \
  } while (0)

static const int kSigmas[] = {4, 6, 8, 12, 16, 24, 32};

static int pick_sigma(int s) {
  // kernels are instantiated for a few sigmas; round up to the next one
  for (int v : kSigmas) if (s <= v) return v;
  return 32;
}

extern "C" int spmx_csr5_preprocess(spmx_handle_t h) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  if (!h->has_csr || (!h->val && h->nnz > 0))
    return set_error(SPMX_ERR_NOT_READY, "CSR5 needs the CSR input with values");
  spmx_csr5_postprocess(h);
  Csr5Tables* t = new Csr5Tables();
  h->csr5 = t;
  const int m = h->m, nnz = h->nnz;
  const int want = h->sigma == -1 ? csr5_auto_sigma(m, nnz) : h->sigma;
  t->sigma = pick_sigma(want);
  t->K = 32 * t->sigma;
  t->ntiles = (nnz + t->K - 1) / t->K;
  cudaStream_t st = h->stream;
  int *flag = nullptr, *rank = nullptr;
  CSR5_TRY(dalloc((void**)&flag, 4 * (size_t)std::max(m, 1), "csr5 flags"));
  CSR5_TRY(dalloc((void**)&rank, 4 * (size_t)std::max(m, 1), "csr5 rank"));
  int* d_mnz = h->d_counts + kCntTotal - 1;
  if (m > 0) {
    note_launch();
    nonempty_flag_kernel<<<(m + 255) / 256, 256, 0, st>>>(m, h->rowptr, flag);
    if (launch_scan_exclusive(flag, rank, m, d_mnz, h->ls, h->d_err, st)) {
      dfree(flag); dfree(rank);
      spmx_csr5_postprocess(h);
      return set_error(SPMX_ERR_INVALID_VALUE, "scan capacity");
    }
  }
  int mnz = 0;
  cudaMemcpyAsync(&mnz, d_mnz, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) {
    dfree(flag); dfree(rank);
    spmx_csr5_postprocess(h);
    return set_error(SPMX_ERR_CUDA, "csr5 preprocess");
  }
  if (m == 0) mnz = 0;
  t->m_nz = mnz;
  const size_t lanes = (size_t)std::max(t->ntiles, 1) * 32;
  const size_t padded = (size_t)std::max(t->ntiles, 1) * t->K;
  CSR5_TRY(dalloc((void**)&t->nz_rows, 4 * (size_t)std::max(mnz, 1), "csr5 nz rows"));
  CSR5_TRY(dalloc((void**)&t->bits, 4 * lanes, "csr5 bits"));
  CSR5_TRY(dalloc((void**)&t->lane_rank, 4 * lanes, "csr5 lane rank"));
  CSR5_TRY(dalloc((void**)&t->col5, 4 * padded, "csr5 col"));
  CSR5_TRY(dalloc((void**)&t->val5, 4 * padded, "csr5 val"));
  CSR5_TRY(dalloc((void**)&t->carry, 16 * (size_t)std::max(t->ntiles, 1), "csr5 carry"));
  CSR5_TRY(dalloc((void**)&t->arrive, 4 * (size_t)std::max(t->ntiles, 1), "csr5 arrive"));
  cudaMemsetAsync(t->arrive, 0, 4 * (size_t)std::max(t->ntiles, 1), st);
  if (m > 0) {
    note_launch(2);
    nonempty_list_kernel<<<(m + 255) / 256, 256, 0, st>>>(m, h->rowptr, rank, t->nz_rows);
    if (t->ntiles > 0)
      csr5_tiles_kernel<<<(unsigned)((lanes + 255) / 256), 256, 0, st>>>(
          m, nnz, t->sigma, t->ntiles, h->rowptr, h->col, h->val, rank, mnz, t->bits,
          t->lane_rank, t->col5, t->val5);
  }
  cudaError_t e = cudaStreamSynchronize(st);
  dfree(flag);
  dfree(rank);
  if (e != cudaSuccess) {
    spmx_csr5_postprocess(h);
    return set_error(SPMX_ERR_CUDA, std::string("csr5 preprocess: ") + cudaGetErrorString(e));
  }
  return SPMX_SUCCESS;
}

int csr5_spmv_impl(spmx_handle_t h, float alpha, float* y, bool gated) {
  Csr5Tables* t = tables(h);
  if (!t) return set_error(SPMX_ERR_NOT_READY, "call spmx_csr5_preprocess first");
  if (!h->x_dense) return set_error(SPMX_VEC_FORMAT_ERR, "CSR5 needs the dense x (set_x / sparse2dense)");
  if (gated && !h->bitvec) return set_error(SPMX_VEC_FORMAT_ERR, "CSR5 SpMSpV needs the bitarray");
  if (!y && h->m > 0) return set_error(SPMX_ERR_INVALID_VALUE, "y is NULL");
  cudaStream_t st = h->stream;
  if (h->m == 0) return SPMX_SUCCESS;
  if (t->ntiles == 0 || t->m_nz == 0) {
    cudaMemsetAsync(y, 0, 4 * (size_t)h->m, st);
    return SPMX_SUCCESS;
  }
  const long long threads = (long long)t->ntiles * 32;
  const unsigned grid = (unsigned)((threads + 255) / 256);
  const int* xb = gated ? h->bitvec : nullptr;
#define SPMX_CSR5_CASE(S)                                                                 \
  case S:                                                                                \
    if (gated)                                                                           \
      e = launch_l2_window(csr5_spmv_kernel<S, true>, dim3(grid), dim3(256), 0, st,      \
          h->x_dense, 4 * (size_t)h->n,                                                  \
          h->m, h->n, t->ntiles, h->rowptr, (const int*)t->col5, (const float*)t->val5,  \
          (const unsigned*)t->bits, (const int*)t->lane_rank, (const int*)t->nz_rows,    \
          t->m_nz, (const float*)h->x_dense, xb, (double)alpha, y, t->carry, t->arrive,   \
          h->d_err);                                                                     \
    else                                                                                 \
      e = launch_l2_window(csr5_spmv_kernel<S, false>, dim3(grid), dim3(256), 0, st,     \
          h->x_dense, 4 * (size_t)h->n,                                                  \
          h->m, h->n, t->ntiles, h->rowptr, (const int*)t->col5, (const float*)t->val5,  \
          (const unsigned*)t->bits, (const int*)t->lane_rank, (const int*)t->nz_rows,    \
          t->m_nz, (const float*)h->x_dense, xb, (double)alpha, y, t->carry, t->arrive,   \
          h->d_err);                                                                     \
    break;
  cudaError_t e = cudaSuccess;
  note_launch();
  switch (t->sigma) {
    SPMX_CSR5_CASE(4)
    SPMX_CSR5_CASE(6)
    SPMX_CSR5_CASE(8)
    SPMX_CSR5_CASE(12)
    SPMX_CSR5_CASE(16)
    SPMX_CSR5_CASE(24)
    SPMX_CSR5_CASE(32)
    default:
      return set_error(SPMX_ERR_INVALID_VALUE, "unsupported sigma");
  }
#undef SPMX_CSR5_CASE
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(SPMX_ERR_CUDA, std::string("csr5 spmv: ") + cudaGetErrorString(e));
  return SPMX_SUCCESS;
}

extern "C" int spmx_csr5_sigma(spmx_handle_t h, int* sigma) {
  if (!h || !sigma) return set_error(SPMX_ERR_INVALID_VALUE, "NULL argument");
  Csr5Tables* t = tables(h);
  *sigma = t ? t->sigma : (h->sigma == -1 ? csr5_auto_sigma(h->m, h->nnz) : h->sigma);
  return SPMX_SUCCESS;
}
