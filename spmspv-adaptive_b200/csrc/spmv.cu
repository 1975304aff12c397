// CSR SpMV and bitmap-gated CSR SpMSpV kernels (y = alpha * A * x).
//
// naive ("row group"): G threads per row, FP64 accumulation, shuffle reduce.
//   Replaces naive_spmv_ker / naive_spmspv_ker (DEV/naivespmv.h:13-51), which
//   is the G = 1 case.
//
// hola ("fixed nnz per CTA"): each CTA owns K = NT*VT consecutive nonzeros,
//   like hola_spmv's fixed-work blocks (DEV/holaspmv.h:2070-2220) with its
//   block-start table (DetermineBlockStarts, DEV/holaspmv.h:40-63).  The design
//   is our own: products are formed exactly in FP64 (float*float fits a
//   double), a CTA-wide FP64 prefix P[] is kept in shared memory and every row
//   inside the chunk is P[end]-P[begin], rounded once to FP32.  Rows that cross
//   chunk boundaries leave one FP64 partial per chunk; the last chunk to arrive
//   (atomic counter per row) adds the partials in chunk order and writes y, so
//   the result is deterministic and needs no zero-fill of y and no second
//   launch.
#include "kernels.h"
#include "common.cuh"

namespace spmx {

__device__ __forceinline__ bool bit_is_set(const int* bits, int idx) {
  unsigned w = __ldg((const unsigned*)bits + (idx >> 5));
  return (w >> (idx & 31)) & 1u;
}

// --------------------------------------------------------------------------
// naive: G lanes per row
// --------------------------------------------------------------------------
template <int G, bool GATED>
__global__ void __launch_bounds__(256)
spmv_rowgroup_kernel(int m, int n, const int* __restrict__ rowptr,
                     const int* __restrict__ col, const float* __restrict__ val,
                     const float* __restrict__ x, const int* __restrict__ bits,
                     double alpha, float* __restrict__ y, int* err) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int row = (int)(gid / G);
  const int g = (int)(gid % G);
  double sum = 0.0;
  if (row < m) {
    const int a = __ldg(rowptr + row), b = __ldg(rowptr + row + 1);
    int k = a + g;
#pragma unroll 4
    for (; k < b; k += G) {
      int c = __ldg(col + k);
      if ((unsigned)c >= (unsigned)n) { flag_error(err, kDevErrOob); continue; }
      if (GATED && !bit_is_set(bits, c)) continue;
      sum += (double)__ldg(val + k) * (double)__ldg(x + c);
    }
  }
  if (G > 1) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, G);
  }
  if (row < m && g == 0) y[row] = (float)(alpha * sum);
}

// --------------------------------------------------------------------------
// hola: fixed nnz per CTA
// --------------------------------------------------------------------------

// chunk_row[c] = first row r with rowptr[r] >= c*K (lower bound over
// rowptr[0..m)); chunk_row[nchunks] = m.
__global__ void chunk_rows_kernel(int m, const int* __restrict__ rowptr, int K,
                                  int nchunks, int* __restrict__ chunk_row) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > nchunks) return;
  if (c == nchunks) { chunk_row[c] = m; return; }
  long long target = (long long)c * K;
  int lo = 0, hi = m;  // search in [0, m)
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (__ldg(rowptr + mid) < target) lo = mid + 1; else hi = mid;
  }
  chunk_row[c] = lo;
}

// One partial of a row that crosses chunk boundaries.  slot 1: the chunk in
// which the row starts; slot 0: a later chunk the row continues into.
template <int K>
__device__ __forceinline__ void split_row_contribute(
    int R, int c, int slot, double part, const int* __restrict__ rowptr,
    double* carry, unsigned* arrive, double alpha, float* y) {
  const int rs = __ldg(rowptr + R), re = __ldg(rowptr + R + 1);
  const int c_first = rs / K, c_last = (re - 1) / K;
  carry[2 * c + slot] = part;
  __threadfence();
  unsigned old = atomicAdd(&arrive[c_first], 1u);
  if ((int)old == c_last - c_first) {
    __threadfence();
    const volatile double* vc = carry;
    double sum = vc[2 * c_first + 1];
    for (int cc = c_first + 1; cc <= c_last; ++cc) sum += vc[2 * cc];
    y[R] = (float)(alpha * sum);
    arrive[c_first] = 0u;  // ready for the next call
  }
}

template <int NT, int VT, bool GATED>
__global__ void __launch_bounds__(NT)
spmv_chunk_kernel(int m, int n, int nnz, const int* __restrict__ rowptr,
                  const int* __restrict__ col, const float* __restrict__ val,
                  const float* __restrict__ x, const int* __restrict__ bits,
                  double alpha, float* __restrict__ y,
                  const int* __restrict__ chunk_row, double* carry,
                  unsigned* arrive, int vec_ok, int* err) {
  constexpr int K = NT * VT;
  __shared__ double sP[K];
  __shared__ double s_wtmp[NT / 32 + 1];
  __shared__ int s_tf[NT / 32 + 1];
  __shared__ unsigned s_flag[K / 32];
  const int c = blockIdx.x;
  const int s = c * K;
  const int e = min(s + K, nnz);
  const int base = s + (int)threadIdx.x * VT;

  double pr[VT];
#pragma unroll
  for (int j = 0; j < VT; ++j) pr[j] = 0.0;

  if (vec_ok && s + K <= nnz && (VT % 4) == 0) {
#pragma unroll
    for (int q = 0; q < VT / 4; ++q) {
      const int4 c4 = __ldcs(reinterpret_cast<const int4*>(col + base) + q);
      const int cc[4] = {c4.x, c4.y, c4.z, c4.w};
      bool want[4];
      bool any = false;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        bool ok = (unsigned)cc[t] < (unsigned)n;
        if (!ok) flag_error(err, kDevErrOob);
        want[t] = ok && (!GATED || bit_is_set(bits, cc[t]));
        any |= want[t];
      }
      if (!GATED || any) {
        const float4 v4 = __ldcs(reinterpret_cast<const float4*>(val + base) + q);
        const float vv[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
        for (int t = 0; t < 4; ++t)
          if (want[t]) pr[q * 4 + t] = (double)vv[t] * (double)__ldg(x + cc[t]);
      }
    }
  } else {
#pragma unroll
    for (int j = 0; j < VT; ++j) {
      const int k = base + j;
      if (k < e) {
        const int cj = __ldg(col + k);
        if ((unsigned)cj >= (unsigned)n) { flag_error(err, kDevErrOob); continue; }
        if (GATED && !bit_is_set(bits, cj)) continue;
        pr[j] = (double)__ldg(val + k) * (double)__ldg(x + cj);
      }
    }
  }

  // row-start flags of the rows that begin inside the chunk
  const int lo = __ldg(chunk_row + c), hi = __ldg(chunk_row + c + 1);
  for (int i = threadIdx.x; i < K / 32; i += NT) s_flag[i] = 0u;
  __syncthreads();
  for (int r = lo + (int)threadIdx.x; r < hi; r += NT) {
    const int p = __ldg(rowptr + r) - s;
    if (p < e - s) atomicOr(&s_flag[p >> 5], 1u << (p & 31));
  }
  __syncthreads();
  // segmented scan: every row is summed from its own products only (no
  // differences of running sums), so all-zero rows stay exactly zero
  unsigned myf;
  {
    const int bit0 = threadIdx.x * VT;
    const unsigned w = s_flag[bit0 >> 5];
    myf = (w >> (bit0 & 31)) & ((VT >= 32) ? 0xffffffffu : ((1u << VT) - 1u));
  }
  double run = 0.0;
#pragma unroll
  for (int j = 0; j < VT; ++j) {
    run = ((myf >> j) & 1u) ? pr[j] : run + pr[j];
    pr[j] = run;
  }
  const double carry_in = block_exclusive_segscan<NT>(myf != 0u, run, s_tf, s_wtmp);
  const int first = myf ? __ffs(myf) - 1 : VT;
#pragma unroll
  for (int j = 0; j < VT; ++j) {
    if (j < first) pr[j] += carry_in;
    sP[threadIdx.x * VT + j] = pr[j];
  }
  __syncthreads();

  for (int r = lo + (int)threadIdx.x; r < hi; r += NT) {
    const int a = __ldg(rowptr + r), b = __ldg(rowptr + r + 1);
    if (b == a) {
      y[r] = 0.f;
    } else if (b <= e) {
      y[r] = (float)(alpha * sP[b - 1 - s]);
    } else {
      split_row_contribute<K>(r, c, 1, sP[e - 1 - s], rowptr, carry, arrive, alpha, y);
    }
  }
  if (threadIdx.x == 0 && lo > 0) {
    const int R = lo - 1;
    const int endR = __ldg(rowptr + lo);
    if (endR > s) {
      const int stop = min(endR, e);
      split_row_contribute<K>(R, c, 0, sP[stop - 1 - s], rowptr, carry, arrive, alpha, y);
    }
  }
}

// --------------------------------------------------------------------------
// host launchers
// --------------------------------------------------------------------------
int launch_spmv_naive(const SpmvArgs& a, int group, cudaStream_t st) {
  if (a.m <= 0) return 0;
  const int NT = 256;
#define SPMX_NAIVE_CASE(G)                                                        \
  case G: {                                                                      \
    long long threads = (long long)a.m * G;                                      \
    unsigned grid = (unsigned)((threads + NT - 1) / NT);                         \
    if (a.bits)                                                                  \
      spmv_rowgroup_kernel<G, true><<<grid, NT, 0, st>>>(                        \
          a.m, a.n, a.rowptr, a.col, a.val, a.x, a.bits, a.alpha, a.y, a.err);   \
    else                                                                         \
      spmv_rowgroup_kernel<G, false><<<grid, NT, 0, st>>>(                       \
          a.m, a.n, a.rowptr, a.col, a.val, a.x, a.bits, a.alpha, a.y, a.err);   \
    break;                                                                       \
  }
  note_launch();
  switch (group) {
    SPMX_NAIVE_CASE(1)
    SPMX_NAIVE_CASE(2)
    SPMX_NAIVE_CASE(4)
    SPMX_NAIVE_CASE(8)
    SPMX_NAIVE_CASE(16)
    SPMX_NAIVE_CASE(32)
    default: return -1;
  }
#undef SPMX_NAIVE_CASE
  return 0;
}

int hola_chunk_nnz(int vt) { return 256 * vt; }

int launch_chunk_rows(int m, const int* rowptr, int K, int nchunks,
                      int* chunk_row, cudaStream_t st) {
  int threads = nchunks + 1;
  note_launch();
  chunk_rows_kernel<<<(threads + 255) / 256, 256, 0, st>>>(m, rowptr, K, nchunks,
                                                         chunk_row);
  return 0;
}

int launch_spmv_hola(const SpmvArgs& a, const HolaTables& t, cudaStream_t st) {
  if (a.m <= 0) return 0;
  if (a.nnz == 0 || t.nchunks == 0) {
    cudaMemsetAsync(a.y, 0, sizeof(float) * (size_t)a.m, st);
    return 0;
  }
  const int vec_ok = (((uintptr_t)a.col | (uintptr_t)a.val) & 15u) == 0;
  constexpr int NT = 256;
#define SPMX_HOLA_CASE(VT)                                                       \
  case VT:                                                                       \
    if (a.bits)                                                                  \
      e = launch_l2_window(spmv_chunk_kernel<NT, VT, true>, dim3(t.nchunks), dim3(NT), 0, st, \
          a.x, 4 * (size_t)a.n, a.m, a.n, a.nnz, a.rowptr, a.col, a.val, a.x, a.bits, \
          a.alpha, a.y, (const int*)t.chunk_row, t.carry, t.arrive, vec_ok, a.err); \
    else                                                                         \
      e = launch_l2_window(spmv_chunk_kernel<NT, VT, false>, dim3(t.nchunks), dim3(NT), 0, st, \
          a.x, 4 * (size_t)a.n, a.m, a.n, a.nnz, a.rowptr, a.col, a.val, a.x, a.bits, \
          a.alpha, a.y, (const int*)t.chunk_row, t.carry, t.arrive, vec_ok, a.err); \
    break;
  cudaError_t e = cudaSuccess;
  note_launch();
  switch (t.vt) {
    SPMX_HOLA_CASE(4)
    SPMX_HOLA_CASE(8)
    SPMX_HOLA_CASE(16)
    default: return -1;
  }
  (void)e;
#undef SPMX_HOLA_CASE
  return 0;
}

}  // namespace spmx
