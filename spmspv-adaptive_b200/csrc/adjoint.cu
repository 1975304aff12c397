// Adjoint of y = A x for the FP32 semiring (no reference counterpart: the
// reference has no differentiation).  For a loss L(y):
//   dx    = A^T dy                  (the transpose product)
//   dvals = dy[row_k] * x[col_k]    (the gradient on the nonzero pattern)
//
// dense dy, handle with a CSC: dx is the row-ordered SpMV of the transpose
//   (the CSC read as the CSR of A^T, dy as its x: a gather, no atomics) and
//   dvals a streaming pass over the CSR.  Both are deterministic.
// dense dy, CSR only: ONE pass over the CSR, fixed 2048 nonzeros per CTA
//   (the Hola chunks): every nonzero writes its dvals entry and adds
//   val*dy[row] into dx[col] with an FP32 atomic, so the matrix is streamed
//   once for both gradients.  The row of each nonzero comes from a max-scan
//   of row-start marks in shared memory (no per-element search).
// sparse dy (dy_key, dy_val): only the rows in dy's support contribute, so a
//   group of lanes per dy entry walks that row (the CSR of A is the CSC of
//   A^T: this is the CSC SpMSpV of the transpose) after dx and dvals are
//   zeroed.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace spmx {

template <int NT, int VT>
__global__ void __launch_bounds__(NT)
spmv_backward_kernel(int m, int n, int nnz, const int* __restrict__ rowptr,
                     const int* __restrict__ col, const float* __restrict__ val,
                     const float* __restrict__ x, const float* __restrict__ dy,
                     const int* __restrict__ chunk_row, float* __restrict__ dx,
                     float* __restrict__ dvals, int* err) {
  constexpr int K = NT * VT;
  __shared__ int s_mark[K];
  __shared__ int s_incl[NT];
  __shared__ int s_wtmp[NT / 32 + 1];
  const int c = blockIdx.x;
  const int s = c * K;
  const int e = min(s + K, nnz);
  const int lo = __ldg(chunk_row + c), hi = __ldg(chunk_row + c + 1);
  for (int q = threadIdx.x; q < K; q += NT) s_mark[q] = -1;
  __syncthreads();
  // rows that start inside the chunk mark their first element; several empty
  // rows at one position leave the largest index, the non-empty one
  for (int r = lo + (int)threadIdx.x; r < hi; r += NT) {
    const int p = __ldg(rowptr + r) - s;
    if (p < e - s) atomicMax(&s_mark[p], r);
  }
  __syncthreads();
  int loc[VT];
  int run = INT_MIN;
  const int head = lo - 1;  // the row open at the chunk start (if any)
#pragma unroll
  for (int j = 0; j < VT; ++j) {
    const int q = threadIdx.x * VT + j;
    int v = s_mark[q];
    if (q == 0) v = max(v, head);
    run = max(run, v);
    loc[j] = run;
  }
  const int inc = block_inclusive_max<NT>(run, s_wtmp);
  s_incl[threadIdx.x] = inc;
  __syncthreads();
  const int carry = threadIdx.x ? s_incl[threadIdx.x - 1] : INT_MIN;
#pragma unroll
  for (int j = 0; j < VT; ++j) s_mark[threadIdx.x * VT + j] = max(loc[j], carry);
  __syncthreads();
#pragma unroll
  for (int j = 0; j < VT; ++j) {
    const int q = j * NT + threadIdx.x;  // coalesced over the chunk
    const int k = s + q;
    if (k < e) {
      const int r = s_mark[q];
      const int cc = __ldg(col + k);
      if ((unsigned)r >= (unsigned)m || (unsigned)cc >= (unsigned)n) {
        flag_error(err, kDevErrOob);
        continue;
      }
      const float g = __ldg(dy + r);
      if (dvals) dvals[k] = g * __ldg(x + cc);
      if (dx && g != 0.0f) atomicAdd(dx + cc, __ldg(val + k) * g);
    }
  }
}

// Dense-dy adjoint on a handle with a CSC, one launch: even CTAs compute dx
// (G1 lanes per column of the CSC, a gather of dy with FP64 sums, every dx
// entry written once), odd CTAs write dvals (G2 lanes per row of the CSR).
// The two halves stream different arrays side by side; neither uses atomics.
template <int G1, int G2>
__global__ void __launch_bounds__(256)
adjoint_csc_kernel(int m, int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                   const int* __restrict__ colptr, const int* __restrict__ crow,
                   const float* __restrict__ cval, const float* __restrict__ x,
                   const float* __restrict__ dy, float* __restrict__ dx,
                   float* __restrict__ dvals, int* err) {
  const long long gid = (long long)(blockIdx.x >> 1) * blockDim.x + threadIdx.x;
  if ((blockIdx.x & 1) == 0) {
    if (!dx || gid / G1 >= ((long long)n + 31) / 32 * 32) return;  // whole warps past the end
    const long long j = gid / G1;
    const int g = (int)(gid % G1);
    double sum = 0.0;
    if (j < n) {
      const int a = __ldg(colptr + j), b = __ldg(colptr + j + 1);
      for (int k = a + g; k < b; k += G1) {
        const int r = __ldg(crow + k);
        if ((unsigned)r >= (unsigned)m) {
          flag_error(err, kDevErrOob);
          continue;
        }
        sum += (double)__ldg(cval + k) * (double)__ldg(dy + r);
      }
    }
    if (G1 > 1) {
#pragma unroll
      for (int o = G1 / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, G1);
    }
    if (j < n && g == 0) dx[j] = (float)sum;
  } else {
    const long long row = gid / G2;
    if (!dvals || row >= m) return;
    const int g = (int)(gid % G2);
    const float d = __ldg(dy + row);
    const int a = __ldg(rowptr + row), b = __ldg(rowptr + row + 1);
    for (int k = a + g; k < b; k += G2) {
      const int c = __ldg(col + k);
      if ((unsigned)c >= (unsigned)n) {
        flag_error(err, kDevErrOob);
        dvals[k] = 0.f;
        continue;
      }
      dvals[k] = d * __ldg(x + c);
    }
  }
}

template <int G>
__global__ void __launch_bounds__(256)
spmv_backward_sparse_kernel(int m, int n, const int* __restrict__ rowptr,
                            const int* __restrict__ col, const float* __restrict__ val,
                            const float* __restrict__ x, int dy_nnz,
                            const int* __restrict__ dy_key, const float* __restrict__ dy_val,
                            float* __restrict__ dx, float* __restrict__ dvals, int* err) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(gid / G), g = (int)(gid % G);
  if (i >= dy_nnz) return;
  const int r = __ldg(dy_key + i);
  if ((unsigned)r >= (unsigned)m) { if (g == 0) flag_error(err, kDevErrOob); return; }
  const float d = __ldg(dy_val + i);
  const int a = __ldg(rowptr + r), b = __ldg(rowptr + r + 1);
  for (int k = a + g; k < b; k += G) {
    const int cc = __ldg(col + k);
    if ((unsigned)cc >= (unsigned)n) { flag_error(err, kDevErrOob); continue; }
    if (dvals) dvals[k] = d * __ldg(x + cc);
    if (dx) atomicAdd(dx + cc, __ldg(val + k) * d);
  }
}

int launch_spmv_backward(int m, int n, int nnz, const int* rowptr, const int* col,
                         const float* val, const float* x, const float* dy,
                         const HolaTables& t, float* dx, float* dvals, int* err,
                         cudaStream_t st) {
  if (nnz <= 0 || t.nchunks == 0) return 0;
  if (t.K != 2048) return -1;  // the backward pass uses 256 x 8 chunks
  note_launch();
  spmv_backward_kernel<256, 8><<<t.nchunks, 256, 0, st>>>(m, n, nnz, rowptr, col, val, x, dy,
                                                          t.chunk_row, dx, dvals, err);
  return 0;
}

template <int G1>
static void adjoint_csc_g2(int g2, unsigned grid, cudaStream_t st, int m, int n, const int* rowptr,
                           const int* col, const int* colptr, const int* crow, const float* cval,
                           const float* x, const float* dy, float* dx, float* dvals, int* err) {
  switch (g2) {
    case 1: adjoint_csc_kernel<G1, 1><<<grid, 256, 0, st>>>(m, n, rowptr, col, colptr, crow, cval, x, dy, dx, dvals, err); break;
    case 2: adjoint_csc_kernel<G1, 2><<<grid, 256, 0, st>>>(m, n, rowptr, col, colptr, crow, cval, x, dy, dx, dvals, err); break;
    case 4: adjoint_csc_kernel<G1, 4><<<grid, 256, 0, st>>>(m, n, rowptr, col, colptr, crow, cval, x, dy, dx, dvals, err); break;
    default: adjoint_csc_kernel<G1, 8><<<grid, 256, 0, st>>>(m, n, rowptr, col, colptr, crow, cval, x, dy, dx, dvals, err); break;
  }
}

int launch_spmv_backward_csc(int m, int n, const int* rowptr, const int* col, const int* colptr,
                             const int* crow, const float* cval, const float* x, const float* dy,
                             int g1, int g2, float* dx, float* dvals, int* err, cudaStream_t st) {
  if ((!dx || n <= 0) && (!dvals || m <= 0)) return 0;
  const long long t1 = dx ? ((long long)n + 31) / 32 * 32 * g1 : 0;
  const long long t2 = dvals ? (long long)m * g2 : 0;
  const long long half = (std::max(t1, t2) + 255) / 256;
  const unsigned grid = (unsigned)(2 * half);
  note_launch();
  switch (g1) {
    case 1: adjoint_csc_g2<1>(g2, grid, st, m, n, rowptr, col, colptr, crow, cval, x, dy, dx, dvals, err); break;
    case 2: adjoint_csc_g2<2>(g2, grid, st, m, n, rowptr, col, colptr, crow, cval, x, dy, dx, dvals, err); break;
    case 4: adjoint_csc_g2<4>(g2, grid, st, m, n, rowptr, col, colptr, crow, cval, x, dy, dx, dvals, err); break;
    case 8: adjoint_csc_g2<8>(g2, grid, st, m, n, rowptr, col, colptr, crow, cval, x, dy, dx, dvals, err); break;
    case 16: adjoint_csc_g2<16>(g2, grid, st, m, n, rowptr, col, colptr, crow, cval, x, dy, dx, dvals, err); break;
    default: adjoint_csc_g2<32>(g2, grid, st, m, n, rowptr, col, colptr, crow, cval, x, dy, dx, dvals, err); break;
  }
  return 0;
}

int launch_spmv_backward_sparse(int m, int n, const int* rowptr, const int* col,
                                const float* val, const float* x, int dy_nnz,
                                const int* dy_key, const float* dy_val, int group,
                                float* dx, float* dvals, int* err, cudaStream_t st) {
  if (dy_nnz <= 0) return 0;
  const long long threads = (long long)dy_nnz * group;
  const unsigned grid = (unsigned)((threads + 255) / 256);
  note_launch();
  switch (group) {
    case 1: spmv_backward_sparse_kernel<1><<<grid, 256, 0, st>>>(m, n, rowptr, col, val, x, dy_nnz, dy_key, dy_val, dx, dvals, err); break;
    case 2: spmv_backward_sparse_kernel<2><<<grid, 256, 0, st>>>(m, n, rowptr, col, val, x, dy_nnz, dy_key, dy_val, dx, dvals, err); break;
    case 4: spmv_backward_sparse_kernel<4><<<grid, 256, 0, st>>>(m, n, rowptr, col, val, x, dy_nnz, dy_key, dy_val, dx, dvals, err); break;
    case 8: spmv_backward_sparse_kernel<8><<<grid, 256, 0, st>>>(m, n, rowptr, col, val, x, dy_nnz, dy_key, dy_val, dx, dvals, err); break;
    case 16: spmv_backward_sparse_kernel<16><<<grid, 256, 0, st>>>(m, n, rowptr, col, val, x, dy_nnz, dy_key, dy_val, dx, dvals, err); break;
    default: spmv_backward_sparse_kernel<32><<<grid, 256, 0, st>>>(m, n, rowptr, col, val, x, dy_nnz, dy_key, dy_val, dx, dvals, err); break;
  }
  return 0;
}

}  // namespace spmx
