// Batched SpMSpV and its adjoint (no reference counterpart: the reference
// runs one sparse vector per call).
//
// A batch is nvec sparse vectors in one concatenated list: vector v owns the
// entries [xptr[v], xptr[v+1]) of (xkey, xval).  Forward: Y[v][:] = alpha *
// A * x_v for every v (Y dense, nvec x m, row-major).  Backward, for an
// upstream gradient dY (nvec x m):
//   dxval[e] = alpha * sum_k A[k] * dY[v][row_k]     over column xkey[e]
//              (the gradient of the stored values of x_v, same layout as xval)
//   dvals[k] = alpha * sum_v sum_{e in v, xkey[e] = col_k} xval[e] * dY[v][row_k]
//              (the gradient of A's values, summed over the batch, CSR order)
//
// One persistent kernel serves the whole batch from a device work queue: a
// CTA takes the next chunk of kBatchChunk consecutive entries of the
// concatenated list (chunks cross vector boundaries, so uneven vectors
// balance by themselves), scans the entries' column lengths in shared memory
// and walks the chunk's products in tiles of equal size, each thread a run
// of consecutive products found by one binary search.  The forward adds
// into Y with FP32 atomics; the backward reads dY at the same positions,
// reduces each entry's products in shared memory and adds dvals with
// atomics.  The intermediates of the forward expansion are recomputed, never
// stored.  Nothing is read back to the host (the entry count comes from
// xptr[nvec] on the device), so both calls can be captured in a CUDA graph
// once the handle's scratch exists (first call outside capture).
#include <algorithm>
#include <string>

#include "common.cuh"
#include "engine.h"
#include "kernels.h"
#include "sort.h"

namespace spmx {

constexpr int kBatchNT = 256;
constexpr int kBatchChunk = 256;  // entries per work item
constexpr int kBatchPT = 8;       // products per thread per tile

template <bool FWD>
__global__ void __launch_bounds__(kBatchNT)
spmspv_batched_kernel(int m, int n, int nvec, const int* __restrict__ xptr, const int* __restrict__ xkey,
                      const float* __restrict__ xval, const int* __restrict__ colptr,
                      const int* __restrict__ row, const float* __restrict__ aval,
                      const int* __restrict__ perm, float alpha, float* __restrict__ Y,
                      const float* __restrict__ dY, float* __restrict__ dxval, float* __restrict__ dvals,
                      unsigned* work, int* err) {
  __shared__ int s_off[kBatchChunk + 1];  // exclusive scan of column lengths
  __shared__ int s_col0[kBatchChunk];     // first CSC position of each entry's column
  __shared__ long long s_ybase[kBatchChunk];  // v * m of each entry
  __shared__ float s_xv[kBatchChunk];
  __shared__ float s_dx[kBatchChunk];
  __shared__ int s_wtmp[kBatchNT / 32 + 1];
  __shared__ int s_item;
  const int tid = threadIdx.x;
  const int total = __ldg(xptr + nvec);
  if (total > 0 && (!xkey || !xval)) {  // entries but no arrays: nothing to read
    if (tid == 0 && blockIdx.x == 0) flag_error(err, kDevErrOob);
    return;
  }
  while (true) {
    if (tid == 0) s_item = (int)atomicAdd(work, 1u);
    __syncthreads();
    const long long e0 = (long long)s_item * kBatchChunk;
    if (e0 >= total) break;
    const int ne = (int)min((long long)kBatchChunk, (long long)total - e0);
    int len = 0;
    if (tid < ne) {
      const int e = (int)e0 + tid;
      const int j = __ldg(xkey + e);
      int v = 0;  // vector of entry e: last v with xptr[v] <= e
      int lo = 0, hi = nvec;
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(xptr + mid) <= e) lo = mid;
        else hi = mid;
      }
      v = lo;
      if ((unsigned)j < (unsigned)n) {
        const int a = __ldg(colptr + j);
        len = __ldg(colptr + j + 1) - a;
        s_col0[tid] = a;
      } else {
        flag_error(err, kDevErrOob);
        s_col0[tid] = 0;
      }
      s_ybase[tid] = (long long)v * m;
      s_xv[tid] = __ldg(xval + e);
      s_dx[tid] = 0.f;
    }
    int tot = 0;
    const int ex = block_exclusive_sum<kBatchNT, int>(len, s_wtmp, &tot);
    if (tid < kBatchChunk) s_off[tid] = ex;
    if (tid == 0) s_off[kBatchChunk] = tot;
    __syncthreads();
    // products of the chunk in tiles of kBatchNT * kBatchPT
    for (int t0 = 0; t0 < tot; t0 += kBatchNT * kBatchPT) {
      const int p0 = t0 + tid * kBatchPT;
      if (p0 < tot) {
        int lo = 0, hi = ne;  // entry holding product p0: last i with s_off[i] <= p0
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (s_off[mid] <= p0) lo = mid;
          else hi = mid;
        }
        int i = lo;
        float dx_acc = 0.f;
#pragma unroll
        for (int q = 0; q < kBatchPT; ++q) {
          const int p = p0 + q;
          if (p >= tot) break;
          while (s_off[i + 1] <= p) {
            if (!FWD && dx_acc != 0.f) atomicAdd(&s_dx[i], dx_acc);
            dx_acc = 0.f;
            ++i;
          }
          const int k = s_col0[i] + (p - s_off[i]);
          const int r = __ldg(row + k);
          if ((unsigned)r >= (unsigned)m) {
            flag_error(err, kDevErrOob);
            continue;
          }
          const float a = __ldg(aval + k);
          if (FWD) {
            atomicAdd(Y + s_ybase[i] + r, alpha * s_xv[i] * a);
          } else {
            const float g = __ldg(dY + s_ybase[i] + r);
            dx_acc += a * g;
            if (dvals) atomicAdd(dvals + __ldg(perm + k), alpha * s_xv[i] * g);
          }
        }
        if (!FWD && dx_acc != 0.f) atomicAdd(&s_dx[i], dx_acc);
      }
    }
    __syncthreads();
    if (!FWD && dxval && tid < ne) dxval[e0 + tid] = alpha * s_dx[tid];
    __syncthreads();  // s_item, s_off, s_dx are reused by the next chunk
  }
}

__global__ void iota_kernel(int n, unsigned* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = (unsigned)i;
}

}  // namespace spmx

using namespace spmx;

static int batched_grid(spmx_handle_t h) {
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, spmspv_batched_kernel<true>, kBatchNT, 0) !=
          cudaSuccess ||
      per < 1) {
    cudaGetLastError();
    per = 4;
  }
  return per * h->num_sms;
}

// CSR index of every CSC position (stable sort of the CSR column keys with
// the CSR index as payload), built once per matrix
static int ensure_csc_perm(spmx_handle_t h) {
  if (h->csc_perm && h->csc_perm_nnz == h->nnz && h->csc_perm_col == h->col) return SPMX_SUCCESS;
  if (!h->has_csr) return set_error(SPMX_ERR_NOT_READY, "dvals needs the CSR input (spmx_input_csr)");
  cudaStream_t st = h->stream;
  const int nnz = h->nnz, n = h->n;
  dfree(h->csc_perm);
  h->csc_perm = nullptr;
  SPMX_TRY(dalloc((void**)&h->csc_perm, 4 * (size_t)std::max(nnz, 1), "csc to csr permutation"));
  if (nnz > 0) {
    unsigned *k0 = nullptr, *k1 = nullptr, *p0 = nullptr, *p1 = nullptr;
    int *hist = nullptr, *hoff = nullptr;
    const size_t b = 4 * (size_t)nnz;
    const size_t hn = radix_hist_ints(nnz);
    int rc = SPMX_SUCCESS;
    rc = rc ? rc : dalloc((void**)&k0, b, "perm keys");
    rc = rc ? rc : dalloc((void**)&k1, b, "perm keys alt");
    rc = rc ? rc : dalloc((void**)&p0, b, "perm payload");
    rc = rc ? rc : dalloc((void**)&p1, b, "perm payload alt");
    rc = rc ? rc : dalloc((void**)&hist, 4 * hn, "perm hist");
    rc = rc ? rc : dalloc((void**)&hoff, 4 * hn, "perm hist off");
    if (!rc) {
      cudaMemcpyAsync(k0, h->col, b, cudaMemcpyDeviceToDevice, st);
      note_launch();
      iota_kernel<<<std::min((nnz + 255) / 256, h->num_sms * 16), 256, 0, st>>>(nnz, p0);
      int bits = 1;
      while ((1LL << bits) < (long long)std::max(n, 2)) ++bits;
      RadixBuffers rb{k0, k1, p0, p1, nullptr, nullptr, hist, hoff, false};
      if (radix_sort_pairs(rb, nnz, bits, h->ls, h->d_err, st))
        rc = set_error(SPMX_ERR_INVALID_VALUE, "permutation sort capacity");
      else
        cudaMemcpyAsync(h->csc_perm, rb.result_in_alt ? p1 : p0, b, cudaMemcpyDeviceToDevice, st);
    }
    const cudaError_t se = cudaStreamSynchronize(st);
    dfree(k0); dfree(k1); dfree(p0); dfree(p1); dfree(hist); dfree(hoff);
    if (!rc && se != cudaSuccess) rc = set_error(SPMX_ERR_CUDA, cudaGetErrorString(se));
    if (rc) {
      dfree(h->csc_perm);
      h->csc_perm = nullptr;
      return rc;
    }
  }
  h->csc_perm_nnz = h->nnz;
  h->csc_perm_col = h->col;
  return SPMX_SUCCESS;
}

static int batched_common(spmx_handle_t h, int nvec, const int* xptr, const int* xkey, const float* xval) {
  if (nvec < 1) return set_error(SPMX_ERR_INVALID_VALUE, "nvec must be >= 1");
  // xkey / xval may be NULL for a batch without entries (the kernel checks
  // xptr[nvec] on the device and records an error if entries exist)
  if (!xptr) return set_error(SPMX_ERR_INVALID_VALUE, "xptr is NULL");
  if (!h->has_csc || !h->csc_val) return set_error(SPMX_ERR_NOT_READY, "batched SpMSpV needs the CSC with values");
  if (!h->batch_work) SPMX_TRY(dalloc((void**)&h->batch_work, 4, "batch work counter"));
  return SPMX_SUCCESS;
}

extern "C" int spmx_spmspv_batched(spmx_handle_t h, int nvec, const int* d_xptr, const int* d_xkey,
                                   const float* d_xval, float alpha, float* d_Y) {
  SPMX_CHECK_HANDLE(h);
  SPMX_TRY(batched_common(h, nvec, d_xptr, d_xkey, d_xval));
  if (!d_Y) return set_error(SPMX_ERR_INVALID_VALUE, "Y is NULL");
  cudaStream_t st = h->stream;
  SPMX_CUDA(cudaMemsetAsync(d_Y, 0, 4 * (size_t)nvec * (size_t)h->m, st));
  SPMX_CUDA(cudaMemsetAsync(h->batch_work, 0, 4, st));
  note_launch();
  spmspv_batched_kernel<true><<<batched_grid(h), kBatchNT, 0, st>>>(
      h->m, h->n, nvec, d_xptr, d_xkey, d_xval, h->csc_colptr, h->csc_row, h->csc_val, nullptr, alpha, d_Y,
      nullptr, nullptr, nullptr, h->batch_work, h->d_err);
  return launch_ok("batched spmspv");
}

extern "C" int spmx_spmspv_batched_backward(spmx_handle_t h, int nvec, const int* d_xptr, const int* d_xkey,
                                            const float* d_xval, float alpha, const float* d_dY,
                                            float* d_dxval, float* d_dvals) {
  SPMX_CHECK_HANDLE(h);
  SPMX_TRY(batched_common(h, nvec, d_xptr, d_xkey, d_xval));
  if (!d_dY) return set_error(SPMX_ERR_INVALID_VALUE, "dY is NULL");
  if (d_dvals) SPMX_TRY(ensure_csc_perm(h));
  cudaStream_t st = h->stream;
  if (d_dvals) SPMX_CUDA(cudaMemsetAsync(d_dvals, 0, 4 * (size_t)std::max(h->nnz, 0), st));
  SPMX_CUDA(cudaMemsetAsync(h->batch_work, 0, 4, st));
  note_launch();
  spmspv_batched_kernel<false><<<batched_grid(h), kBatchNT, 0, st>>>(
      h->m, h->n, nvec, d_xptr, d_xkey, d_xval, h->csc_colptr, h->csc_row, h->csc_val, h->csc_perm, alpha,
      nullptr, d_dY, d_dxval, d_dvals, h->batch_work, h->d_err);
  return launch_ok("batched spmspv backward");
}
