// Device COO -> CSR for a handle: the GPU side of matrix ingestion.  It
// replaces the host std::sort by (row, col) after ReadMTX
// (hice-spmspv/hice/la/include/spmspv/mtx.hpp:335-360) and the cuSPARSE
// coo2csr of the reference's drivers.
//
// 1. coo_check_kernel: range check of every index, and whether the entries
//    are already in (row, col) order, or at least in non-decreasing column
//    order (a column-major file such as a SuiteSparse export).
// 2. stable LSD radix sort (sort.cu): by column, skipped when the columns are
//    already non-decreasing, then by row, both skipped when the input is
//    already in (row, col) order.  Stability keeps duplicates in input order.
// 3. coo_rowptr_kernel: position i writes the row pointers of the rows that
//    start there (rows[i-1]+1 .. rows[i]); every rowptr entry is written
//    once, empty rows included, with no atomics and no search.
#include <algorithm>

#include "common.cuh"
#include "engine.h"
#include "sort.h"

namespace spmx {
namespace {

constexpr int kIngestNT = 256;

__global__ void __launch_bounds__(kIngestNT)
coo_check_kernel(int nnz, int m, int n, const int* __restrict__ row,
                 const int* __restrict__ col, int* __restrict__ flags) {
  int oob = 0, unsorted = 0, col_desc = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nnz;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = __ldg(row + i), c = __ldg(col + i);
    oob |= (unsigned)r >= (unsigned)m || (unsigned)c >= (unsigned)n;
    if (i > 0) {
      const int rp = __ldg(row + i - 1), cp = __ldg(col + i - 1);
      unsorted |= rp > r || (rp == r && cp > c);
      col_desc |= cp > c;
    }
  }
  oob = __syncthreads_or(oob);
  unsorted = __syncthreads_or(unsorted);
  col_desc = __syncthreads_or(col_desc);
  if (threadIdx.x == 0) {
    if (oob) atomicOr(flags + 0, 1);
    if (unsorted) atomicOr(flags + 1, 1);
    if (col_desc) atomicOr(flags + 2, 1);
  }
}

__global__ void __launch_bounds__(kIngestNT)
coo_rowptr_kernel(int nnz, int m, const int* __restrict__ rows, int* __restrict__ rowptr) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i <= nnz;
       i += (long long)gridDim.x * blockDim.x) {
    const int lo = i == 0 ? 0 : __ldg(rows + i - 1) + 1;
    const int hi = i == nnz ? m : __ldg(rows + i);
    for (int r = lo; r <= hi; ++r) rowptr[r] = (int)i;
  }
}

int ingest_grid(long long work) {
  const long long g = (work + kIngestNT - 1) / kIngestNT;
  return (int)std::max<long long>(1, std::min<long long>(g, 148LL * 16));
}

int key_bits(int extent) {
  int b = 1;
  while (b < 31 && (1LL << b) < extent) ++b;
  return b;
}

}  // namespace
}  // namespace spmx

using namespace spmx;

extern "C" int spmx_input_coo(spmx_handle_t h, int nnz, const int* row, const int* col,
                              const float* val) {
  SPMX_CHECK_HANDLE(h);
  if (nnz != h->nnz) return set_error(SPMX_ERR_INVALID_VALUE, "nnz differs from the handle's nnz");
  if (nnz > 0 && (!row || !col)) return set_error(SPMX_ERR_INVALID_VALUE, "NULL COO array");
  const int m = h->m, n = h->n;
  cudaStream_t st = h->stream;
  const size_t b = 4 * (size_t)std::max(nnz, 1);

  // 1. range and order check (synchronous: the result picks the sort passes)
  int* flags = nullptr;
  SPMX_TRY(dalloc((void**)&flags, 4 * sizeof(int), "coo flags"));
  int oob = 0, unsorted = 0, col_desc = 0;
  cudaError_t ce = cudaMemsetAsync(flags, 0, 4 * sizeof(int), st);
  if (ce == cudaSuccess && nnz > 0) {
    note_launch();
    coo_check_kernel<<<ingest_grid(nnz), kIngestNT, 0, st>>>(nnz, m, n, row, col, flags);
    ce = cudaGetLastError();
  }
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(h->h_pinned, flags, 3 * sizeof(int), cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  dfree(flags);
  if (ce != cudaSuccess) return set_error(SPMX_ERR_CUDA, std::string("coo check: ") + cudaGetErrorString(ce));
  if (nnz > 0) {
    oob = h->h_pinned[0];
    unsorted = h->h_pinned[1];
    col_desc = h->h_pinned[2];
  }
  if (oob) return set_error(SPMX_ERR_INVALID_VALUE, "COO index out of range");

  // 2. the new CSR (swapped in only on success).  The radix passes alternate
  // between two buffer sets; the pass count is known here, so the set the
  // last pass writes is the new CSR's column / value arrays themselves.  All
  // other scratch is one allocation.
  int *nrp = nullptr, *ncol = nullptr;
  float* nval = nullptr;
  int rc = SPMX_SUCCESS;
  rc = rc ? rc : dalloc((void**)&nrp, 4 * ((size_t)m + 1), "csr rowptr");
  rc = rc ? rc : dalloc((void**)&ncol, b, "csr col");
  if (val) rc = rc ? rc : dalloc((void**)&nval, b, "csr val");
  char* scratch = nullptr;
  const int* rows_sorted = row;
  const void* cols_sorted = col;
  const void* vals_sorted = val;
  if (!rc && unsorted) {
    const int bits_c = key_bits(n), bits_r = key_bits(m);
    const int passes = (col_desc ? (bits_c + 7) / 8 : 0) + (bits_r + 7) / 8;
    const int fin = passes & 1;  // set holding the result after the last pass
    const size_t hn = radix_hist_ints(nnz);
    const size_t al = (b + 255) & ~(size_t)255;
    const size_t hb = (4 * hn + 255) & ~(size_t)255;
    rc = dalloc((void**)&scratch, al * (val ? 4 : 3) + 2 * hb, "coo sort scratch");
    if (!rc) {
      unsigned *k[2], *r[2], *v[2] = {nullptr, nullptr};
      char* q = scratch;
      k[fin] = (unsigned*)ncol;
      k[1 - fin] = (unsigned*)q; q += al;
      r[0] = (unsigned*)q; q += al;
      r[1] = (unsigned*)q; q += al;
      if (val) {
        v[fin] = (unsigned*)nval;
        v[1 - fin] = (unsigned*)q; q += al;
      }
      int* hist = (int*)q; q += hb;
      int* hoff = (int*)q;
      cudaMemcpyAsync(k[0], col, 4 * (size_t)nnz, cudaMemcpyDeviceToDevice, st);
      cudaMemcpyAsync(r[0], row, 4 * (size_t)nnz, cudaMemcpyDeviceToDevice, st);
      if (val) cudaMemcpyAsync(v[0], val, 4 * (size_t)nnz, cudaMemcpyDeviceToDevice, st);
      int s = 0;  // set holding the current order
      if (col_desc) {
        RadixBuffers ra{k[s], k[1 - s], r[s], r[1 - s], v[s], v[1 - s], hist, hoff, false};
        if (radix_sort_pairs(ra, nnz, bits_c, h->ls, h->d_err, st))
          rc = set_error(SPMX_ERR_INVALID_VALUE, "radix capacity");
        if (ra.result_in_alt) s = 1 - s;
      }
      if (!rc) {
        RadixBuffers rb{r[s], r[1 - s], k[s], k[1 - s], v[s], v[1 - s], hist, hoff, false};
        if (radix_sort_pairs(rb, nnz, bits_r, h->ls, h->d_err, st))
          rc = set_error(SPMX_ERR_INVALID_VALUE, "radix capacity");
        if (rb.result_in_alt) s = 1 - s;
      }
      if (!rc && s != fin) rc = set_error(SPMX_ERR_INVALID_VALUE, "radix pass count");
      rows_sorted = (const int*)r[s];
      cols_sorted = k[s];
      vals_sorted = v[s];
    }
  }
  // 3. row pointers from the sorted rows; columns and values into place
  if (!rc) {
    note_launch();
    coo_rowptr_kernel<<<ingest_grid((long long)nnz + 1), kIngestNT, 0, st>>>(nnz, m, rows_sorted, nrp);
    if (nnz > 0 && cols_sorted != ncol) {
      cudaMemcpyAsync(ncol, cols_sorted, 4 * (size_t)nnz, cudaMemcpyDeviceToDevice, st);
      if (val) cudaMemcpyAsync(nval, vals_sorted, 4 * (size_t)nnz, cudaMemcpyDeviceToDevice, st);
    }
    ce = cudaGetLastError();
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) rc = set_error(SPMX_ERR_CUDA, std::string("coo to csr: ") + cudaGetErrorString(ce));
  } else {
    cudaStreamSynchronize(st);
  }
  dfree(scratch);
  if (rc) {
    dfree(nrp);
    dfree(ncol);
    dfree(nval);
    return rc;
  }
  dfree(h->own_csr_rowptr);
  dfree(h->own_csr_col);
  dfree(h->own_csr_val);
  h->own_csr_rowptr = nrp;
  h->own_csr_col = ncol;
  h->own_csr_val = nval;
  h->rowptr = nrp;
  h->col = ncol;
  h->val = nval;
  h->has_csr = true;
  h->mat_feat_ready = false;
  h->std_row_ready = false;
  // a CSC derived from the previous CSR by spmx_to_csc is stale now
  if (h->has_csc && h->csc_colptr == h->own_colptr) h->has_csc = false;
  return SPMX_SUCCESS;
}

extern "C" int spmx_copy_csr(spmx_handle_t h, int* rowptr, int* col, float* val) {
  SPMX_CHECK_HANDLE(h);
  if (!h->has_csr) return set_error(SPMX_ERR_NOT_READY, "no CSR (call spmx_input_csr or spmx_input_coo)");
  cudaStream_t st = h->stream;
  if (rowptr)
    SPMX_CUDA(cudaMemcpyAsync(rowptr, h->rowptr, 4 * ((size_t)h->m + 1), cudaMemcpyDeviceToDevice, st));
  if (col && h->nnz)
    SPMX_CUDA(cudaMemcpyAsync(col, h->col, 4 * (size_t)h->nnz, cudaMemcpyDeviceToDevice, st));
  if (val && h->val && h->nnz)
    SPMX_CUDA(cudaMemcpyAsync(val, h->val, 4 * (size_t)h->nnz, cudaMemcpyDeviceToDevice, st));
  return SPMX_SUCCESS;
}
