// Host-side launchers of the spmx kernels (implemented in the .cu files of
// this directory).  All launches are asynchronous on the given stream.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace spmx {

// number of kernels this library has launched (all handles, all threads)
void note_launch(int k = 1);

struct SpmvArgs {
  int m, n, nnz;
  const int* rowptr;
  const int* col;
  const float* val;
  const float* x;
  const int* bits;  // non-NULL selects the bitmap-gated SpMSpV form
  double alpha;
  float* y;
  int* err;
};

struct HolaTables {
  int vt;        // nonzeros per thread (4, 8 or 16); 256 threads per CTA
  int K;         // nonzeros per CTA = 256 * vt
  int nchunks;   // ceil(nnz / K)
  int* chunk_row;  // [nchunks + 1]
  double* carry;   // [2 * nchunks]
  unsigned* arrive;  // [nchunks], zero between calls
};

// ---- spmv.cu
int launch_spmv_naive(const SpmvArgs& a, int group, cudaStream_t st);
int launch_spmv_hola(const SpmvArgs& a, const HolaTables& t, cudaStream_t st);
int launch_chunk_rows(int m, const int* rowptr, int K, int nchunks,
                      int* chunk_row, cudaStream_t st);
int hola_chunk_nnz(int vt);

// ---- adjoint.cu
int launch_spmv_backward(int m, int n, int nnz, const int* rowptr, const int* col,
                         const float* val, const float* x, const float* dy,
                         const HolaTables& t, float* dx, float* dvals, int* err,
                         cudaStream_t st);
int launch_spmv_backward_csc(int m, int n, const int* rowptr, const int* col, const int* colptr,
                             const int* crow, const float* cval, const float* x, const float* dy,
                             int g1, int g2, float* dx, float* dvals, int* err, cudaStream_t st);
int launch_spmv_backward_sparse(int m, int n, const int* rowptr, const int* col,
                                const float* val, const float* x, int dy_nnz,
                                const int* dy_key, const float* dy_val, int group,
                                float* dx, float* dvals, int* err, cudaStream_t st);

// ---- lookback scratch shared by the single-pass scans
struct ScanScratch {
  unsigned long long* status;  // tile status words
  int status_len;              // capacity in tiles
  unsigned* ticket;            // 4 words, zeroed once: ticket, epoch, publish count
  unsigned* counts;            // status_len per-range counts (the compaction's first pass)
};

// indices into the handle's device counter block
enum CounterSlot : int {
  kCntYnnz = 0,
  kCntBinlen = 1,
  kCntXnnz = 2,
  kCntBlocksTL = 3,
  kCntBlocksMG = 4,
  kCntFeatSum = 8,   // 64-bit (slots 8..9)
  kCntFeatMax = 10,
  kCntFeatMinInv = 11,
  kCntTotal = 16
};

// ---- csc.cu
struct CscArgs {
  int m, n;
  const int* colptr;   // [n+1]
  const int* row;      // [nnz]
  const float* val;    // [nnz]
  int x_nnz;
  const int* x_key;
  const float* x_val;
  double alpha;
  int* err;
  int* counts;         // device counter block
};

struct CscScratch {
  int* off;        // [x_nnz + 1] exclusive scan of column lengths
  int* colstart;   // [x_nnz]     colptr[x_key[i]]
  int* bstart_tl;  // block -> first x entry (fixed nnz per block)
  int* bstart_mg;  // block -> first x entry (merge-path items)
  int tl_cap, mg_cap;  // capacities of the two tables
};

constexpr int kCscScanNT = 256, kCscScanVT = 8;   // 2048 x entries per tile
constexpr int kCscLbNT = 256, kCscLbVT = 8;       // 2048 items per LB block

int launch_csc_scan(const CscArgs& a, const CscScratch& s, ScanScratch& ls,
                    int block_items, cudaStream_t st);
// variant: 1 merge, 2 twolayer.  pairs_row/pairs_val non-NULL: write (row,
// alpha*val*x) pairs at their scanned position instead of atomics into y.
int launch_csc_lb(const CscArgs& a, const CscScratch& s, int variant, float* y,
                  int* pairs_row, float* pairs_val, int grid, cudaStream_t st);
int launch_csc_naive(const CscArgs& a, int group, float* y, cudaStream_t st);
// y = 0 then the naive CSC SpMSpV, as a programmatic dependent launch pair
int launch_csc_naive_zeroed(const CscArgs& a, int group, float* y, int num_sms, cudaStream_t st);
int launch_csc_naive_pairs(const CscArgs& a, const CscScratch& s, int group,
                           int* pairs_row, float* pairs_val, cudaStream_t st);

// ---- vecconv.cu
// y[0..m) = 0 with a kernel that lets the next grid launch early
int launch_zero_fill(float* y, long long m, int num_sms, cudaStream_t st);
// dense[0..len) from (key, val): a zero fill, then the scatter as a
// programmatic dependent launch that reads its keys and values while the
// fill runs; the scatter in turn lets the next grid start early
int launch_dense_from_sparse(int nvals, int len, const int* key, const float* val, float* dense,
                             int* err, int num_sms, cudaStream_t st);
int launch_scatter(int nvals, int len, const int* key, const float* val,
                   float* dense, int* bits, int* err, cudaStream_t st);
int launch_dense2bits(int len, const float* dense, int* bits, cudaStream_t st);
// keys/vals of the entries != 0 of dense[0..len), in order; count -> *d_count
int launch_compact_nonzero(int len, const float* dense, int* key, float* val,
                           int* d_count, ScanScratch& ls, int* err,
                           cudaStream_t st);

}  // namespace spmx
