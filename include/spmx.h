/*
 * spmx.h — C ABI of the B200-native adaptive SpMV / SpMSpV engine.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, returns an
 * int status (SPMX_SUCCESS == 0) and never exits the process.  Pointers named
 * d_* are device pointers; everything else is host memory.  Index type is
 * int32, value type is float32 (the reference's SpmspvHandle<int, unsigned,
 * float> instantiation).
 *
 * Each declaration names the reference interface it replaces, as a path inside
 * hpc-research-2020/spmspv-adaptive, abbreviated:
 *   H    = hice-spmspv/hice/la/include/spmspv/csc-spmspv/spmspv.h
 *   DEV  = hice-spmspv/hice/la/include/spmspv/csc-spmspv/detail/device/
 *   TEST = hice-spmspv/hice/la/test/
 *   INC  = hice-spmspv/hice/la/include/spmspv/
 *
 * Ownership follows the reference: CSR arrays and x buffers are caller-owned
 * device memory; CSC built by spmx_to_csc, Hola / CSR5 tables and scratch are
 * handle-owned.  Unlike the reference, a CSC passed with spmx_input_csc is
 * borrowed and never freed by the handle (H:2870-2876 frees it regardless).
 *
 * Streams: all work of a handle is issued on one stream (spmx_set_stream,
 * default: the legacy default stream).  Entry points do not synchronise unless
 * a HOST output pointer (e.g. `int* ynnz`) is non-NULL; device-side counts are
 * always also available through spmx_get_device_counts.
 */
#ifndef SPMX_H_
#define SPMX_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes: the reference's SPMSPV_* values are kept (common.h:11-26) */
#define SPMX_SUCCESS                   0
#define SPMX_UNKNOWN_FORMAT           -1
#define SPMX_UNSUPPORTED_CSR_SPMV     -2
#define SPMX_UNSUPPORTED_VALUE_TYPE   -3
#define SPMX_UNSUPPORTED_CSR_SPMSPV   -4
#define SPMX_UNSUPPORTED_COO_SPMSPV   -5
#define SPMX_FORMAT_ERR_HOLA_SPMV     -6
#define SPMX_MAT_FORMAT_ERR          -13
#define SPMX_VEC_FORMAT_ERR          -14
/* additions */
#define SPMX_ERR_INVALID_VALUE       -20  /* bad argument (size, NULL, range)   */
#define SPMX_ERR_CUDA                -21  /* a CUDA runtime call failed          */
#define SPMX_ERR_TIMEOUT             -22  /* a bounded device wait gave up       */
#define SPMX_ERR_OOB                 -23  /* device bounds check tripped         */
#define SPMX_ERR_ALLOC               -24  /* device allocation failed            */
#define SPMX_ERR_NOT_READY           -25  /* missing input / preprocess step     */
#define SPMX_ERR_NO_DEVICE           -26  /* no CUDA device visible              */

/* ---- vector type codes, as in set_vector_type (H:979): 0 sparse, 1 dense, 2 bitarray */
#define SPMX_VEC_SPARSE   0
#define SPMX_VEC_DENSE    1
#define SPMX_VEC_BITARRAY 2

/* ---- SpMV back-ends for spmx_spmv / spmx_spmspv (set_spmv_type, H:1767) */
#define SPMX_SPMV_HOLA 0
#define SPMX_SPMV_CSR5 1
#define SPMX_SPMV_TILED 2  /* row-block x column-window tiles (no reference counterpart) */
#define SPMX_SPMV_ROUND 3  /* column-ordered rounds, row-owner reduction (no reference counterpart) */

/* ---- CSC SpMSpV work distributions and write-backs (H:1824-2201) */
#define SPMX_CSC_NAIVE     0  /* group of threads per x nonzero            */
#define SPMX_CSC_LB_MERGE  1  /* merge-path partition over (x entries, nnz) */
#define SPMX_CSC_LB_TWOLAYER 2/* fixed nnz per CTA, block-start table      */
#define SPMX_CSC_BUCKET    3  /* row-block buckets, no global atomics      */
#define SPMX_WB_ATOMIC     0  /* dense y via atomics (+ optional compaction)*/
#define SPMX_WB_SORT       1  /* (row,val) pairs -> sort -> reduce_by_key   */

/* ---- the eight adaptive kernels, in the reference's three-stage tree order
 *      (TEST/new_test_app.cu:406-456): solution x workload x write-back      */
#define SPMX_K_CSC_NAIVE_SORT    0
#define SPMX_K_CSC_NAIVE_ATOMIC  1
#define SPMX_K_CSC_LB_SORT       2
#define SPMX_K_CSC_LB_ATOMIC     3
#define SPMX_K_CSR_NAIVE_SPMSPV  4
#define SPMX_K_CSR_LB_SPMSPV     5
#define SPMX_K_NAIVE_SPMV        6
#define SPMX_K_LB_SPMV           7
#define SPMX_NUM_KERNELS         8

/* number of entries of the feature vector written by spmx_features; the order
 * is the reference's 23-feature schema (model/1-test_dtree.py:63):
 * m,n,nnz,maxRow,minRow,avgRow,range,stdRow,edge_equlity,gini,x_nnz,bin_len,
 * max,min,xnnz/n,bin_len/nnz,xnnz_range,GM1,GM2,GM3,GM1/GM2,GM2/GM3,GM1/GM3 */
#define SPMX_NUM_FEATURES 23

typedef struct spmx_handle_s* spmx_handle_t;

/* ======================= lifecycle ======================================= */
/* SpmspvHandle(m, n, nnz) — H:91-141 */
int spmx_create(int m, int n, int nnz, spmx_handle_t* out);
/* Destroy() — H:2866-2887 (frees only handle-owned memory) */
int spmx_destroy(spmx_handle_t h);
/* no reference counterpart (the reference uses stream 0 everywhere) */
int spmx_set_stream(spmx_handle_t h, void* cuda_stream);
/* warmup() — H:347 */
int spmx_warmup(spmx_handle_t h);
/* number of kernels the library has launched so far (all handles); no
 * reference counterpart */
unsigned long long spmx_launch_count(void);
/* thread-local text of the last error; never NULL */
const char* spmx_last_error_string(void);
/* sticky device error word of the handle (bounded waits, bounds checks);
 * reading it synchronises the handle's stream and clears it */
int spmx_check_device_error(spmx_handle_t h);

/* ======================= matrix input ==================================== */
/* InputCSR(nnz, csr_row, csr_col, csr_val) — H:356-366; csr_row = row pointer
 * [m+1], csr_col = column indices [nnz]; d_csr_val may be NULL (pattern only,
 * used by BFS) */
int spmx_input_csr(spmx_handle_t h, int nnz, const int* d_csr_row,
                   const int* d_csr_col, const float* d_csr_val);
/* InputCSC(nnz, csc_row, csc_col, csc_val) — H:369-379; csc_row = row indices
 * [nnz], csc_col = column pointer [n+1] (borrowed) */
int spmx_input_csc(spmx_handle_t h, int nnz, const int* d_csc_row,
                   const int* d_csc_col, const float* d_csc_val);
/* ToCSC() — H:384-419 (cusparseScsr2csc there).  Handle-owned CSC with row
 * indices sorted inside each column (a stable transpose). */
int spmx_to_csc(spmx_handle_t h);
/* copy the handle's CSC into caller buffers (row[nnz], colptr[n+1],
 * val[nnz]; any may be NULL); asynchronous on the handle's stream */
int spmx_copy_csc(spmx_handle_t h, int* d_row, int* d_colptr, float* d_val);
/* COO (device arrays, any order, duplicates kept) -> handle-owned CSR sorted
 * by (row, col), duplicates in input order.  The GPU replacement of the host
 * sort after ReadMTX (mtx.hpp:335-360) and the coo2csr of the reference's
 * drivers.  Synchronous; d_val may be NULL (pattern).  An index outside
 * [0,m) x [0,n) returns SPMX_ERR_INVALID_VALUE and leaves the handle as it
 * was.  Replaces the handle's CSR like spmx_input_csr (a CSC derived from
 * the previous CSR by spmx_to_csc is dropped). */
int spmx_input_coo(spmx_handle_t h, int nnz, const int* d_row, const int* d_col,
                   const float* d_val);
/* copy the handle's CSR into caller buffers (rowptr[m+1], col[nnz],
 * val[nnz]; any may be NULL); asynchronous on the handle's stream */
int spmx_copy_csr(spmx_handle_t h, int* d_rowptr, int* d_col, float* d_val);
/* read access to the handle's CSC (device pointers, valid until destroy) */
int spmx_get_csc(spmx_handle_t h, const int** d_csc_row, const int** d_csc_col,
                 const float** d_csc_val);

/* ======================= vectors ========================================= */
/* set_x — H:985 */
int spmx_set_x(spmx_handle_t h, float* d_x);
/* set_sparse_x — H:992-1002 */
int spmx_set_sparse_x(spmx_handle_t h, int* d_x_key, float* d_x_val, int xnnz);
/* set_bitvector — H:1005-1011 (num_ints = ceil(n/32)) */
int spmx_set_bitvector(spmx_handle_t h, int* d_bitvector, int num_ints);
/* set_sparse_x_dense_x — H:1014-1025 */
int spmx_set_sparse_x_dense_x(spmx_handle_t h, int* d_x_key, float* d_x_val,
                              float* d_x_dense, int xnnz);
/* set_vector_type — H:979 */
int spmx_set_vector_type(spmx_handle_t h, int code);

/* sparse2dense — H:1240-1268 (memset + scatter) */
int spmx_sparse2dense(spmx_handle_t h);
/* sparse2bitarray — H:1271-1308 (dense x and bitarray from sparse x) */
int spmx_sparse2bitarray(spmx_handle_t h);
/* dense2sparse — H:1177-1222.  Writes x's key/val buffers from the dense x and
 * updates the handle's x_nnz (the reference leaves it stale); if xnnz != NULL
 * the count is also returned to the host (synchronises). */
int spmx_dense2sparse(spmx_handle_t h, int* xnnz);
/* bitarray2sparse — H:1311-1351 (same compaction, from the dense x) */
int spmx_bitarray2sparse(spmx_handle_t h, int* xnnz);
/* dense2bitarray — H:1373-1388, kernel H:1355.  Sets the bit of every NONZERO entry (the
 * reference sets bits of zeros, H:1362). */
int spmx_dense2bitarray(spmx_handle_t h);
/* dense2sparse_outer — H:1953-1998 (no cudaMalloc per call here) */
int spmx_dense2sparse_outer(spmx_handle_t h, int m, const float* d_dense,
                            int* ynnz, int* d_key, float* d_val);
/* dense2sparse_outer — H:1953-1998, with the result written straight into
 * host memory: the nonzeros of d_dense[m] (in index order) go to h_key /
 * h_val and their count to *h_count, all three page-locked host buffers
 * mapped into the device's address space (cudaHostAlloc / cudaMallocHost on
 * a unified-addressing system; anything else is rejected).  No host
 * synchronisation: the values are there once the handle's stream has
 * reached this call (synchronise it, or wait on an event, before reading).
 * h_key / h_val need room for m entries. */
int spmx_dense2sparse_to_host(spmx_handle_t h, int m, const float* d_dense, int* h_key,
                              float* h_val, int* h_count);
/* sparse2dense_outer — H:1931-1950 */
int spmx_sparse2dense_outer(spmx_handle_t h, int ynnz, const int* d_key,
                            const float* d_val, int m, float* d_dense);

/* ======================= scratch / preprocess ============================= */
/* allocPreBuffer / deallocPreBuffer — H:1726-1763, H:2849-2864.  Sizes the scratch for the
 * worst case (bin_len = nnz) so later calls never allocate. */
int spmx_alloc_pre_buffer(spmx_handle_t h);
int spmx_dealloc_pre_buffer(spmx_handle_t h);
/* holaPreprocess / holaPostprocess — H:1654-1672 (block-start table) */
int spmx_hola_preprocess(spmx_handle_t h);
int spmx_hola_postprocess(spmx_handle_t h);
/* setSigma / CSR5Preprocess / CSR5Postprocess — H:1396-1651.  sigma = -1
 * selects the reference's auto rule (H:1396-1416). */
int spmx_set_sigma(spmx_handle_t h, int sigma);
int spmx_csr5_preprocess(spmx_handle_t h);
int spmx_csr5_postprocess(spmx_handle_t h);
/* the sigma in use (after CSR5Preprocess) or that the auto rule would pick */
int spmx_csr5_sigma(spmx_handle_t h, int* sigma);
/* Tiled SpMV format (no reference counterpart; a third back-end for
 * spmv / spmspv): rows cut into blocks whose y fits in shared memory (at
 * most rb_rows rows; 0 = as many as fit), columns into windows of win
 * entries of x (a multiple of 128, <= 65536; 0 = 8192), tiles cut into
 * stages of at most chunk nonzeros (0 = 2048); warps = row-owning warps per
 * CTA (4, 8 or 16; 0 = 8).  Each stage's x window and
 * nonzeros are streamed into shared memory with bulk copies; a row block is
 * shared by a cluster of CTAs whose partial y vectors are combined through
 * distributed shared memory.  The result is deterministic. */
int spmx_tiled_preprocess(spmx_handle_t h, int rb_rows, int win, int chunk, int warps);
int spmx_tiled_postprocess(spmx_handle_t h);
/* geometry chosen by spmx_tiled_preprocess: info[0..7] = row blocks, CTAs
 * per cluster, stages, win, chunk, shared y rows, shared bytes, row warps */
int spmx_tiled_info(spmx_handle_t h, int* info);
int spmx_tiledspmv(spmx_handle_t h, float alpha, float* d_y);
int spmx_tiledspmspv(spmx_handle_t h, float alpha, float* d_y);
/* Round SpMV / bitmap-gated SpMSpV (no reference counterpart; a fourth
 * back-end for the load-balanced SpMV of the selector, spmv_type 3).  Rows
 * are cut into row blocks (at most rb_rows rows; 0 = as many as fit), one per
 * CTA (spmx_round_preprocess_parts below has the clustered layouts); a CTA
 * streams its block's nonzeros sorted by (column, row) in rounds of 4096.  Every row owns as many shared-memory
 * accumulators as it has nonzeros in its densest round; the k-th nonzero of
 * a row in a round adds into the row's k-th accumulator with a plain
 * read-modify-write (all distinct within a round), one barrier per round;
 * at the end each row's accumulators are summed.  Deterministic.  When a
 * row block needs more accumulators than shared memory holds, the
 * preprocessing retries with row blocks half as tall (up to 5 times).  Fails
 * with SPMX_ERR_INVALID_VALUE (the other back-ends still apply) when a column
 * index is out of range, when the accumulators still do not fit, or when
 * row blocks x columns need a sort key of more than 32 bits.  When 128
 * consecutive nonzeros of a row block (a very sparse row block) span 2^16
 * columns or more, the format is rebuilt with every 2^16-column segment
 * starting a new 128-entry chunk. */
int spmx_round_preprocess(spmx_handle_t h, int rb_rows);
/* No reference counterpart.  The round format with `parts` CTAs per row
 * block: 1 (what spmx_round_preprocess builds: one CTA per row block over all
 * columns, no cluster, each row's accumulators summed straight into y; the
 * fastest layout measured), 2 (one 2-CTA cluster per row block, twice as
 * tall, each CTA over half the columns, the row sums combined through
 * distributed shared memory) or 4 (two clusters per row block, each row block
 * four times as tall, the
 * row sums folded into each row's first accumulator slot; the two clusters'
 * sums meet in a small device buffer and the second to finish a row slice
 * stores y, so every row is still added in a fixed order).  Taller row blocks
 * put more nonzeros on each column range of x, so fewer x cache lines are
 * gathered per nonzero. */
int spmx_round_preprocess_parts(spmx_handle_t h, int rb_rows, int parts);
int spmx_round_postprocess(spmx_handle_t h);
/* geometry chosen by spmx_round_preprocess(_parts): info[0..7] = row blocks,
 * CTAs per row block (1, 2 or 4; clusters, where used, are 2 CTAs), rounds, nonzeros
 * per round, accumulator slots per CTA, rows per row block (at most), shared
 * bytes, grid */
int spmx_round_info(spmx_handle_t h, int* info);
int spmx_roundspmv(spmx_handle_t h, float alpha, float* d_y);
int spmx_roundspmspv(spmx_handle_t h, float alpha, float* d_y);
/* Hybrid CSR/CSC split (a candidate ninth kernel; the reference's
 * COO2Hybrid, INC/mtx.hpp:436-701, driven by TEST/test_coo2hybrid.cu:276-312).
 * Preprocess: copies the CSR to the host and visits the nonzeros in (row,
 * column) order with the current row and column counts: a nonzero joins the
 * CSR part when count_row >= count_col (count_col is then decremented), else
 * the CSC part (count_row decremented).  Row priority only (the reference's
 * column-priority branch swaps its row and column indices).  hybridspmv:
 * y = alpha * (A_csr x + A_csc x), the CSC part added with FP32 atomics. */
int spmx_hybrid_preprocess(spmx_handle_t h);
int spmx_hybrid_postprocess(spmx_handle_t h);
/* nonzeros in the CSR and CSC parts */
int spmx_hybrid_info(spmx_handle_t h, int* csr_nnz, int* csc_nnz);
/* copy the parts into caller buffers (CSR: rowptr[m+1], col, val; CSC:
 * colptr[n+1], row, cval; any may be NULL); asynchronous on the stream */
int spmx_hybrid_copy(spmx_handle_t h, int* d_rowptr, int* d_col, float* d_val, int* d_colptr,
                     int* d_row, float* d_cval);
int spmx_hybridspmv(spmx_handle_t h, float alpha, float* d_y);
/* set_spmv_type — H:1767 (0 Hola, 1 CSR5, 2 tiled, 3 round) */
int spmx_set_spmv_type(spmx_handle_t h, int code);

/* ======================= SpMV / CSR SpMSpV (y = alpha*A*x) =============== */
/* naivespmv — H:1677-1684, DEV/naivespmv.h:34 */
int spmx_naivespmv(spmx_handle_t h, float alpha, float* d_y);
/* holaspmv — H:1687-1698, DEV/holaspmv.h:2070 */
int spmx_holaspmv(spmx_handle_t h, float alpha, float* d_y);
/* csr5spmv — H:1586-1605, DEV/csr5_spmv_cuda.h:440 */
int spmx_csr5spmv(spmx_handle_t h, float alpha, float* d_y);
/* naivespmspv — H:1701-1706, DEV/naivespmv.h:13 (x gated by the bitarray) */
int spmx_naivespmspv(spmx_handle_t h, float alpha, float* d_y);
/* holaspmspv — H:1709-1721, DEV/holaspmv.h:2224 */
int spmx_holaspmspv(spmx_handle_t h, float alpha, float* d_y);
/* csr5spmspv — H:1607-1627, DEV/csr5_spmspv.h:450 */
int spmx_csr5spmspv(spmx_handle_t h, float alpha, float* d_y);
/* spmv / spmspv dispatch by spmv_type — H:1790-1821 */
int spmx_spmv(spmx_handle_t h, float alpha, float* d_y);
int spmx_spmspv(spmx_handle_t h, float alpha, float* d_y);

/* ======================= CSC SpMSpV (y = alpha*A*x, x sparse) ============= */
/* Generic form.  variant: SPMX_CSC_*, writeback: SPMX_WB_*.
 *  - atomic: d_y (dense, m) is overwritten; if d_y_key/d_y_val are non-NULL the
 *    nonzeros of y (entries != 0) are also compacted into them, in row order.
 *  - sort:   d_y_key/d_y_val receive the rows touched by x's columns, sorted,
 *    with their sums (zeros kept — reduce_by_key semantics); d_y may be NULL,
 *    otherwise it is also written densely.
 *  - bucket: as sort for the sparse output, plus dense d_y if non-NULL.
 * ynnz (host, may be NULL) receives the output count (synchronises). */
int spmx_spmspv_csc(spmx_handle_t h, int variant, int writeback, float alpha,
                    float* d_y, int* d_y_key, float* d_y_val, int* ynnz);
/* CscBasedNoSortNaiveSpmspv — H:2119-2139 */
int spmx_csc_naive_atomic(spmx_handle_t h, float alpha, int* ynnz, float* d_y);
/* CscBasedNoSortNaiveSpmspv_keyval — H:2143-2169 */
int spmx_csc_naive_atomic_keyval(spmx_handle_t h, float alpha, int* ynnz,
                                 float* d_y, int* d_y_key, float* d_y_val);
/* CscBasedSortNaiveSpmspv — H:2172-2201 */
int spmx_csc_naive_sort(spmx_handle_t h, float alpha, int* ynnz, int* d_y_key,
                        float* d_y_val);
/* CscBasedNoSortMergeSpmspv(_keyval) — H:2033-2088 (binlen_ready ignored:
 * bin_len never leaves the device here) */
int spmx_csc_merge_atomic(spmx_handle_t h, int binlen_ready, float alpha,
                          int* ynnz, float* d_y, int* d_y_key, float* d_y_val);
int spmx_csc_merge_atomic_keyval(spmx_handle_t h, int binlen_ready, float alpha,
                                 int* ynnz, float* d_y, int* d_y_key,
                                 float* d_y_val);
/* CscBasedSortMergeSpmspv — H:2091-2115 */
int spmx_csc_merge_sort(spmx_handle_t h, int binlen_ready, float alpha,
                        int* ynnz, float* d_y, int* d_y_key, float* d_y_val);
/* CscBasedMyNoSortSpmspv(_keyval) / CscBasedSortMySpmspv — H:1824-1878, H:2001-2029 */
int spmx_csc_twolayer_atomic(spmx_handle_t h, int binlen_ready, float alpha,
                             int* ynnz, float* d_y, int* d_y_key,
                             float* d_y_val);
int spmx_csc_twolayer_atomic_keyval(spmx_handle_t h, int binlen_ready,
                                    float alpha, int* ynnz, float* d_y,
                                    int* d_y_key, float* d_y_val);
int spmx_csc_twolayer_sort(spmx_handle_t h, int binlen_ready, float alpha,
                           int* ynnz, float* d_y, int* d_y_key, float* d_y_val);
/* CscBasedBucketSpmspvDriver — DEV/csc_bucket_spmspv.cuh:768-1087 (whose
 * reduction is disabled in the reference; completed here).  buckets <= 0
 * selects the tuned/default count. */
int spmx_csc_bucket(spmx_handle_t h, float alpha, int* ynnz, float* d_y,
                    int* d_y_key, float* d_y_val, int buckets);

/* No counterpart in the reference.  The load-balanced (merge-path) CSC
 * SpMSpV with atomic write-back, y = alpha*A*x, for callers that cannot let
 * the library allocate device memory (a host framework that owns the device
 * heap through its own allocator; a latency-critical loop in which cudaMalloc
 * / cudaFree could synchronise the device).  No handle: the caller passes the
 * CSC (csc_row = row indices [nnz], csc_col = column pointer [n+1]), the sparse
 * x and the dense output y[m]; all scratch lives in one fixed array of device
 * global memory (about 8.6 MB on every GPU that loads the library, held until
 * the process exits).  Limits: x_nnz <= 1,048,576 and nnz + x_nnz <=
 * 134,217,728; larger calls return SPMX_ERR_INVALID_VALUE without launching.
 * The first call on a device looks up the array's device address (make it
 * before any stream capture).  Calls share the array: calls that overlap on
 * the GPU race, so serialise them (e.g. on one stream).  Nothing is allocated,
 * no cudaMalloc / cudaFree is called; work is queued on `stream`. */
int spmx_spmspv_csc_noalloc(int m, int n, int nnz, const int* d_csc_row,
                            const int* d_csc_col, const float* d_csc_val,
                            int x_nnz, const int* d_x_key, const float* d_x_val,
                            float alpha, float* d_y, void* stream);
/* No counterpart in the reference.  Reads the device error word of the last
 * spmx_spmspv_csc_noalloc call on the current device: synchronises `stream`,
 * copies 4 bytes out of the fixed scratch array (nothing is allocated) and
 * returns SPMX_ERR_OOB for an x key outside [0, n) or a row index outside
 * [0, m) that the kernels skipped, SPMX_ERR_TIMEOUT for a bounded wait that
 * gave up, else SPMX_SUCCESS.  Call it after the SpMSpV call, on the same
 * stream, before the next one (each call clears the word). */
int spmx_spmspv_csc_noalloc_check(void* stream);

/* ======================= features / selector ============================== */
/* computeBinlenVer2 — H:2703-2723 (sum of the column lengths of x's keys) */
int spmx_compute_binlen(spmx_handle_t h, long long* bin_len);
/* computeGM1/2/3 — H:2727-2752 (needs bin_len) */
int spmx_compute_gm(spmx_handle_t h, double gm[3]);
/* computeMatFeture_serial — H:2275-2335, computed on the device:
 * out = {m, n, nnz, maxRow, minRow, avgRow, range, stdRow, edge_equlity, gini} */
int spmx_mat_features(spmx_handle_t h, double out[10]);
/* extractMatFeatureParallel — H:921-976 (stdRow with the int-truncated mean) */
int spmx_std_row(spmx_handle_t h, float* std_row);
/* computeVecFeture_serial — H:2338-2361 without the per-call colptr copy:
 * out = {bin_len, max, min} */
int spmx_vec_features(spmx_handle_t h, long long out[3]);
/* full 23-entry feature vector (SPMX_NUM_FEATURES order above) */
int spmx_features(spmx_handle_t h, double out[SPMX_NUM_FEATURES]);
/* predictSolution / predictWorkloadDistribution / predictWritingBack —
 * TEST/new_test_app.cu:121-131 (stubs there); a decision tree here.
 * kernel_id receives one of SPMX_K_*. */
int spmx_select(spmx_handle_t h, int* kernel_id);
/* the feature vector spmx_select decides on: the 23-entry schema with the
 * host-known values (bin_len estimated as x_nnz*nnz/n unless measured, the
 * matrix's longest column in the "max" slot, 0 in the "min" slot) */
int spmx_selector_inputs(spmx_handle_t h, double out[SPMX_NUM_FEATURES]);
/* the selector on a caller-supplied feature vector (host only, no handle, no
 * GPU): predictSolution / predictWorkloadDistribution / predictWritingBack
 * combined (TEST/new_test_app.cu:121-131) */
int spmx_select_features(const double f[SPMX_NUM_FEATURES], int* kernel_id);
/* the adaptive iteration of TEST/new_test_app.cu:349-465 (#if 0 there):
 * select, convert x as the chosen kernel needs (s2d / s2a), run it.
 * d_y (dense, m) always receives y; kernel_used (host, may be NULL). */
int spmx_run_adaptive(spmx_handle_t h, float alpha, float* d_y, int* kernel_used);
/* Per-matrix autotuner (no reference counterpart beyond the reference's
 * Hola-vs-CSR5 timing, TEST/generate_model_data.cu:487-516): times the
 * load-balanced SpMV back-ends (Hola 4/8/16 nonzeros per thread, CSR5, tiled
 * geometries), the naive kernels' lanes per row / column, merge-path vs
 * fixed-nonzero CSC blocks and the bucket count, and keeps the fastest.
 * cache_path (may be NULL): a text file of tuned parameters keyed by a matrix
 * fingerprint; a hit applies them without timing.  spmv_type_out (may be NULL)
 * receives the chosen SpMV back-end. */
int spmx_autotune(spmx_handle_t h, const char* cache_path, int* spmv_type_out);
/* run one of the eight kernels by id (used by the exhaustive timing harness) */
int spmx_run_kernel(spmx_handle_t h, int kernel_id, float alpha, float* d_y);
/* The naive kernels' lanes per row (CSR SpMV) and per column (CSC SpMSpV),
 * as the autotuner sets them (no reference counterpart: the reference fixes
 * one thread per row / column, DEV/csc_sort_spmspv.cuh:98-119).  Each is 0
 * (derived from the mean row / column length) or 1, 2, 4, 8, 16, 32. */
int spmx_set_naive_lanes(spmx_handle_t h, int row_lanes, int col_lanes);

/* ======================= BFS (Boolean OR-AND semiring) ==================== */
/* The SpMSpV-driven BFS the replay loops of TEST/test_application.cu:240-415
 * and TEST/new_test_app.cu:280-469 stand in for.  Needs a symmetric pattern
 * (CSR; CSC is taken as the same arrays).  d_levels[n] receives hop counts,
 * -1 for unreachable; depth (host, may be NULL) the number of levels. */
int spmx_bfs(spmx_handle_t h, int source, int* d_levels, int* depth);
/* 0 (default): the whole traversal in one cooperative persistent launch with
 * the push/pull choice on the device; 1: one launch per level with the
 * frontier size read back by the host (the reference's replay-loop shape) */
int spmx_set_bfs_mode(spmx_handle_t h, int mode);
/* Batched BFS (no reference counterpart): up to 64 sources (host array) in
 * one persistent launch, one bit per source per vertex.  layout 0: d_levels
 * is vertex-major, d_levels[v * nsrc + s]; layout 1: source-major,
 * d_levels[s * n + v].  depth (host, may be NULL): levels of the deepest
 * traversal. */
int spmx_bfs_batched(spmx_handle_t h, const int* srcs, int nsrc, int* d_levels,
                     int layout, int* depth);

/* ======================= adjoint (FP32) ==================================== */
/* No reference counterpart (the reference has no differentiation).  For
 * y = A x and an upstream gradient dy[m]: dx[n] = A^T dy and dvals[nnz] =
 * dy[row_k] * x[col_k] on the CSR pattern.  Either output may be NULL.
 * With a CSC on the handle (spmx_to_csc / spmx_input_csc, with values), dx is
 * a gather over the CSC and dvals a pass over the CSR: no atomics,
 * deterministic.  Without one, both come from one pass over the CSR with
 * atomic adds into dx (Hola chunk table, built on demand). */
int spmx_spmv_backward(spmx_handle_t h, const float* d_x, const float* d_dy,
                       float* d_dx, float* d_dvals);
/* the same with a sparse dy (keys = rows); dvals is zero outside dy's rows */
int spmx_spmv_backward_sparse(spmx_handle_t h, const float* d_x,
                              const int* d_dy_key, const float* d_dy_val,
                              int dy_nnz, float* d_dx, float* d_dvals);

/* ======================= batched SpMSpV (FP32) ============================= */
/* No reference counterpart (the reference runs one vector per call).  nvec
 * (<= 1024) sparse vectors in one concatenated list: vector v owns entries
 * [xptr[v], xptr[v+1]) of (xkey, xval); xptr has nvec + 1 entries and
 * x_total = xptr[nvec] is also passed on the host (it sizes the scratch).  All
 * arrays are device pointers.  Together the vectors are a sparse n x nvec
 * matrix X and the call computes Y = alpha * A X, Y dense m x nvec row-major
 * (Y[i * nvec + v]), every entry written.  The batch is inverted by column,
 * then one warp per row of A accumulates the row of Y in shared memory.
 * Needs the CSR with values.  No host synchronisation once the scratch for
 * x_total exists: after one call outside stream capture with the largest
 * x_total, both entry points can be captured in a CUDA graph. */
int spmx_spmspv_batched(spmx_handle_t h, int nvec, int x_total, const int* d_xptr,
                        const int* d_xkey, const float* d_xval, float alpha, float* d_Y);
/* Adjoint of the batch for an upstream gradient dY (m x nvec, row-major):
 *   dxval[e] = alpha * sum_i A[i][xkey[e]] * dY[i * nvec + v(e)]   (needs the CSC)
 *   dvals[k] = alpha * sum over the batch's entries e in column col_k of
 *              xval[e] * dY[row_k * nvec + v(e)]                    (CSR order)
 * Both are written in full, deterministically (dxval not bitwise so with
 * SPMX_BATCH_FUSED_DXVAL, below).  Either output may be NULL. */
int spmx_spmspv_batched_backward(spmx_handle_t h, int nvec, int x_total, const int* d_xptr,
                                 const int* d_xkey, const float* d_xval, float alpha,
                                 const float* d_dY, float* d_dxval, float* d_dvals);
/* No reference counterpart.  Options of the batched entry points (flags,
 * default 0):
 *   SPMX_BATCH_REUSE_INVERSION: a backward call on the same batch (the same
 *     xptr / xkey / xval pointers, nvec and x_total) as the handle's last
 *     forward call reuses that call's inversion of the batch instead of
 *     sorting it again.  The caller promises that xptr, xkey and xval were not
 *     changed in between.
 *   SPMX_BATCH_FUSED_DXVAL: when a backward call asks for both dxval and
 *     dvals, dxval is accumulated during the dvals pass (which holds dY's rows
 *     in shared memory) with atomic adds, instead of a separate pass over the
 *     CSC that reads dY one element at a time.  dxval is then not bitwise
 *     reproducible (the order of its additions varies); dvals still is. */
#define SPMX_BATCH_REUSE_INVERSION 1
#define SPMX_BATCH_FUSED_DXVAL 2
int spmx_set_batch_options(spmx_handle_t h, int flags);

/* ======================= device counters ================================== */
/* device pointers to the handle's counters: [0] y_nnz of the last SpMSpV,
 * [1] bin_len of the last scan, [2] x_nnz after dense2sparse */
int spmx_get_device_counts(spmx_handle_t h, const int** d_counts);

/* ======================= host-side generators (no GPU) =================== */
/* Deterministic synthetic inputs (counter-based RNG; identical for any thread
 * count).  Output arrays are allocated with malloc by the generator and must
 * be released with spmx_host_free. */
void spmx_host_free(void* p);
/* symmetric R-MAT (no vertex permutation), self-loops and duplicates removed,
 * columns sorted per row */
int spmx_gen_rmat(int scale, int edge_factor, double a, double b, double c,
                  uint64_t seed, int* m_out, long long* nnz_out, int** rowptr,
                  int** col);
/* m x m, truncated Zipf(s) row lengths on [1, maxlen] scaled to mean `mean`
 * with stochastic rounding, total nnz fixed to mean*m, distinct uniform
 * columns per row, values U(-1,1) */
int spmx_gen_zipf_rows(int m, double s, int mean, int maxlen, uint64_t seed,
                       long long* nnz_out, int** rowptr, int** col, float** val);
/* Chung-Lu power law (degree exponent gamma, average expected degree avg),
 * symmetric pattern, self-loops and duplicates removed, values N(0,1) */
int spmx_gen_chung_lu(int n, double gamma, double avg, uint64_t seed,
                      long long* nnz_out, int** rowptr, int** col, float** val);
/* 2-D 5-point Laplacian on a g x g grid, diagonal 4, off-diagonals
 * -1 + N(0, sigma^2) */
int spmx_gen_laplacian(int g, double sigma, uint64_t seed, long long* nnz_out,
                       int** rowptr, int** col, float** val);
/* k distinct positions in [0,n) (sorted) into caller buffers, values U(-1,1)
 * (dist 0) or N(0,1) (dist 1) */
int spmx_gen_sparse_vector(int n, int k, int dist, uint64_t seed, int* key,
                           float* val);
/* host CSR -> CSC (stable; rows sorted within columns); val/cval may be NULL */
int spmx_host_csr2csc(int m, int n, const int* rowptr, const int* col,
                      const float* val, int* colptr, int* row, float* cval);

/* ======================= matrix files (host, no GPU) ====================== */
/* MatrixMarket coordinate file -> COO, 0-based, in file order: the reading
 * half of ReadMTX (INC/mtx.hpp:218-333).  "real" values are parsed as double
 * and rounded to float, "integer" values converted, "pattern" and "complex"
 * entries store 1 (as the reference does).  For a "symmetric" file each
 * off-diagonal entry is followed by its mirror; "skew-symmetric" and
 * "hermitian" files are not expanded (as in the reference).  Duplicates are
 * kept.  row/col/val are malloc'ed (release with spmx_host_free), NULL when
 * *nnz is 0.  info (may be NULL) receives [0] field: 0 real, 1 integer,
 * 2 pattern, 3 complex; [1] symmetry: 0 general, 1 symmetric, 2
 * skew-symmetric, 3 hermitian.  Malformed files (bad banner, "array" format,
 * missing size line, an index out of range, fewer or more entries than
 * declared) return SPMX_ERR_INVALID_VALUE naming the line. */
int spmx_mtx_read(const char* path, int* m, int* n, long long* nnz, int** row,
                  int** col, float** val, int* info);
/* COO (0-based, host) -> MatrixMarket coordinate file, "real" (or "pattern"
 * when val is NULL), banner symmetry "symmetric" when symmetric != 0 (the
 * caller passes one triangle) else "general".  Values are written as the
 * shortest text that reads back to the same float. */
int spmx_mtx_write(const char* path, int m, int n, long long nnz, const int* row,
                   const int* col, const float* val, int symmetric);
/* The reference's binary CSR cache (INC/mtx.hpp:706-808): 9-byte magic
 * "Hola\1CSR\1", 3 padding bytes, int32 rows, cols, nnz, then float
 * val[nnz], int32 col[nnz], int32 rowptr[rows+1].  Host arrays.
 * storeCSR (mtx.hpp:795-808) */
int spmx_csr_store(const char* path, int m, int n, int nnz, const int* rowptr,
                   const int* col, const float* val);
/* loadCSR_header (mtx.hpp:750-772) */
int spmx_csr_load_header(const char* path, int* m, int* n, int* nnz);
/* loadCSR (mtx.hpp:775-793); the sizes must match the header (the reference
 * does not check); val may be NULL to skip the values */
int spmx_csr_load(const char* path, int m, int n, int nnz, int* rowptr,
                  int* col, float* val);

#ifdef __cplusplus
}
#endif
#endif /* SPMX_H_ */
