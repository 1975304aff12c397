// The handle behind the C ABI (spmx.h).  Host-side state of one matrix: the
// borrowed CSR, the CSC (owned after spmx_to_csc), the current x in its
// sparse / dense / bitarray forms, the scratch of every kernel family, cached
// features and tuned launch parameters.  Mirrors the members of
// SpmspvHandle (H:246-344).
#pragma once
#include <cuda_runtime.h>
#include <string>
#include "spmx.h"
#include "kernels.h"
#include "sort.h"

struct spmx_handle_s {
  int m = 0, n = 0, nnz = 0;
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;

  // CSR (borrowed via input_csr, or owned after input_coo)
  const int* rowptr = nullptr;
  const int* col = nullptr;
  const float* val = nullptr;
  bool has_csr = false;
  int* own_csr_rowptr = nullptr;
  int* own_csr_col = nullptr;
  float* own_csr_val = nullptr;
  // CSC (borrowed via input_csc or owned via to_csc)
  const int* csc_colptr = nullptr;
  const int* csc_row = nullptr;
  const float* csc_val = nullptr;
  bool has_csc = false;
  int* own_colptr = nullptr;
  int* own_row = nullptr;
  float* own_cval = nullptr;

  // x
  float* x_dense = nullptr;
  int* x_key = nullptr;
  float* x_val = nullptr;
  int x_nnz = 0;
  int* bitvec = nullptr;
  int num_ints = 0;
  int vec_type = -1;
  float* own_xdense = nullptr;
  int* own_bits = nullptr;

  int spmv_type = SPMX_SPMV_HOLA;
  int sigma = -1;

  // device counters, error word, feature accumulators
  int* d_counts = nullptr;         // spmx::kCntTotal ints
  int* d_err = nullptr;            // sticky error bits
  double* d_facc = nullptr;        // 4 doubles
  int* d_iacc = nullptr;           // 4 ints
  unsigned long long* d_u64 = nullptr;  // 4 words
  int* h_pinned = nullptr;         // 16 ints of pinned host memory

  spmx::ScanScratch ls{};          // look-back status + ticket

  // CSC SpMSpV scratch
  spmx::CscScratch cs{};
  bool cs_ready = false;
  // sort write-back scratch (pairs + radix)
  unsigned* sk = nullptr;
  unsigned* sk_alt = nullptr;
  unsigned* sv = nullptr;
  unsigned* sv_alt = nullptr;
  int* shist = nullptr;
  int* shist_off = nullptr;
  int* sslot = nullptr;
  int* sy_key = nullptr;      // internal sparse y (adaptive path)
  float* sy_val = nullptr;
  bool sort_ready = false;
  int* bk_gcount = nullptr;   // bucket histogram / offsets / cursors
  int* bk_boff = nullptr;
  int* bk_cursor = nullptr;
  int buckets = 0;            // 0 = default (256)

  // CSR5 tile tables (csr5.cu) and tiled-SpMV tables (tiled.cu)
  void* csr5 = nullptr;
  void* tiled = nullptr;
  // round-SpMV tables (round.cu)
  void* round = nullptr;
  void* hybrid = nullptr;  // CSR/CSC split tables (hybrid.cu)

  // Hola tables
  spmx::HolaTables hola{};
  bool hola_ready = false;

  // tuned parameters
  int naive_row_group = 0;    // 0 = derive from mean row length
  int naive_col_group = 0;    // 0 = derive from mean column length
  int hola_vt = 8;
  int lb_variant = SPMX_CSC_LB_MERGE;
  int lb_grid = 0;

  // cached features
  bool mat_feat_ready = false;
  double mat_feat[10] = {0};
  bool std_row_ready = false;
  long long col_max = -1;     // longest CSC column (-1 = not computed)
  float std_row = 0.f;
  long long bin_len = -1;
  long long vec_max = 0, vec_min = 0;
  double gm[3] = {-1, -1, -1};

  // BFS buffers (level-stepped and persistent)
  int bfs_mode = 0;                        // 0 persistent, 1 level-stepped
  unsigned* bfs_fb1 = nullptr;
  void* bfs_ctrl = nullptr;                // BfsCtrl
  // batched (multi-source) BFS buffers
  unsigned long long* ms_visit = nullptr;
  unsigned long long* ms_front0 = nullptr;
  unsigned long long* ms_front1 = nullptr;
  unsigned long long* ms_next = nullptr;
  int* ms_q0 = nullptr;
  int* ms_q1 = nullptr;
  int* ms_srcs = nullptr;
  int* ms_tmp = nullptr;                   // vertex-major levels for layout 1
  size_t ms_tmp_len = 0;
  void* ms_ctrl = nullptr;
  int ms_n = 0;
  // batched SpMSpV: the batch inverted by column (radix sort buffers for
  // keys / entries / vectors and their alternates, column pointers)
  void* batch_buf[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  int* batch_hist = nullptr;
  int* batch_hoff = nullptr;
  int* batch_invptr = nullptr;
  int batch_cap = 0;
  int batch_invptr_n = -1;
  int batch_opts = 0;  // SPMX_BATCH_* flags (spmx_set_batch_options)
  // the batch the current inversion belongs to (valid after a forward call)
  const void* inv_xptr = nullptr;
  const void* inv_xkey = nullptr;
  int inv_nvec = -1, inv_total = -1;
  const void* inv_xval = nullptr;
  const unsigned* inv_ent = nullptr;
  const unsigned* inv_vec = nullptr;
  // per inverted pair: int2 (vector, x value bits), then, at a 256-byte
  // boundary, int4 (vector, x value bits, entry, 0)
  void* batch_rec = nullptr;
  // row chunks of the batched row walks (rows cut where rowptr[i] + 32 i
  // crosses a multiple of 2,048; warps take chunks from a device counter)
  int* batch_chunk = nullptr;
  int batch_nch = 0;
  bool batch_chunk_ready = false;
  int* batch_ctr = nullptr;  // [0] the forward walk's chunk counter, [1] the dvals walk's
  // hub chunks of the multi-source pull (built once per matrix)
  int4* ms_hchunk = nullptr;
  int* ms_hcnt = nullptr;
  unsigned long long* ms_hacc = nullptr;
  int* ms_hleft = nullptr;
  int* ms_hcounters = nullptr;
  long long ms_nhchunks = 0;
  int ms_nhubs = 0;
  const int* ms_hub_rowptr = nullptr;
  int ms_hub_nnz = -1;
  double bfs_alpha = 14.0, bfs_beta = 24.0, msbfs_alpha = 12.0;
  unsigned* bfs_visited = nullptr;
  unsigned* bfs_front = nullptr;
  unsigned* bfs_fb2 = nullptr;
  int* bfs_q[2] = {nullptr, nullptr};
  int* bfs_cnt = nullptr;                  // [0..1] queue counts
  unsigned long long* bfs_edges = nullptr; // [0..1]
  int bfs_n = 0;
};

namespace spmx {
int set_error(int code, const std::string& msg);
int dalloc(void** p, size_t bytes, const char* what);
void dfree(void* p);
// A kernel's dynamic shared-memory limit is a property of the function on a
// device, shared by every handle: set it to `bytes` unless it already is
// (cached per function and device), right before a launch that needs it.
cudaError_t kernel_smem_limit(const void* kernel, size_t bytes);
}  // namespace spmx

// Status plumbing shared by the entry points: return the first failure.
#define SPMX_CUDA(call)                                                        \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      return set_error(SPMX_ERR_CUDA,                                          \
                       std::string(#call) + ": " + cudaGetErrorString(e_));    \
    }                                                                          \
  } while (0)

#define SPMX_TRY(expr)                                                         \
  do {                                                                         \
    int r_ = (expr);                                                           \
    if (r_ != SPMX_SUCCESS) return r_;                                         \
  } while (0)

#define SPMX_CHECK_HANDLE(h)                                                   \
  do {                                                                         \
    if (!(h)) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");         \
  } while (0)

// status of the last kernel launch on this thread
inline int launch_ok(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return spmx::set_error(SPMX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return SPMX_SUCCESS;
}
