// Allocation-free CSC SpMSpV: spmx_spmspv_csc_noalloc.
//
// Some callers cannot let a library call cudaMalloc: a host framework that
// owns the device heap through its own pooling allocator (memory taken
// behind its back is invisible to its accounting and can make it run out),
// or a latency-critical service loop, where cudaMalloc / cudaFree may
// synchronise the device and stall unrelated streams.  This entry point
// serves them: it runs the load-balanced (merge-path) CSC SpMSpV with atomic
// write-back, y = alpha * A * x, taking every input and output from the
// caller and all of its scratch from one fixed array in device global memory,
// declared below.  It needs no handle (creating one allocates).
//
// The scratch array is a file-scope __device__ variable: each GPU that loads
// this library holds it (kNoAllocScratchBytes, about 8.6 MB) until the process
// exits.  Its size bounds the problem: x_nnz <= kNoAllocMaxX and
// nnz + x_nnz <= kNoAllocMaxItems; larger calls are rejected with
// SPMX_ERR_INVALID_VALUE before anything is launched.
//
// Host code cannot use the array's name as a device address (in host code it
// names a host-side stand-in), so the first call on each device looks up the
// real address with cudaGetSymbolAddress while that device is current, sizes
// the launch grid from the device's SM count and caches both; make that first
// call before any stream capture.  Every call on a device shares the one array
// and leaves its contents behind: what must start at zero (the look-back
// status words, the tile ticket and epoch, the error word) is cleared by a
// small memset at the start of every call.  Calls whose work overlaps on the
// GPU (different streams, or host threads racing) would corrupt each other's
// scratch: serialise them, e.g. on one stream.
//
// Bad input (an x key outside [0, n), a row index outside [0, m)) and a
// bounded wait that gave up are recorded in an error word in the same array,
// never as a fault.  spmx_spmspv_csc_noalloc_check reads that word after a
// call (it synchronises the stream and copies 4 bytes; it allocates nothing).
#include <algorithm>
#include <mutex>
#include <string>

#include "common.cuh"
#include "engine.h"
#include "kernels.h"

namespace {

constexpr int kNoAllocMaxX = 1 << 20;                 // x nonzeros per call
constexpr long long kNoAllocMaxItems = 1LL << 27;      // nnz + x_nnz per call
constexpr int kNoAllocBlockItems = spmx::kCscLbNT * spmx::kCscLbVT;  // 2048
constexpr int kNoAllocMaxBlocks = (int)(kNoAllocMaxItems / kNoAllocBlockItems) + 2;
constexpr int kNoAllocMaxTiles =
    kNoAllocMaxX / (spmx::kCscScanNT * spmx::kCscScanVT) + 4;

constexpr size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
// regions of the scratch array, in order
constexpr size_t kOffBytes = align256(4 * (size_t)(kNoAllocMaxX + 1));
constexpr size_t kColstartBytes = align256(4 * (size_t)kNoAllocMaxX);
constexpr size_t kBstartBytes = align256(4 * (size_t)kNoAllocMaxBlocks);
constexpr size_t kStatusBytes = align256(8 * (size_t)kNoAllocMaxTiles);
constexpr size_t kWordsBytes = 256;  // ticket words (4) + counts (16) + err
constexpr size_t kStatusOffset = kOffBytes + kColstartBytes + 2 * kBstartBytes;
constexpr size_t kWordsOffset = kStatusOffset + kStatusBytes;
constexpr size_t kErrOffset = kWordsOffset + 16 + 4 * (size_t)spmx::kCntTotal;
constexpr size_t kNoAllocScratchBytes = kWordsOffset + kWordsBytes;
static_assert(kErrOffset + 4 <= kNoAllocScratchBytes, "error word inside the scratch array");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char* g_base[kMaxDevices] = {nullptr};
int g_grid[kMaxDevices] = {0};

}  // namespace

namespace spmx {
int csc_lb_blocks_per_sm();
}

namespace {

// device address of the scratch array and the load-balanced kernel's grid on
// the current device (set-up on the first call per device)
int scratch_base(int dev, unsigned char** base, int* grid) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_base[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return spmx::set_error(SPMX_ERR_CUDA, std::string("cudaGetSymbolAddress(noalloc scratch): ") +
                                                cudaGetErrorString(e));
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
      cudaGetLastError();
      sms = 1;
    }
    g_grid[dev] = std::max(1, sms) * std::max(1, spmx::csc_lb_blocks_per_sm());
    g_base[dev] = static_cast<unsigned char*>(p);
  }
  *base = g_base[dev];
  *grid = g_grid[dev];
  return SPMX_SUCCESS;
}

}  // namespace

using namespace spmx;

extern "C" int spmx_spmspv_csc_noalloc(int m, int n, int nnz, const int* d_csc_row,
                                       const int* d_csc_col, const float* d_csc_val,
                                       int x_nnz, const int* d_x_key, const float* d_x_val,
                                       float alpha, float* d_y, void* stream) {
  if (m < 0 || n < 0 || nnz < 0 || x_nnz < 0)
    return set_error(SPMX_ERR_INVALID_VALUE, "noalloc SpMSpV: negative size");
  if (x_nnz > n) return set_error(SPMX_ERR_INVALID_VALUE, "noalloc SpMSpV: x_nnz exceeds n");
  if (x_nnz > kNoAllocMaxX)
    return set_error(SPMX_ERR_INVALID_VALUE,
                     "noalloc SpMSpV: x_nnz " + std::to_string(x_nnz) + " exceeds the fixed scratch "
                     "limit of " + std::to_string(kNoAllocMaxX));
  if ((long long)nnz + x_nnz > kNoAllocMaxItems)
    return set_error(SPMX_ERR_INVALID_VALUE,
                     "noalloc SpMSpV: nnz + x_nnz exceeds the fixed scratch limit of " +
                         std::to_string(kNoAllocMaxItems));
  if ((m > 0 && !d_y) || !d_csc_col || (nnz > 0 && (!d_csc_row || !d_csc_val)) ||
      (x_nnz > 0 && (!d_x_key || !d_x_val)))
    return set_error(SPMX_ERR_INVALID_VALUE, "noalloc SpMSpV: NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  if (m == 0) return SPMX_SUCCESS;
  if (cudaMemsetAsync(d_y, 0, 4 * (size_t)m, st) != cudaSuccess)
    return set_error(SPMX_ERR_CUDA, "noalloc SpMSpV: y memset failed");
  if (x_nnz == 0) return SPMX_SUCCESS;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return set_error(SPMX_ERR_NO_DEVICE, "noalloc SpMSpV: no usable current device");
  }
  unsigned char* base = nullptr;
  int grid = 1;
  const int rc = scratch_base(dev, &base, &grid);
  if (rc) return rc;

  unsigned char* p = base;
  CscScratch s{};
  s.off = reinterpret_cast<int*>(p);
  p += kOffBytes;
  s.colstart = reinterpret_cast<int*>(p);
  p += kColstartBytes;
  s.bstart_tl = reinterpret_cast<int*>(p);
  p += kBstartBytes;
  s.bstart_mg = reinterpret_cast<int*>(p);
  p += kBstartBytes;
  s.tl_cap = kNoAllocMaxBlocks;
  s.mg_cap = kNoAllocMaxBlocks;
  ScanScratch ls{};
  ls.status = reinterpret_cast<unsigned long long*>(base + kStatusOffset);
  ls.status_len = kNoAllocMaxTiles;
  ls.ticket = reinterpret_cast<unsigned*>(base + kWordsOffset);
  int* counts = reinterpret_cast<int*>(base + kWordsOffset + 16);
  int* err = reinterpret_cast<int*>(base + kErrOffset);
  // status words, ticket / epoch / publish words, counts and the error word
  // start at zero in every call (one contiguous region of a few KB)
  if (cudaMemsetAsync(base + kStatusOffset, 0, kStatusBytes + kWordsBytes, st) != cudaSuccess)
    return set_error(SPMX_ERR_CUDA, "noalloc SpMSpV: scratch reset failed");

  const CscArgs a{m, n, d_csc_col, d_csc_row, d_csc_val, x_nnz, d_x_key, d_x_val,
                  (double)alpha, err, counts};
  if (launch_csc_scan(a, s, ls, kNoAllocBlockItems, st))
    return set_error(SPMX_ERR_INVALID_VALUE, "noalloc SpMSpV: scan capacity");
  launch_csc_lb(a, s, 1, d_y, nullptr, nullptr, grid, st);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_error(SPMX_ERR_CUDA, std::string("noalloc SpMSpV launch: ") + cudaGetErrorString(e));
  return SPMX_SUCCESS;
}

extern "C" int spmx_spmspv_csc_noalloc_check(void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  int e = 0;
  if (cudaMemcpyFromSymbolAsync(&e, g_noalloc_scratch, sizeof(int), kErrOffset,
                                cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    const cudaError_t ce = cudaGetLastError();
    return set_error(SPMX_ERR_CUDA, std::string("noalloc SpMSpV check: ") + cudaGetErrorString(ce));
  }
  if (e & kDevErrTimeout) return set_error(SPMX_ERR_TIMEOUT, "noalloc SpMSpV: a bounded device wait timed out");
  if (e & kDevErrOob) return set_error(SPMX_ERR_OOB, "noalloc SpMSpV: an index was out of range (bad input)");
  if (e & kDevErrCapacity) return set_error(SPMX_ERR_OOB, "noalloc SpMSpV: an internal capacity was exceeded");
  return SPMX_SUCCESS;
}
