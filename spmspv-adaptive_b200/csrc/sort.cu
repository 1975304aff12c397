// Stable LSD radix sort of 32-bit keys with up to two 32-bit payloads, a
// generic single-pass exclusive scan, and reduce_by_key over sorted keys.
//
// They replace the Thrust / CUB calls of the reference's sort write-back
// (thrust::sort_by_key + thrust::reduce_by_key, DEV/csc_sort_spmspv.cuh:341,
// :412) and cuSPARSE csr2csc inside ToCSC (H:409): a transpose is a stable
// sort of the row-major COO by column.
//
// One pass = 8 key bits: (1) per-tile digit histograms, stored digit-major,
// (2) exclusive scan of the histograms, (3) stable scatter.  Inside a tile each
// warp owns 512 consecutive items and ranks them round by round with
// __match_any_sync; warp-private digit counters are then offset across warps,
// so the order of equal digits follows the input order (stability).
#include "kernels.h"
#include "sort.h"
#include "common.cuh"

namespace spmx {

constexpr int kRadixNT = 256;
constexpr int kRadixIPT = 16;                       // items per thread
constexpr int kRadixTile = kRadixNT * kRadixIPT;    // 4096
constexpr int kRadixDigits = 256;

__global__ void __launch_bounds__(kRadixNT)
radix_hist_kernel(const unsigned* __restrict__ keys, int n, int shift,
                  int ntiles, int* __restrict__ hist) {
  __shared__ int s_h[kRadixDigits];
  const int tile = blockIdx.x;
  s_h[threadIdx.x] = 0;
  __syncthreads();
  const int base = tile * kRadixTile;
#pragma unroll 4
  for (int j = 0; j < kRadixIPT; ++j) {
    const int i = base + j * kRadixNT + threadIdx.x;
    if (i < n) atomicAdd(&s_h[(__ldg(keys + i) >> shift) & 0xff], 1);
  }
  __syncthreads();
  hist[threadIdx.x * ntiles + tile] = s_h[threadIdx.x];
}

template <int NPAY>
__global__ void __launch_bounds__(kRadixNT)
radix_scatter_kernel(const unsigned* __restrict__ keys_in,
                     const unsigned* __restrict__ p1_in,
                     const unsigned* __restrict__ p2_in, int n, int shift,
                     int ntiles, const int* __restrict__ goff,
                     unsigned* __restrict__ keys_out, unsigned* __restrict__ p1_out,
                     unsigned* __restrict__ p2_out) {
  constexpr int NW = kRadixNT / 32;
  constexpr int WITEMS = kRadixTile / NW;  // 512 items per warp
  constexpr int ROUNDS = WITEMS / 32;      // 16
  __shared__ int s_wc[NW][kRadixDigits];
  const int tile = blockIdx.x;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int d = threadIdx.x; d < NW * kRadixDigits; d += kRadixNT)
    (&s_wc[0][0])[d] = 0;
  __syncthreads();
  const int wbase = tile * kRadixTile + w * WITEMS;
  unsigned k[ROUNDS];
  int rank[ROUNDS];
#pragma unroll
  for (int j = 0; j < ROUNDS; ++j) {
    const int i = wbase + j * 32 + lane;
    const bool valid = i < n;
    k[j] = valid ? __ldg(keys_in + i) : 0xffffffffu;
    const int d = valid ? (int)((k[j] >> shift) & 0xff) : -1 - lane;  // invalid items never match
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    int base = 0;
    if (valid) base = s_wc[w][d];
    __syncwarp();
    if (valid && (peers & lanemask_lt()) == 0) s_wc[w][d] += __popc(peers);
    __syncwarp();
    rank[j] = base + __popc(peers & lanemask_lt());
  }
  __syncthreads();
  {
    const int d = threadIdx.x;  // kRadixNT == kRadixDigits
    int run = 0;
#pragma unroll
    for (int ww = 0; ww < NW; ++ww) {
      const int t = s_wc[ww][d];
      s_wc[ww][d] = run;
      run += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < ROUNDS; ++j) {
    const int i = wbase + j * 32 + lane;
    if (i < n) {
      const int d = (int)((k[j] >> shift) & 0xff);
      const int dst = goff[d * ntiles + tile] + s_wc[w][d] + rank[j];
      keys_out[dst] = k[j];
      if (NPAY >= 1) p1_out[dst] = __ldg(p1_in + i);
      if (NPAY >= 2) p2_out[dst] = __ldg(p2_in + i);
    }
  }
}

// generic exclusive scan of ints (single pass, decoupled look-back)
template <int NT, int VT>
__global__ void __launch_bounds__(NT)
scan_exclusive_kernel(const int* __restrict__ in, int* __restrict__ out, int n,
                      LookbackState st, int ntiles, int* total_out, int* err) {
  __shared__ int s_v[NT * VT];
  __shared__ unsigned s_wtmp[NT / 32 + 1];
  __shared__ int s_tile;
  __shared__ unsigned s_prefix;
  const int tile = lb_acquire_tile(st, ntiles, &s_tile);
  const int base = tile * NT * VT;
  const int tid = threadIdx.x;
#pragma unroll
  for (int j = 0; j < VT; ++j) {
    const int i = base + j * NT + tid;
    s_v[j * NT + tid] = (i < n) ? __ldg(in + i) : 0;
  }
  __syncthreads();
  unsigned loc[VT];
  unsigned sum = 0;
#pragma unroll
  for (int j = 0; j < VT; ++j) { loc[j] = (unsigned)s_v[tid * VT + j]; sum += loc[j]; }
  unsigned total;
  const unsigned ex = block_exclusive_sum<NT>(sum, s_wtmp, &total);
  if (tid < 32) {
    const unsigned p = lb_warp_lookback(st, tile, ntiles, total, err);
    if (tid == 0) s_prefix = p;
  }
  __syncthreads();
  unsigned run = s_prefix + ex;
#pragma unroll
  for (int j = 0; j < VT; ++j) { s_v[tid * VT + j] = (int)run; run += loc[j]; }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < VT; ++j) {
    const int i = base + j * NT + tid;
    if (i < n) out[i] = s_v[j * NT + tid];
  }
  if (tile == ntiles - 1 && tid == 0 && total_out) *total_out = (int)(s_prefix + total);
}

int launch_scan_exclusive(const int* in, int* out, int n, int* total_out,
                          ScanScratch& ls, int* err, cudaStream_t st) {
  constexpr int NT = 256, VT = 8;
  if (n <= 0) return 0;
  const int ntiles = (n + NT * VT - 1) / (NT * VT);
  if (ntiles > ls.status_len) return -1;
  LookbackState lbs{ls.status, ls.ticket};
  note_launch();
  scan_exclusive_kernel<NT, VT><<<ntiles, NT, 0, st>>>(in, out, n, lbs, ntiles,
                                                      total_out, err);
  return 0;
}

size_t radix_hist_ints(int n) {
  const int ntiles = (n + kRadixTile - 1) / kRadixTile;
  return (size_t)ntiles * kRadixDigits;
}

int radix_sort_pairs(RadixBuffers& b, int n, int key_bits, ScanScratch& ls,
                     int* err, cudaStream_t st) {
  b.result_in_alt = false;
  if (n <= 1) return 0;
  const int ntiles = (n + kRadixTile - 1) / kRadixTile;
  const int hn = ntiles * kRadixDigits;
  int passes = (key_bits + 7) / 8;
  if (passes < 1) passes = 1;
  unsigned *kin = b.keys, *kout = b.keys_alt;
  unsigned *p1in = b.p1, *p1out = b.p1_alt;
  unsigned *p2in = b.p2, *p2out = b.p2_alt;
  for (int p = 0; p < passes; ++p) {
    const int shift = p * 8;
    note_launch(2);  // histogram + scatter (the scan counts itself)
    radix_hist_kernel<<<ntiles, kRadixNT, 0, st>>>(kin, n, shift, ntiles, b.hist);
    if (launch_scan_exclusive(b.hist, b.hist_off, hn, nullptr, ls, err, st)) return -1;
    if (b.p2)
      radix_scatter_kernel<2><<<ntiles, kRadixNT, 0, st>>>(kin, p1in, p2in, n, shift, ntiles,
                                                          b.hist_off, kout, p1out, p2out);
    else if (b.p1)
      radix_scatter_kernel<1><<<ntiles, kRadixNT, 0, st>>>(kin, p1in, p2in, n, shift, ntiles,
                                                          b.hist_off, kout, p1out, p2out);
    else
      radix_scatter_kernel<0><<<ntiles, kRadixNT, 0, st>>>(kin, p1in, p2in, n, shift, ntiles,
                                                          b.hist_off, kout, p1out, p2out);
    unsigned* t;
    t = kin; kin = kout; kout = t;
    t = p1in; p1in = p1out; p1out = t;
    t = p2in; p2in = p2out; p2out = t;
    b.result_in_alt = !b.result_in_alt;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// reduce_by_key over sorted keys: unique keys in order and the sum of the
// values of each run.  Pass 1 finds run heads (single-pass scan of head flags)
// and writes the unique keys, zeroes the sums and records each item's output
// slot; pass 2 adds every warp-run of equal slots with one atomic.
// ---------------------------------------------------------------------------
template <int NT, int VT>
__global__ void __launch_bounds__(NT)
rbk_heads_kernel(const unsigned* __restrict__ keys, int n, int* __restrict__ slot,
                 int* __restrict__ out_key, float* __restrict__ out_val,
                 int* d_count, LookbackState st, int ntiles, int* err) {
  constexpr int NW = NT / 32;
  __shared__ unsigned s_cnt[VT * NW];
  __shared__ unsigned s_wtmp[NT / 32 + 1];
  __shared__ int s_tile;
  __shared__ unsigned s_prefix, s_total;
  const int tile = lb_acquire_tile(st, ntiles, &s_tile);
  const int base = tile * NT * VT;
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  bool head[VT];
  unsigned mask[VT];
  unsigned kk[VT];
#pragma unroll
  for (int j = 0; j < VT; ++j) {
    const int i = base + j * NT + tid;
    head[j] = false;
    kk[j] = 0;
    if (i < n) {
      kk[j] = __ldg(keys + i);
      head[j] = (i == 0) || (__ldg(keys + i - 1) != kk[j]);
    }
    mask[j] = __ballot_sync(0xffffffffu, head[j]);
    if (lane == 0) s_cnt[j * NW + w] = __popc(mask[j]);
  }
  __syncthreads();
  unsigned c = (tid < VT * NW) ? s_cnt[tid] : 0u;
  unsigned total;
  const unsigned ex = block_exclusive_sum<NT>(c, s_wtmp, &total);
  if (tid < VT * NW) s_cnt[tid] = ex;
  if (tid < 32) {
    const unsigned p = lb_warp_lookback(st, tile, ntiles, total, err);
    if (tid == 0) { s_prefix = p; s_total = total; }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < VT; ++j) {
    const int i = base + j * NT + tid;
    if (i < n) {
      // slot = number of heads at or before i, minus one
      const int pos = (int)(s_prefix + s_cnt[j * NW + w] +
                            __popc(mask[j] & lanemask_lt())) + (head[j] ? 0 : -1);
      slot[i] = pos;
      if (head[j]) { out_key[pos] = (int)kk[j]; out_val[pos] = 0.0f; }
    }
  }
  if (tile == ntiles - 1 && tid == 0) *d_count = (int)(s_prefix + s_total);
}

__global__ void rbk_add_kernel(const int* __restrict__ slot,
                               const float* __restrict__ vals, int n,
                               float* __restrict__ out_val) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool valid = i < n;
  const int s = valid ? __ldg(slot + i) : -1;
  float v = valid ? __ldg(vals + i) : 0.0f;
  // runs of equal slots are contiguous lanes (slots are non-decreasing);
  // a segmented suffix sum leaves each run's total in its first lane
  const unsigned same = __match_any_sync(0xffffffffu, s);
  const int first = __ffs(same) - 1;
  const int run_end = 31 - __clz(same);
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const float t = __shfl_down_sync(0xffffffffu, v, o);
    if (lane + o <= run_end) v += t;
  }
  if (valid && lane == first) atomicAdd(out_val + s, v);
}

int reduce_by_key_sorted(const unsigned* keys, const float* vals, int n,
                         int* slot_scratch, int* out_key, float* out_val,
                         int* d_count, ScanScratch& ls, int* err,
                         cudaStream_t st) {
  constexpr int NT = 256, VT = 8;
  if (n <= 0) { cudaMemsetAsync(d_count, 0, sizeof(int), st); return 0; }
  const int ntiles = (n + NT * VT - 1) / (NT * VT);
  if (ntiles > ls.status_len) return -1;
  LookbackState lbs{ls.status, ls.ticket};
  note_launch(2);
  rbk_heads_kernel<NT, VT><<<ntiles, NT, 0, st>>>(keys, n, slot_scratch, out_key, out_val,
                                                 d_count, lbs, ntiles, err);
  rbk_add_kernel<<<(n + 255) / 256, 256, 0, st>>>(slot_scratch, vals, n, out_val);
  return 0;
}

}  // namespace spmx
