// Vector-format conversions (H:1121-1393, H:1883-1998; DEV/bitvector.h).
//
// scatter: sparse -> dense and/or bitarray in one kernel (the reference uses a
//   scatter plus a separate set_sparse_x_bitvector launch, H:1271-1308).
// dense2bits: one warp per 32-bit word, ballot of (x != 0); no atomics, no
//   memset (the reference memsets and atomically ORs, and tests `!val`,
//   setting the bits of zeros, H:1362).
// compact: dense -> (key, val) of the entries != 0, in index order, in two
//   chained grids: per-range nonzero counts, then per-range prefixes from
//   those counts and the writes (per-warp ballot/popc ranks, a block scan of
//   warp counts); the reference runs a flag kernel, a CUB scan with a
//   temporary allocation and a compaction kernel, H:1883-1928.
#include "kernels.h"
#include "common.cuh"

namespace spmx {

__global__ void scatter_kernel(int nvals, int len, const int* __restrict__ key,
                               const float* __restrict__ val,
                               float* __restrict__ dense, int* bits, int* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nvals) return;
  const int k = __ldg(key + i);
  if ((unsigned)k >= (unsigned)len) { flag_error(err, kDevErrOob); return; }
  if (dense) dense[k] = val ? __ldg(val + i) : 1.0f;
  if (bits) atomicOr(bits + (k >> 5), (int)(1u << (k & 31)));
}

// scatter after a zero fill of `dense` launched just before (programmatic
// dependent launch): keys and values are read before the wait
__global__ void scatter_after_fill_kernel(int nvals, int len, const int* __restrict__ key,
                                          const float* __restrict__ val, float* __restrict__ dense,
                                          int* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int k = 0;
  float v = 0.f;
  if (i < nvals) {
    k = __ldg(key + i);
    v = val ? __ldg(val + i) : 1.0f;
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;");
  if (i >= nvals) return;
  if ((unsigned)k >= (unsigned)len) {
    flag_error(err, kDevErrOob);
    return;
  }
  dense[k] = v;
}

__global__ void dense2bits_kernel(int len, const float* __restrict__ dense,
                                  int* __restrict__ bits) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long word = gid >> 5;
  const int lane = threadIdx.x & 31;
  const long long idx = word * 32 + lane;
  const bool nz = idx < len && __ldg(dense + idx) != 0.0f;
  const unsigned b = __ballot_sync(0xffffffffu, nz);
  if (lane == 0 && word * 32 < len) bits[word] = (int)b;
}

// Compaction in two grids, chained by programmatic dependent launch.  Pass 1
// counts the nonzeros of each CTA's range of `per` elements; pass 2 adds the
// counts of the ranges before its own (at most kCompactMaxRanges of them, a
// few loads per thread), then writes its range's nonzeros sub-tile by sub-tile
// of NT * VT elements.  A single pass with a decoupled look-back took 11-14 us
// for 1M elements whatever the look-back window: its CTAs sat at a barrier
// while warp 0 took a ticket, published and looked back.  Here nothing waits
// on another CTA.
constexpr int kCompactMaxRanges = 1024;

template <int NT, int VT>
__global__ void __launch_bounds__(NT)
compact_count_kernel(long long len, long long per, const float* __restrict__ dense,
                     unsigned* __restrict__ counts) {
  constexpr int NW = NT / 32;
  __shared__ unsigned s_w[NW];
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;");
  const long long r0 = (long long)blockIdx.x * per, r1 = min(len, r0 + per);
  unsigned c = 0;
  for (long long b = r0; b < r1; b += (long long)NT * VT) {
#pragma unroll
    for (int j = 0; j < VT; ++j) {
      const long long i = b + j * NT + threadIdx.x;
      c += (i < r1 && __ldg(dense + i) != 0.0f) ? 1u : 0u;
    }
  }
  c = warp_sum(c);
  if (lane_id() == 0) s_w[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x < 32) {
    unsigned t = threadIdx.x < NW ? s_w[threadIdx.x] : 0u;
    t = warp_sum(t);
    if (threadIdx.x == 0) counts[blockIdx.x] = t;
  }
}

template <int NT, int VT>
__global__ void __launch_bounds__(NT)
compact_write_kernel(long long len, long long per, const float* __restrict__ dense,
                     const unsigned* __restrict__ counts, int* __restrict__ key,
                     float* __restrict__ val, int* d_count) {
  constexpr int NW = NT / 32;
  __shared__ unsigned s_cnt[VT * NW];
  __shared__ unsigned s_wtmp[NW + 1];
  __shared__ unsigned s_red[NW];
  __shared__ int s_key[NT * VT];
  __shared__ float s_val[NT * VT];
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const long long r0 = (long long)blockIdx.x * per, r1 = min(len, r0 + per);
  // the first sub-tile's values: dense was written before pass 1 waited, so
  // it is complete once this grid starts
  float v[VT];
#pragma unroll
  for (int j = 0; j < VT; ++j) {
    const long long i = r0 + j * NT + tid;
    v[j] = (i < r1) ? __ldg(dense + i) : 0.0f;
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;");
  // nonzeros before this range
  unsigned pre = 0;
  for (int t = tid; t < (int)blockIdx.x; t += NT) pre += __ldcg(counts + t);
  pre = warp_sum(pre);
  if (lane == 0) s_red[w] = pre;
  __syncthreads();
  unsigned run = 0;
#pragma unroll
  for (int q = 0; q < NW; ++q) run += s_red[q];
  for (long long b = r0; b < r1; b += (long long)NT * VT) {
    if (b != r0) {
#pragma unroll
      for (int j = 0; j < VT; ++j) {
        const long long i = b + j * NT + tid;
        v[j] = (i < r1) ? __ldg(dense + i) : 0.0f;
      }
    }
    unsigned mask[VT];
#pragma unroll
    for (int j = 0; j < VT; ++j) {
      mask[j] = __ballot_sync(0xffffffffu, v[j] != 0.0f);
      if (lane == 0) s_cnt[j * NW + w] = __popc(mask[j]);
    }
    __syncthreads();
    // exclusive scan of the VT * NW counts, in (j, w) order == index order
    const unsigned c = (tid < VT * NW) ? s_cnt[tid] : 0u;
    unsigned total;
    const unsigned ex = block_exclusive_sum<NT>(c, s_wtmp, &total);
    if (tid < VT * NW) s_cnt[tid] = ex;
    __syncthreads();
    // staged in index order, then written by consecutive threads: a warp's
    // stores are contiguous (full PCIe write packets for pinned host memory)
#pragma unroll
    for (int j = 0; j < VT; ++j) {
      if (v[j] != 0.0f) {
        const unsigned pos = s_cnt[j * NW + w] + __popc(mask[j] & lanemask_lt());
        s_key[pos] = (int)(b + j * NT + tid);
        s_val[pos] = v[j];
      }
    }
    __syncthreads();
    for (unsigned t = tid; t < total; t += NT) {
      key[run + t] = s_key[t];
      val[run + t] = s_val[t];
    }
    run += total;
    __syncthreads();
  }
  if (blockIdx.x == gridDim.x - 1 && tid == 0) *d_count = (int)run;
}

int launch_scatter(int nvals, int len, const int* key, const float* val,
                   float* dense, int* bits, int* err, cudaStream_t st) {
  if (nvals <= 0) return 0;
  note_launch();
  scatter_kernel<<<(nvals + 255) / 256, 256, 0, st>>>(nvals, len, key, val, dense,
                                                     bits, err);
  return 0;
}

int launch_dense_from_sparse(int nvals, int len, const int* key, const float* val, float* dense,
                             int* err, int num_sms, cudaStream_t st) {
  launch_zero_fill(dense, len, num_sms, st);
  if (nvals <= 0) return 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)((nvals + 255) / 256));
  cfg.blockDim = dim3(256);
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  note_launch();
  return cudaLaunchKernelEx(&cfg, scatter_after_fill_kernel, nvals, len, key, val, dense, err) == cudaSuccess
             ? 0
             : -2;
}

int launch_dense2bits(int len, const float* dense, int* bits, cudaStream_t st) {
  if (len <= 0) return 0;
  const long long words = (len + 31) / 32;
  const long long threads = words * 32;
  note_launch();
  dense2bits_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(len, dense, bits);
  return 0;
}

int launch_compact_nonzero(int len, const float* dense, int* key, float* val,
                           int* d_count, ScanScratch& ls, int* err,
                           cudaStream_t st) {
  constexpr int NT = 256, VT = 8;
  (void)err;
  if (len <= 0) { cudaMemsetAsync(d_count, 0, sizeof(int), st); return 0; }
  // ranges of whole sub-tiles, at most kCompactMaxRanges of them
  const long long sub = NT * VT;
  const long long subs = (len + sub - 1) / sub;
  const long long per = sub * ((subs + kCompactMaxRanges - 1) / kCompactMaxRanges);
  const long long ranges = (len + per - 1) / per;
  if (ranges > ls.status_len || !ls.counts) return -1;
  note_launch(2);
  if (launch_pdl(compact_count_kernel<NT, VT>, dim3((unsigned)ranges), dim3(NT), 0, st, (long long)len, per,
                 dense, ls.counts) != cudaSuccess ||
      launch_pdl(compact_write_kernel<NT, VT>, dim3((unsigned)ranges), dim3(NT), 0, st, (long long)len, per,
                 dense, (const unsigned*)ls.counts, key, val, d_count) != cudaSuccess)
    return -2;
  return 0;
}

}  // namespace spmx
