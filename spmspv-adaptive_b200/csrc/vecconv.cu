// Vector-format conversions (H:1121-1393, H:1883-1998; DEV/bitvector.h).
//
// scatter: sparse -> dense and/or bitarray in one kernel (the reference uses a
//   scatter plus a separate set_sparse_x_bitvector launch, H:1271-1308).
// dense2bits: one warp per 32-bit word, ballot of (x != 0); no atomics, no
//   memset (the reference memsets and atomically ORs, and tests `!val`,
//   setting the bits of zeros, H:1362).
// compact_nonzero: dense -> (key, val) of the entries != 0, in index order, in
//   ONE pass: per-warp ballot/popc ranks, a block scan of warp counts and a
//   decoupled look-back across tiles (the reference runs a flag kernel, a CUB
//   scan with a temporary allocation and a compaction kernel, H:1883-1928).
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

template <int NT, int VT>
__global__ void __launch_bounds__(NT)
compact_nonzero_kernel(int len, const float* __restrict__ dense,
                       int* __restrict__ key, float* __restrict__ val,
                       int* d_count, LookbackState st, int ntiles, int* err) {
  constexpr int NW = NT / 32;
  __shared__ unsigned s_cnt[VT * NW];
  __shared__ unsigned s_wtmp[NT / 32 + 1];
  __shared__ int s_tile;
  __shared__ unsigned s_prefix;
  __shared__ unsigned s_total;
  const int tile = lb_acquire_tile(st, ntiles, &s_tile);
  const int base = tile * NT * VT;
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  float v[VT];
  unsigned mask[VT];
#pragma unroll
  for (int j = 0; j < VT; ++j) {
    const int i = base + j * NT + tid;
    v[j] = (i < len) ? __ldg(dense + i) : 0.0f;
    mask[j] = __ballot_sync(0xffffffffu, v[j] != 0.0f);
    if (lane == 0) s_cnt[j * NW + w] = __popc(mask[j]);
  }
  __syncthreads();
  // exclusive scan of the VT*NW counts, in (j, w) order == index order
  unsigned c = (tid < VT * NW) ? s_cnt[tid] : 0u;
  unsigned total;
  const unsigned ex = block_exclusive_sum<NT>(c, s_wtmp, &total);
  if (tid < VT * NW) s_cnt[tid] = ex;
  if (tid < 32) {
    const unsigned p = lb_warp_lookback(st, tile, ntiles, total, err);
    if (tid == 0) { s_prefix = p; s_total = total; }
  }
  __syncthreads();
  const unsigned prefix = s_prefix;
#pragma unroll
  for (int j = 0; j < VT; ++j) {
    if (v[j] != 0.0f) {
      const unsigned pos = prefix + s_cnt[j * NW + w] + __popc(mask[j] & lanemask_lt());
      key[pos] = base + j * NT + tid;
      val[pos] = v[j];
    }
  }
  if (tile == ntiles - 1 && tid == 0) *d_count = (int)(prefix + s_total);
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
  if (len <= 0) { cudaMemsetAsync(d_count, 0, sizeof(int), st); return 0; }
  const int ntiles = (len + NT * VT - 1) / (NT * VT);
  if (ntiles > ls.status_len) return -1;
  LookbackState lbs{ls.status, ls.ticket};
  note_launch();
  compact_nonzero_kernel<NT, VT><<<ntiles, NT, 0, st>>>(len, dense, key, val, d_count,
                                                       lbs, ntiles, err);
  return 0;
}

}  // namespace spmx
