#include <algorithm>
// CSC SpMSpV kernels: y = alpha * A * x with x sparse (x_key, x_val).
//
// Stage 1, csc_scan_kernel: gathers the length of every selected column
//   (colptr[k+1]-colptr[k]), scans them into offsets in one pass (decoupled
//   look-back with status words, bounded waits) and, fused into the same pass,
//   writes the block-start tables of both load-balanced partitions.  This
//   replaces scanFuseKernel + DetermineBlockStarts / my_KernelMergePartition
//   (DEV/scan_kernel.cuh:12-143, DEV/csc_two_layer_load_balance.cuh:576,
//   DEV/csc_sort_load_balance.cuh:295) whose look-back spins without bound on
//   `sum[gid-1]==0` (scan_kernel.cuh:99).
//
// Stage 2, csc_lb_kernel: persistent CTAs take blocks of 2048 work items.
//   "twolayer" blocks hold 2048 nonzeros (DEV/csc_two_layer_load_balance_
//   fuse_reduction_modify.cuh:155); "merge" blocks hold 2048 merge-path items
//   = nonzeros + column ends (DEV/csc_sort_load_balance_fuse_reduction_
//   modify.cuh:7), which bounds the number of x entries per block.  Inside a
//   block the owner entry of every item comes from a max-scan over entry-start
//   marks in shared memory (no per-item search), and consecutive threads read
//   consecutive nonzeros of a column.
//
// naive: a group of G lanes per x entry walks its column (ExtractFuseKernel,
//   DEV/csc_sort_spmspv.cuh:98-119, is G = 1).
#include "kernels.h"
#include "common.cuh"
#include "csc_lb.cuh"

namespace spmx {

template <int NT, int VT>
__global__ void __launch_bounds__(NT)
csc_scan_kernel(CscArgs a, CscScratch s, LookbackState st, int ntiles, int K) {
  __shared__ int s_len[NT * VT];
  __shared__ unsigned s_wtmp[NT / 32 + 1];
  __shared__ int s_tile;
  __shared__ unsigned s_prefix;
  const int tile = lb_acquire_tile(st, ntiles, &s_tile);
  const int base = tile * NT * VT;
  const int tid = threadIdx.x;
#pragma unroll
  for (int j = 0; j < VT; ++j) {
    const int i = base + j * NT + tid;
    int len = 0;
    if (i < a.x_nnz) {
      const int key = __ldg(a.x_key + i);
      int cs = 0;
      if ((unsigned)key >= (unsigned)a.n) {
        flag_error(a.err, kDevErrOob);
      } else {
        cs = __ldg(a.colptr + key);
        len = __ldg(a.colptr + key + 1) - cs;
      }
      s.colstart[i] = cs;
    }
    s_len[j * NT + tid] = len;
  }
  __syncthreads();
  unsigned lens[VT];
  unsigned sum = 0;
#pragma unroll
  for (int j = 0; j < VT; ++j) { lens[j] = (unsigned)s_len[tid * VT + j]; sum += lens[j]; }
  unsigned total;
  const unsigned ex = block_exclusive_sum<NT>(sum, s_wtmp, &total);
  if (tid < 32) {
    const unsigned p = lb_warp_lookback(st, tile, ntiles, total, a.err);
    if (tid == 0) s_prefix = p;
  }
  __syncthreads();
  unsigned prefix = s_prefix + ex;
#pragma unroll
  for (int j = 0; j < VT; ++j) {
    const int i = base + tid * VT + j;
    if (i < a.x_nnz) {
      s.off[i] = (int)prefix;
      const long long p = prefix, len = lens[j];
      if (len > 0) {
        for (long long b = (p + K - 1) / K; b * K < p + len; ++b) {
          if (b < s.tl_cap) s.bstart_tl[b] = i; else flag_error(a.err, kDevErrCapacity);
        }
      }
      const long long lo = p + i, hi = p + len + i + 1;
      for (long long b = (lo + K - 1) / K; b * K < hi; ++b) {
        if (b < s.mg_cap) s.bstart_mg[b] = i; else flag_error(a.err, kDevErrCapacity);
      }
      prefix += lens[j];
    }
  }
  if (tile == ntiles - 1 && tid == 0) {
    const long long bl = (long long)s_prefix + total;
    s.off[a.x_nnz] = (int)bl;
    a.counts[kCntBinlen] = (int)bl;
    a.counts[kCntBlocksTL] = (int)((bl + K - 1) / K);
    a.counts[kCntBlocksMG] = (int)((bl + a.x_nnz + K - 1) / K);
  }
}

template <int NT, int VT, bool PAIRS>
__global__ void __launch_bounds__(NT)
csc_lb_kernel(CscArgs a, CscScratch s, int variant, float* __restrict__ y,
              int* __restrict__ prow, float* __restrict__ pval) {
  __shared__ LbSmem<NT, VT> sh;
  const int nblocks = lb_num_blocks(a, s, variant);
  for (int b = blockIdx.x; b < nblocks; b += gridDim.x) {
    const LbBlock bl = lb_block_setup<NT, VT>(a, s, variant, b, nblocks, sh);
    for (int q = threadIdx.x; q < bl.nk; q += NT) {
      int k, r;
      float v;
      lb_item<NT, VT>(a, s, bl, sh, q, k, r, v);
      if (PAIRS) {
        prow[k] = r;
        pval[k] = v;
      } else if ((unsigned)r < (unsigned)a.m) {
        atomicAdd(y + r, v);
      } else {
        flag_error(a.err, kDevErrOob);
      }
    }
    __syncthreads();
  }
}

// y is zero-filled by the grid launched before this one (zero_fill_kernel).
// With programmatic dependent launch this grid starts early: it reads x, the
// column bounds and the first row / value while y is being cleared, and waits
// (griddepcontrol.wait, a no-op without the launch attribute) only before its
// first atomic.
template <int G, int U>
__global__ void __launch_bounds__(256)
csc_naive_kernel(CscArgs a, float* __restrict__ y) {
  // G lanes per x entry; each lane group takes U entries, gid / G + u * groups,
  // whose loads are issued phase by phase (all keys, then all column bounds,
  // then all first nonzeros), so one chain of memory round trips covers U
  // entries
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long groups = (long long)gridDim.x * blockDim.x / G;
  const int g = (int)(gid % G);
  int key[U], cs[U], ce[U], r0[U];
  float xv[U], v0[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const long long i = gid / G + u * groups;
    key[u] = i < a.x_nnz ? __ldg(a.x_key + i) : -1;
    xv[u] = i < a.x_nnz ? __ldg(a.x_val + i) : 0.f;
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const long long i = gid / G + u * groups;
    const bool ok = (unsigned)key[u] < (unsigned)a.n;
    if (i < a.x_nnz && !ok && g == 0) flag_error(a.err, kDevErrOob);
    cs[u] = ok ? __ldg(a.colptr + key[u]) : 0;
    ce[u] = ok ? __ldg(a.colptr + key[u] + 1) : 0;
    xv[u] = (float)(a.alpha * (double)xv[u]);
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    r0[u] = -1;
    v0[u] = 0.f;
    if (cs[u] + g < ce[u]) {
      r0[u] = __ldg(a.row + cs[u] + g);
      v0[u] = __ldg(a.val + cs[u] + g);
    }
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");
  // the next call's first grid may launch now (it waits for this one before
  // it touches memory)
  asm volatile("griddepcontrol.launch_dependents;");
#pragma unroll
  for (int u = 0; u < U; ++u) {
    if (cs[u] + g < ce[u]) {
      if ((unsigned)r0[u] < (unsigned)a.m) atomicAdd(y + r0[u], v0[u] * xv[u]);
      else flag_error(a.err, kDevErrOob);
    }
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
#pragma unroll 4
    for (int k = cs[u] + g + G; k < ce[u]; k += G) {
      const int r = __ldg(a.row + k);
      if ((unsigned)r < (unsigned)a.m) atomicAdd(y + r, __ldg(a.val + k) * xv[u]);
      else flag_error(a.err, kDevErrOob);
    }
  }
}

template <int G>
__global__ void __launch_bounds__(256)
csc_naive_pairs_kernel(CscArgs a, CscScratch s, int* __restrict__ prow,
                       float* __restrict__ pval) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(gid / G);
  const int g = (int)(gid % G);
  if (i >= a.x_nnz) return;
  const int cs = __ldg(s.colstart + i);
  const int o = __ldg(s.off + i);
  const int len = __ldg(s.off + i + 1) - o;
  const float xv = (float)(a.alpha * (double)__ldg(a.x_val + i));
  for (int q = g; q < len; q += G) {
    prow[o + q] = __ldg(a.row + cs + q);
    pval[o + q] = __ldg(a.val + cs + q) * xv;
  }
}

// --------------------------------------------------------------------------
int launch_csc_scan(const CscArgs& a, const CscScratch& s, ScanScratch& ls,
                    int block_items, cudaStream_t st) {
  constexpr int NT = kCscScanNT, VT = kCscScanVT;
  const int ntiles = (a.x_nnz + NT * VT - 1) / (NT * VT);
  if (ntiles <= 0) return 0;
  if (ntiles > ls.status_len) return -1;
  LookbackState lbs{ls.status, ls.ticket};
  note_launch();
  csc_scan_kernel<NT, VT><<<ntiles, NT, 0, st>>>(a, s, lbs, ntiles, block_items);
  return 0;
}

int launch_csc_lb(const CscArgs& a, const CscScratch& s, int variant, float* y,
                  int* pairs_row, float* pairs_val, int grid, cudaStream_t st) {
  constexpr int NT = kCscLbNT, VT = kCscLbVT;
  if (a.x_nnz <= 0 || grid <= 0) return 0;
  note_launch();
  if (pairs_row)
    csc_lb_kernel<NT, VT, true><<<grid, NT, 0, st>>>(a, s, variant, y, pairs_row, pairs_val);
  else
    csc_lb_kernel<NT, VT, false><<<grid, NT, 0, st>>>(a, s, variant, y, pairs_row, pairs_val);
  return 0;
}

#define SPMX_GROUP_SWITCH(G_, BODY)                                              \
  switch (G_) {                                                                 \
    case 1: { constexpr int G = 1; BODY; break; }                               \
    case 2: { constexpr int G = 2; BODY; break; }                               \
    case 4: { constexpr int G = 4; BODY; break; }                               \
    case 8: { constexpr int G = 8; BODY; break; }                               \
    case 16: { constexpr int G = 16; BODY; break; }                             \
    case 32: { constexpr int G = 32; BODY; break; }                             \
    default: return -1;                                                         \
  }

// y[0..m) = 0.  Launched as a programmatic dependent of the grid before it on
// the stream, it waits for that grid before its first store, and only then
// lets the next grid launch: a dependent that reads its inputs before its own
// wait (x keys, column bounds) therefore never starts while a grid that
// writes them is still running.
__global__ void zero_fill_kernel(float* __restrict__ y, long long m) {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;");
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nt = (long long)gridDim.x * blockDim.x;
  if ((((uintptr_t)y) & 15u) == 0) {
    float4* y4 = reinterpret_cast<float4*>(y);
    const long long m4 = m >> 2;
    for (long long i = tid; i < m4; i += nt) y4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (long long i = (m4 << 2) + tid; i < m; i += nt) y[i] = 0.f;
  } else {
    for (long long i = tid; i < m; i += nt) y[i] = 0.f;
  }
}

// The zero fill opens a call, so it is launched as a programmatic dependent of
// whatever grid ran before it (the previous call's last kernel): its launch
// and CTA start-up overlap that grid's tail (2.4 -> 1.2 us per kernel boundary
// measured on B200), and its griddepcontrol.wait keeps the order.
int launch_zero_fill(float* y, long long m, int num_sms, cudaStream_t st) {
  if (m <= 0) return 0;
  const long long blocks = std::min<long long>((m + 1023) / 1024, (long long)num_sms * 4);
  note_launch();
  return launch_pdl(zero_fill_kernel, dim3((unsigned)std::max(1LL, blocks)), dim3(256), 0, st, y, m) ==
                 cudaSuccess
             ? 0
             : -2;
}

// zero y, then the naive CSC SpMSpV as a programmatic dependent launch
int launch_csc_naive_zeroed(const CscArgs& a, int group, float* y, int num_sms, cudaStream_t st) {
  if (a.m > 0 && launch_zero_fill(y, a.m, num_sms, st)) return -2;
  if (a.x_nnz <= 0) return 0;
  // entries per lane group: enough that the grid is about one wave of
  // resident threads (2,048 per SM), at most 4
  const long long threads = (long long)a.x_nnz * group;
  const long long resident = (long long)num_sms * 2048;
  const int U = threads <= resident ? 1 : threads <= 2 * resident ? 2 : 4;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)((threads + 256LL * U - 1) / (256LL * U)));
  cfg.blockDim = dim3(256);
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  note_launch();
  cudaError_t e = cudaSuccess;
  if (U == 1) {
    SPMX_GROUP_SWITCH(group, (e = cudaLaunchKernelEx(&cfg, csc_naive_kernel<G, 1>, a, y)));
  } else if (U == 2) {
    SPMX_GROUP_SWITCH(group, (e = cudaLaunchKernelEx(&cfg, csc_naive_kernel<G, 2>, a, y)));
  } else {
    SPMX_GROUP_SWITCH(group, (e = cudaLaunchKernelEx(&cfg, csc_naive_kernel<G, 4>, a, y)));
  }
  return e == cudaSuccess ? 0 : -2;
}

int launch_csc_naive(const CscArgs& a, int group, float* y, cudaStream_t st) {
  if (a.x_nnz <= 0) return 0;
  const long long threads = (long long)a.x_nnz * group;
  const unsigned grid = (unsigned)((threads + 255) / 256);
  note_launch();
  SPMX_GROUP_SWITCH(group, (csc_naive_kernel<G, 1><<<grid, 256, 0, st>>>(a, y)));
  return 0;
}

int launch_csc_naive_pairs(const CscArgs& a, const CscScratch& s, int group,
                           int* pairs_row, float* pairs_val, cudaStream_t st) {
  if (a.x_nnz <= 0) return 0;
  const long long threads = (long long)a.x_nnz * group;
  const unsigned grid = (unsigned)((threads + 255) / 256);
  note_launch();
  SPMX_GROUP_SWITCH(group, (csc_naive_pairs_kernel<G><<<grid, 256, 0, st>>>(a, s, pairs_row, pairs_val)));
  return 0;
}

}  // namespace spmx

namespace spmx {
int csc_lb_blocks_per_sm() {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &b, csc_lb_kernel<kCscLbNT, kCscLbVT, false>, kCscLbNT, 0) != cudaSuccess) {
    cudaGetLastError();
    return 2;
  }
  return b > 0 ? b : 1;
}
}  // namespace spmx
