// Block mapping shared by the load-balanced CSC kernels (csc.cu, bucket.cu).
//
// Work item k (0 <= k < bin_len) is the k-th nonzero of the concatenation of
// x's columns, in x order.  A block covers a contiguous range of items:
//   variant 1 ("merge"):    2048 merge-path items (nonzeros + column ends), so
//                           at most 2049 x entries touch a block;
//   variant 2 ("twolayer"): 2048 nonzeros; a block may span many empty columns.
// lb_block_setup stages the entries of the block in shared memory and resolves
// the owner entry of every item with a max-scan over entry-start marks;
// lb_item then maps item q of the block to (k, row, alpha*val*x).
#pragma once
#include "common.cuh"
#include "kernels.h"

namespace spmx {

template <int NT, int VT>
struct LbSmem {
  static constexpr int K = NT * VT;
  static constexpr int CAP = K + 1;
  int off[CAP];
  int cs[CAP];
  float xv[CAP];
  int mark[K];
  int incl[NT];
  int wtmp[NT / 32 + 1];
};

struct LbBlock {
  int i0, i1, k0, nk;
  bool in_smem;
};

__device__ __forceinline__ int lb_num_blocks(const CscArgs& a, const CscScratch& s,
                                             int variant) {
  int nblocks = a.counts[variant == 1 ? kCntBlocksMG : kCntBlocksTL];
  const int cap = variant == 1 ? s.mg_cap : s.tl_cap;
  if (nblocks > cap) {  // only with duplicate x keys (bin_len > nnz)
    if (blockIdx.x == 0 && threadIdx.x == 0) flag_error(a.err, kDevErrCapacity);
    nblocks = cap;
  }
  return nblocks;
}

// Ends with __syncthreads(); the caller must __syncthreads() before the next
// setup reuses the shared memory.
template <int NT, int VT>
__device__ __forceinline__ LbBlock lb_block_setup(const CscArgs& a, const CscScratch& s,
                                                  int variant, int b, int nblocks,
                                                  LbSmem<NT, VT>& sh) {
  constexpr int K = NT * VT;
  const int tid = threadIdx.x;
  const int bin_len = a.counts[kCntBinlen];
  const int x_nnz = a.x_nnz;
  const int* bstart = variant == 1 ? s.bstart_mg : s.bstart_tl;
  LbBlock bl;
  bl.i0 = bstart[b];
  int k1;
  if (variant == 1) {
    const long long d0 = (long long)b * K;
    const long long d1 = min(d0 + K, (long long)bin_len + x_nnz);
    bl.k0 = (int)(d0 - bl.i0);
    if (b + 1 < nblocks) { bl.i1 = bstart[b + 1]; k1 = (int)(d1 - bl.i1); }
    else { bl.i1 = x_nnz - 1; k1 = bin_len; }
  } else {
    bl.k0 = b * K;
    k1 = min(bl.k0 + K, bin_len);
    bl.i1 = (b + 1 < nblocks) ? bstart[b + 1] : x_nnz - 1;
  }
  bl.nk = k1 - bl.k0;
  const int ne = bl.i1 - bl.i0 + 1;
  bl.in_smem = ne <= LbSmem<NT, VT>::CAP;
  if (bl.in_smem) {
    for (int e = tid; e < ne; e += NT) {
      sh.off[e] = __ldg(s.off + bl.i0 + e);
      sh.cs[e] = __ldg(s.colstart + bl.i0 + e);
      sh.xv[e] = (float)(a.alpha * (double)__ldg(a.x_val + bl.i0 + e));
    }
    for (int q = tid; q < K; q += NT) sh.mark[q] = -1;
    __syncthreads();
    for (int e = tid; e < ne; e += NT) {
      const int p = sh.off[e] - bl.k0;
      if (p >= 0 && p < bl.nk) atomicMax(&sh.mark[p], e);
    }
    __syncthreads();
    int loc[VT];
    int run = INT_MIN;
#pragma unroll
    for (int j = 0; j < VT; ++j) {
      const int q = tid * VT + j;
      int v = sh.mark[q];
      if (q == 0) v = max(v, 0);
      run = max(run, v);
      loc[j] = run;
    }
    const int inc = block_inclusive_max<NT>(run, sh.wtmp);
    sh.incl[tid] = inc;
    __syncthreads();
    const int carry = tid ? sh.incl[tid - 1] : INT_MIN;
#pragma unroll
    for (int j = 0; j < VT; ++j) sh.mark[tid * VT + j] = max(loc[j], carry);
  }
  __syncthreads();
  return bl;
}

template <int NT, int VT>
__device__ __forceinline__ void lb_item(const CscArgs& a, const CscScratch& s,
                                        const LbBlock& bl, const LbSmem<NT, VT>& sh,
                                        int q, int& k, int& r, float& v) {
  k = bl.k0 + q;
  if (bl.in_smem) {
    const int e = sh.mark[q];
    const int pos = sh.cs[e] + (k - sh.off[e]);
    r = __ldg(a.row + pos);
    v = __ldg(a.val + pos) * sh.xv[e];
  } else {
    int lo = bl.i0, hi = bl.i1;  // last i in [i0, i1] with off[i] <= k
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(s.off + mid) <= k) lo = mid; else hi = mid - 1;
    }
    const int pos = __ldg(s.colstart + lo) + (k - __ldg(s.off + lo));
    r = __ldg(a.row + pos);
    v = __ldg(a.val + pos) * (float)(a.alpha * (double)__ldg(a.x_val + lo));
  }
}

}  // namespace spmx
