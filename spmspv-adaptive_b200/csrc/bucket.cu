// Bucket-based CSC SpMSpV: y = alpha * A * x with x sparse, written back
// without global atomics on y.
//
// The reference's bucket method (CscBasedBucketSpmspvDriver,
// DEV/csc_bucket_spmspv.cuh:768-1087) counts (row, value) pairs per
// row-block bucket and per x entry, scans and scatters them, but its
// reduction is compiled out (:999-1059) and y is never produced.  This is a
// complete design of our own:
//   1. count:   load-balanced pass over the pairs; per-CTA shared-memory
//               histogram of buckets (bucket = row >> rshift), one global
//               atomic per (CTA, non-empty bucket);
//   2. scan:    bucket offsets (single-pass scan) and a cursor copy;
//   3. scatter: the same pass again; each CTA reserves its range in every
//               bucket with one atomic and places pairs with shared atomics;
//   4. reduce:  one CTA per bucket accumulates its pairs into a dense
//               shared-memory slice of y (shared atomics), writes the slice of
//               the dense y (no memset of y needed) and, in bucket order via a
//               decoupled look-back, the touched rows as sorted (key, value).
#include "kernels.h"
#include "bucket.h"
#include "sort.h"
#include <algorithm>
#include "common.cuh"
#include "engine.h"
#include "csc_lb.cuh"

namespace spmx {

template <int NT, int VT>
__global__ void __launch_bounds__(NT)
bucket_count_kernel(CscArgs a, CscScratch s, int variant, int rshift, int nb,
                    int* __restrict__ gcount) {
  __shared__ LbSmem<NT, VT> sh;
  extern __shared__ int s_hist[];
  const int nblocks = lb_num_blocks(a, s, variant);
  for (int b = blockIdx.x; b < nblocks; b += gridDim.x) {
    for (int i = threadIdx.x; i < nb; i += NT) s_hist[i] = 0;
    const LbBlock bl = lb_block_setup<NT, VT>(a, s, variant, b, nblocks, sh);
    for (int q = threadIdx.x; q < bl.nk; q += NT) {
      int k, r;
      float v;
      lb_item<NT, VT>(a, s, bl, sh, q, k, r, v);
      if ((unsigned)r < (unsigned)a.m) atomicAdd(&s_hist[r >> rshift], 1);
      else flag_error(a.err, kDevErrOob);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += NT)
      if (s_hist[i]) atomicAdd(gcount + i, s_hist[i]);
    __syncthreads();
  }
}

template <int NT, int VT>
__global__ void __launch_bounds__(NT)
bucket_scatter_kernel(CscArgs a, CscScratch s, int variant, int rshift, int nb,
                      int* __restrict__ cursor, int* __restrict__ prow,
                      float* __restrict__ pval, int cap) {
  __shared__ LbSmem<NT, VT> sh;
  extern __shared__ int s_hist[];
  const int nblocks = lb_num_blocks(a, s, variant);
  for (int b = blockIdx.x; b < nblocks; b += gridDim.x) {
    for (int i = threadIdx.x; i < nb; i += NT) s_hist[i] = 0;
    const LbBlock bl = lb_block_setup<NT, VT>(a, s, variant, b, nblocks, sh);
    int rr[VT];
    float vv[VT];
#pragma unroll
    for (int j = 0; j < VT; ++j) {
      const int q = threadIdx.x + j * NT;
      rr[j] = -1;
      if (q < bl.nk) {
        int k;
        lb_item<NT, VT>(a, s, bl, sh, q, k, rr[j], vv[j]);
        if ((unsigned)rr[j] < (unsigned)a.m) atomicAdd(&s_hist[rr[j] >> rshift], 1);
        else rr[j] = -1;
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += NT)
      if (s_hist[i]) s_hist[i] = atomicAdd(cursor + i, s_hist[i]);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < VT; ++j) {
      if (rr[j] >= 0) {
        const int slot = atomicAdd(&s_hist[rr[j] >> rshift], 1);
        if (slot < cap) { prow[slot] = rr[j]; pval[slot] = vv[j]; }
        else flag_error(a.err, kDevErrCapacity);
      }
    }
    __syncthreads();
  }
}

template <int NT>
__global__ void __launch_bounds__(NT)
bucket_reduce_kernel(int m, int rshift, int nb, const int* __restrict__ boff,
                     const int* __restrict__ prow, const float* __restrict__ pval,
                     float* __restrict__ y, int* __restrict__ ykey,
                     float* __restrict__ yval, int* d_count, LookbackState st,
                     int cap, int* err) {
  extern __shared__ float s_dyn[];
  const int R = 1 << rshift;
  float* acc = s_dyn;
  unsigned* tbits = reinterpret_cast<unsigned*>(s_dyn + R);
  const int nwords = R >> 5;
  __shared__ int s_tile;
  __shared__ unsigned s_wtmp[NT / 32 + 1];
  __shared__ unsigned s_prefix, s_total;
  const int bkt = lb_acquire_tile(st, nb, &s_tile);
  const int tid = threadIdx.x;
  for (int i = tid; i < R; i += NT) acc[i] = 0.f;
  for (int i = tid; i < nwords; i += NT) tbits[i] = 0u;
  __syncthreads();
  const int base_row = bkt << rshift;
  const int p0 = min(__ldg(boff + bkt), cap), p1 = min(__ldg(boff + bkt + 1), cap);
  for (int p = p0 + tid; p < p1; p += NT) {
    const int r = __ldg(prow + p) - base_row;
    if ((unsigned)r < (unsigned)R) {
      atomicAdd(&acc[r], __ldg(pval + p));
      atomicOr(&tbits[r >> 5], 1u << (r & 31));
    } else {
      flag_error(err, kDevErrOob);
    }
  }
  __syncthreads();
  const int rows_here = min(R, m - base_row);
  if (y)
    for (int i = tid; i < rows_here; i += NT) y[base_row + i] = acc[i];
  // touched rows of this bucket, in row order, after all earlier buckets
  constexpr int WPT = 1;  // one bitmap word per thread per round
  unsigned cnt = 0;
  for (int wd = tid; wd < nwords; wd += NT * WPT) cnt += __popc(tbits[wd]);
  unsigned total;
  (void)block_exclusive_sum<NT>(cnt, s_wtmp, &total);
  if (tid < 32) {
    const unsigned p = lb_warp_lookback(st, bkt, nb, total, err);
    if (tid == 0) { s_prefix = p; s_total = total; }
  }
  __syncthreads();
  if (ykey) {
    // words in order: round-robin rounds of NT words, exclusive scan per round
    unsigned run = s_prefix;
    for (int w0 = 0; w0 < nwords; w0 += NT) {
      const int wd = w0 + tid;
      const unsigned bits = wd < nwords ? tbits[wd] : 0u;
      unsigned rt;
      const unsigned ex = block_exclusive_sum<NT>((unsigned)__popc(bits), s_wtmp, &rt);
      unsigned pos = run + ex;
      unsigned bb = bits;
      while (bb) {
        const int bit = __ffs(bb) - 1;
        bb &= bb - 1;
        const int rloc = wd * 32 + bit;
        ykey[pos] = base_row + rloc;
        yval[pos] = acc[rloc];
        ++pos;
      }
      run += rt;
    }
  }
  if (bkt == nb - 1 && tid == 0) *d_count = (int)(s_prefix + s_total);
}

int bucket_geometry(int m, int buckets, int* rshift, int* nb) {
  if (buckets <= 0) buckets = 256;
  long long per = ((long long)m + buckets - 1) / buckets;
  int sh = 8;  // at least 256 rows per bucket
  while ((1LL << sh) < per && sh < 13) ++sh;  // at most 8192 rows per bucket
  const long long n = ((long long)m + (1LL << sh) - 1) >> sh;
  if (n > kBucketMax) return -1;
  *rshift = sh;
  *nb = (int)std::max<long long>(n, 1);
  return 0;
}

template <class K>
static void allow_smem(K kernel, int bytes) {
  kernel_smem_limit((const void*)kernel, (size_t)bytes);
}

int launch_bucket_spmspv(const CscArgs& a, const CscScratch& s, const BucketScratch& bs,
                         int variant, int rshift, int nb, float* y, int* ykey,
                         float* yval, int* d_count, ScanScratch& ls, int grid,
                         cudaStream_t st) {
  constexpr int NT = kCscLbNT, VT = kCscLbVT;
  const int hist_bytes = 4 * nb;
  // the limits are per function and device: cached per device, set on each
  // device the first time it runs these kernels
  allow_smem(bucket_count_kernel<NT, VT>, 4 * kBucketMax);
  allow_smem(bucket_scatter_kernel<NT, VT>, 4 * kBucketMax);
  allow_smem(bucket_reduce_kernel<256>, 4 * (8192 + 8192 / 32));
  cudaMemsetAsync(bs.gcount, 0, sizeof(int) * (size_t)nb, st);
  note_launch();
  bucket_count_kernel<NT, VT><<<grid, NT, hist_bytes, st>>>(a, s, variant, rshift, nb, bs.gcount);
  if (launch_scan_exclusive(bs.gcount, bs.boff, nb, bs.boff + nb, ls, a.err, st)) return -1;
  cudaMemcpyAsync(bs.cursor, bs.boff, sizeof(int) * (size_t)nb, cudaMemcpyDeviceToDevice, st);
  note_launch();
  bucket_scatter_kernel<NT, VT><<<grid, NT, hist_bytes, st>>>(a, s, variant, rshift, nb, bs.cursor,
                                                             bs.prow, bs.pval, bs.cap);
  if (nb > ls.status_len) return -1;
  LookbackState lbs{ls.status, ls.ticket};
  const int R = 1 << rshift;
  note_launch();
  bucket_reduce_kernel<256><<<nb, 256, 4 * (R + R / 32), st>>>(
      a.m, rshift, nb, bs.boff, bs.prow, bs.pval, y, ykey, yval, d_count, lbs, bs.cap, a.err);
  return 0;
}

}  // namespace spmx
