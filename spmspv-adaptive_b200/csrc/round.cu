// Round SpMV / bitmap-gated SpMSpV (y = alpha * A * x): a fourth
// load-balanced back-end beside Hola, CSR5 and the tiled SpMV (spmv_type 3;
// no reference counterpart).
//
// Why: a row-ordered SpMV gathers x one cache line per nonzero (about one
// line per cycle per SM on B200), and the tiled back-end, which stages x
// windows in shared memory, pays a producer/consumer handshake per (row
// block, x window) tile.  Here the nonzeros of a row block are streamed in
// COLUMN order, so the 32 lanes of a warp gather x from a few neighbouring
// cache lines, and the accumulation into y is made race-free without atomics
// by a transpose through shared memory:
//
//   - rows are cut into row blocks whose y fits in shared memory; a row block
//     is processed by a cluster of 2 CTAs, each taking one half (in column
//     order) of the block's nonzeros, sorted by (column, row);
//   - a CTA's nonzeros are cut into rounds of E = 8192.  Phase 1: each of the
//     32 warps takes 256 consecutive nonzeros of the round (16-byte loads of
//     the stream, lanes interleaved so that consecutive lanes hold
//     consecutive nonzeros), gathers x, multiplies and stores the product
//     into the nonzero's slot of a shared product buffer.  The slots put the
//     round's products in row order, the rows of each warp together, each
//     warp's part lane-interleaved (entry j of lane l's contiguous range at
//     32 j + l);
//   - after a CTA barrier, phase 2: every warp reduces the products of the
//     rows it owns (fixed row ranges of equal nonzero counts) into the shared
//     y: a lane adds each run of equal rows that ends inside its range, and
//     the runs still open at the range ends are summed with a segmented scan.
//     No two lanes or warps ever update one row at once, and every row's
//     additions happen in a fixed order: the result is deterministic;
//   - the products are double-buffered, so one barrier per round suffices;
//     the row indices of a round (2 bytes per nonzero, in slot order) arrive
//     by a bulk copy issued one round ahead, the stream words of the next
//     round are loaded during the current one and L2 prefetches run three
//     rounds ahead;
//   - at the end the 2 CTAs of a cluster add their partial y vectors in rank
//     order through distributed shared memory and store each row once.
//
// Stream per nonzero: a 32-bit word (column offset from the round's first
// column << 13 | slot), the value (4 bytes) and the local row (2 bytes).
// Every wait is bounded: a timeout sets the device error word and the kernel
// keeps every thread on the same barrier sequence until it returns.
#include <algorithm>
#include <cooperative_groups.h>
#include <string>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "kernels.h"
#include "sort.h"

namespace cg = cooperative_groups;

namespace spmx {

constexpr int kRoundE = 8192;             // nonzeros per round
constexpr int kRoundSlotBits = 13;        // log2(kRoundE)
constexpr int kRoundNW = 32;              // warps per CTA
constexpr int kRoundCS = 2;               // CTAs per cluster (per row block)
constexpr int kRoundPL = kRoundE / (kRoundNW * 32);  // phase-1 nonzeros per lane
constexpr unsigned kRoundSpan = 1u << (32 - kRoundSlotBits);  // column offsets must stay below
constexpr long long kRoundSpin = 1LL << 22;
static_assert(kRoundPL % 4 == 0, "16-byte stream loads");

struct RoundTables {
  int nrb = 0, grid = 0, rmax = 0, nrounds = 0;
  size_t smem = 0;
  int* rb_row = nullptr;     // nrb + 1 row block boundaries
  int* cta_round = nullptr;  // grid + 1: rounds of CTA c are [cta_round[c], cta_round[c + 1])
  unsigned* packed = nullptr;        // nrounds * E stream words (phase-1 order, interleaved)
  float* val = nullptr;              // nrounds * E values (same order)
  unsigned short* row16 = nullptr;   // nrounds * E local rows (slot order)
  int* rbase = nullptr;              // nrounds first columns
  int* roff = nullptr;               // nrounds * (NW + 1) warp part offsets (slot order)
};

static RoundTables* rtab(spmx_handle_t h) { return reinterpret_cast<RoundTables*>(h->round); }

namespace {

__device__ __forceinline__ unsigned rsa(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool round_wait(unsigned long long* b, int parity) {
  for (long long it = 0; it < kRoundSpin; ++it) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(rsa(b)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// bulk copy of one round's rows into shared memory, counted on barrier b
__device__ __forceinline__ void round_copy_rows(unsigned short* dst, const unsigned short* src,
                                                unsigned long long* b) {
  constexpr unsigned bytes = 2u * kRoundE;
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(rsa(b)), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(rsa(dst)),
      "l"(src), "r"(bytes), "r"(rsa(b))
      : "memory");
}

__device__ __forceinline__ void round_l2_prefetch(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// A warp reduces its part [lo, hi) of a round's products (row order,
// lane-interleaved: entry j of lane l's contiguous range at lo + 32 j + l;
// the first (hi - lo) % 32 lanes hold one entry more) into ys.  A run of
// equal rows that ends inside a lane's range is added by that lane when it
// ends; no other lane ends it, and the warp's instructions are ordered, so
// two lanes never update one row in one instruction.  The runs open at the
// range ends have non-decreasing rows across the lanes; a segmented scan sums
// each group and its last lane adds the sum.
template <int G>
__device__ __forceinline__ void round_warp_reduce(int lo, int hi, const unsigned short* __restrict__ R,
                                                  const float* __restrict__ Pp, float* __restrict__ ys) {
  const int lane = threadIdx.x & 31;
  const int len = hi - lo;
  if (len <= 0) return;  // warp-uniform
  const int per = len >> 5, rem = len & 31;
  const int cnt = per + (lane < rem ? 1 : 0);
  int cur = -1;
  float acc = 0.f;
  for (int j0 = 0; j0 < cnt; j0 += G) {
    const int ng = min(G, cnt - j0);
    int rw[G];
    float pr[G];
#pragma unroll
    for (int j = 0; j < G; ++j) {
      rw[j] = j < ng ? (int)R[lo + 32 * (j0 + j) + lane] : 0;
      pr[j] = j < ng ? Pp[lo + 32 * (j0 + j) + lane] : 0.f;
    }
#pragma unroll
    for (int j = 0; j < G; ++j) {
      if (j < ng) {
        if (rw[j] != cur) {
          if (cur >= 0) ys[cur] += acc;
          cur = rw[j];
          acc = pr[j];
        } else {
          acc += pr[j];
        }
      }
    }
  }
  float S = acc;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const float oS = __shfl_up_sync(0xffffffffu, S, d);
    const int oc = __shfl_up_sync(0xffffffffu, cur, d);
    if (lane >= d && oc == cur) S += oS;
  }
  const int nc = __shfl_down_sync(0xffffffffu, cur, 1);
  if (cur >= 0 && (lane == 31 || nc != cur)) ys[cur] += S;
  __syncwarp();
}

// shared memory: 2 mbarriers (128 bytes), products 2 x E floats, rows 2 x E
// shorts, y (rmax floats)
__host__ __device__ constexpr size_t round_smem_fixed() { return 128 + 4 * 2 * kRoundE + 2 * 2 * kRoundE; }

template <bool GATED>
__global__ void __launch_bounds__(kRoundNW * 32, 1)
round_spmv_kernel(const int* __restrict__ rb_row, const int* __restrict__ cta_round,
                  const unsigned* __restrict__ packed, const float* __restrict__ val,
                  const unsigned short* __restrict__ row16, const int* __restrict__ rbase,
                  const int* __restrict__ roff, const float* __restrict__ x, const unsigned* __restrict__ xbits,
                  float alpha, float* __restrict__ y, int* err) {
  constexpr int E = kRoundE, NW = kRoundNW, PL = kRoundPL, DB = kRoundSlotBits;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem);
  float* P = reinterpret_cast<float*>(smem + 128);
  unsigned short* Rs = reinterpret_cast<unsigned short*>(P + 2 * E);
  float* ys = reinterpret_cast<float*>(Rs + 2 * E);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rb = blockIdx.x / kRoundCS;
  const int row0 = __ldg(rb_row + rb), rows = __ldg(rb_row + rb + 1) - row0;
  const int rows4 = (rows + 3) & ~3;
  for (int r = threadIdx.x; r < rows4; r += blockDim.x) ys[r] = 0.f;
  const int k0 = __ldg(cta_round + blockIdx.x), k1 = __ldg(cta_round + blockIdx.x + 1);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(rsa(bars)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(rsa(bars + 1)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // launched as a programmatic dependent of the grid that writes x: nothing
  // above touches x or y
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (threadIdx.x == 0 && k0 < k1) {
    round_copy_rows(Rs, row16 + (size_t)k0 * E, bars);
    for (int q = k0 + 1; q < min(k1, k0 + 4); ++q) {
      round_l2_prefetch(packed + (size_t)q * E, 4u * E);
      round_l2_prefetch(val + (size_t)q * E, 4u * E);
      round_l2_prefetch(row16 + (size_t)q * E, 2u * E);
    }
  }
  unsigned pw[PL];
  float pv[PL];
  int nbase = 0, nlo = 0, nhi = 0;
  auto load_round = [&](int q) {
#pragma unroll
    for (int i = 0; i < PL / 4; ++i) {
      const size_t e = (size_t)q * E + warp * (E / NW) + 128 * i + 4 * lane;
      const uint4 a = __ldcs(reinterpret_cast<const uint4*>(packed + e));
      const float4 v = __ldcs(reinterpret_cast<const float4*>(val + e));
      pw[4 * i] = a.x;
      pw[4 * i + 1] = a.y;
      pw[4 * i + 2] = a.z;
      pw[4 * i + 3] = a.w;
      pv[4 * i] = v.x;
      pv[4 * i + 1] = v.y;
      pv[4 * i + 2] = v.z;
      pv[4 * i + 3] = v.w;
    }
    nbase = __ldg(rbase + q);
    nlo = __ldg(roff + (size_t)q * (NW + 1) + warp);
    nhi = __ldg(roff + (size_t)q * (NW + 1) + warp + 1);
  };
  if (k0 < k1) load_round(k0);
  bool timed_out = false;
  for (int k = k0; k < k1; ++k) {
    const int b = (k - k0) & 1;
    float* Pk = P + b * E;
    const int base = nbase, lo = nlo, hi = nhi;
    // phase 1: gather in column order, products to their row-order slots
    float xv[PL];
#pragma unroll
    for (int i = 0; i < PL; ++i) xv[i] = __ldg(x + base + (int)(pw[i] >> DB));
    unsigned dst[PL];
    float pr[PL];
#pragma unroll
    for (int i = 0; i < PL; ++i) {
      dst[i] = pw[i] & (E - 1);
      float p = pv[i] * xv[i];
      if (GATED) {
        const int c = base + (int)(pw[i] >> DB);
        if (!((__ldg(xbits + (c >> 5)) >> (c & 31)) & 1u)) p = 0.f;
      }
      pr[i] = p;
    }
    if (k + 1 < k1) load_round(k + 1);
#pragma unroll
    for (int i = 0; i < PL; ++i) Pk[dst[i]] = pr[i];
    __syncthreads();
    // every warp has finished phase 2 of round k - 1: refill its row buffer
    if (threadIdx.x == 0 && k + 1 < k1) {
      round_copy_rows(Rs + (1 - b) * E, row16 + (size_t)(k + 1) * E, bars + (1 - b));
      if (k + 4 < k1) {
        round_l2_prefetch(packed + (size_t)(k + 4) * E, 4u * E);
        round_l2_prefetch(val + (size_t)(k + 4) * E, 4u * E);
        round_l2_prefetch(row16 + (size_t)(k + 4) * E, 2u * E);
      }
    }
    // phase 2: every lane waits for the rows (acquire); a timeout skips the
    // reduction but keeps the barrier sequence
    const bool got = __all_sync(0xffffffffu, round_wait(bars + b, ((k - k0) >> 1) & 1));
    if (got) {
      round_warp_reduce<8>(lo, hi, Rs + b * E, Pk, ys);
    } else if (!timed_out) {
      timed_out = true;
      if (lane == 0) flag_error(err, kDevErrTimeout);
    }
  }
  __syncthreads();
  cg::cluster_group cl = cg::this_cluster();
  cl.sync();
  const int rank = (int)cl.block_rank();
  const int slice = (((rows + kRoundCS - 1) / kRoundCS) + 3) & ~3;
  const int r0 = rank * slice, r1 = min(rows, r0 + slice);
  for (int r = r0 + 4 * (int)threadIdx.x; r < r1; r += 4 * (int)blockDim.x) {
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int q = 0; q < kRoundCS; ++q) {
      const float4 v = *reinterpret_cast<const float4*>(cl.map_shared_rank(ys + r, q));
      acc.x += v.x;
      acc.y += v.y;
      acc.z += v.z;
      acc.w += v.w;
    }
    const float a4[4] = {acc.x, acc.y, acc.z, acc.w};
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (r + j < r1) y[row0 + r + j] = alpha * a4[j];
  }
  cl.sync();  // peers read this CTA's shared y until here
}

// ---------------------------------------------------------------------------
// preprocessing
// ---------------------------------------------------------------------------

// sort key of every nonzero: (row block << cbits) | column, payloads local
// row and value bits.  A column outside [0, n) gets the dump key
// nrb << cbits (it sorts after every valid key and is dropped).
__global__ void round_keys_kernel(int m, int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                                  const float* __restrict__ val, const int* __restrict__ rb_row, int nrb, int cbits,
                                  unsigned* __restrict__ key, unsigned* __restrict__ lrow,
                                  unsigned* __restrict__ vbits, int* __restrict__ flags) {
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // one warp per row
  const int lane = threadIdx.x & 31;
  if (gw >= m) return;
  const int r = (int)gw;
  int lo = 0, hi = nrb;  // row block: the last b with rb_row[b] <= r
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(rb_row + mid) <= r) lo = mid;
    else hi = mid;
  }
  const unsigned lr = (unsigned)(r - __ldg(rb_row + lo));
  const int a = __ldg(rowptr + r), b = __ldg(rowptr + r + 1);
  for (int k = a + lane; k < b; k += 32) {
    const int c = __ldg(col + k);
    if ((unsigned)c >= (unsigned)n) {
      atomicOr(flags, 1);
      key[k] = (unsigned)nrb << cbits;
      lrow[k] = 0;
      vbits[k] = 0;
      continue;
    }
    key[k] = ((unsigned)lo << cbits) | (unsigned)c;
    lrow[k] = lr;
    vbits[k] = __float_as_uint(__ldg(val + k));
  }
}

// out[t] = first sorted position with key >= t << cbits, t in [0, nrb]
__global__ void round_bounds_kernel(int nnz, const unsigned* __restrict__ skey, int nrb, int cbits,
                                    int* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t > nrb) return;
  const unsigned want = (unsigned)t << cbits;
  int lo = 0, hi = nnz;
  while (lo < hi) {
    const int mid = (int)(((long long)lo + hi) >> 1);
    if (__ldg(skey + mid) < want) lo = mid + 1;
    else hi = mid;
  }
  out[t] = lo;
}

// one CTA per round: the second sort's keys (round << 16 | local row, stable
// over the round's column order) and positions; the round's first column;
// a column span beyond the slot word's offset field sets flags bit 1
__global__ void round_key2_kernel(const int* __restrict__ rstart, const int* __restrict__ rlen,
                                  const unsigned* __restrict__ skey, const unsigned* __restrict__ slrow, unsigned cmask,
                                  unsigned* __restrict__ key2, unsigned* __restrict__ pos2, int* __restrict__ rbase,
                                  int* __restrict__ flags) {
  const int q = blockIdx.x;
  const int s = __ldg(rstart + q), len = __ldg(rlen + q);
  for (int i = threadIdx.x; i < len; i += blockDim.x) {
    key2[s + i] = ((unsigned)q << 16) | __ldg(slrow + s + i);
    pos2[s + i] = (unsigned)i;
  }
  if (threadIdx.x == 0) {
    const unsigned c0 = __ldg(skey + s) & cmask, c1 = __ldg(skey + s + len - 1) & cmask;
    rbase[q] = (int)c0;
    if (c1 - c0 >= kRoundSpan) atomicOr(flags, 2);
  }
}

// storage position of phase-1 position p: each 128-entry block is stored so
// that a lane's 16-byte word holds entries l, l + 32, l + 64, l + 96
__device__ __forceinline__ int round_vperm(int p) {
  const int blk = p >> 7, c = (p >> 5) & 3, l = p & 31;
  return (blk << 7) + 4 * l + c;
}

// one CTA per round: warp part offsets (row order), slots, and the streams
__global__ void __launch_bounds__(256)
round_layout_kernel(const int* __restrict__ rstart, const int* __restrict__ rlen, const int* __restrict__ rrb,
                    const int* __restrict__ wsp, const unsigned* __restrict__ skey, const unsigned* __restrict__ sval,
                    unsigned cmask, const unsigned* __restrict__ key2, const unsigned* __restrict__ pos2,
                    const int* __restrict__ rbase, unsigned* __restrict__ packed, float* __restrict__ val,
                    unsigned short* __restrict__ row16, int* __restrict__ roff) {
  constexpr int NW = kRoundNW, E = kRoundE, DB = kRoundSlotBits;
  __shared__ int off[NW + 1];
  const int q = blockIdx.x;
  const int s = __ldg(rstart + q), len = __ldg(rlen + q);
  const int base = __ldg(rbase + q);
  const int* ws = wsp + (size_t)__ldg(rrb + q) * (NW + 1);
  if (threadIdx.x <= NW) {
    // first entry of the round (row order) whose local row >= the split
    const unsigned split = (unsigned)__ldg(ws + threadIdx.x);
    int lo = 0, hi = len;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if ((__ldg(key2 + s + mid) & 0xffffu) < split) lo = mid + 1;
      else hi = mid;
    }
    off[threadIdx.x] = threadIdx.x == NW ? len : lo;
    roff[(size_t)q * (NW + 1) + threadIdx.x] = threadIdx.x == NW ? len : lo;
  }
  __syncthreads();
  const size_t o = (size_t)q * E;
  for (int t = threadIdx.x; t < E; t += blockDim.x) {
    if (t < len) {
      // row-order index t: owner warp, lane range, slot
      int w = 0;
      while (w < NW - 1 && off[w + 1] <= t) ++w;
      const int L = off[w + 1] - off[w], u = t - off[w];
      const int per = L >> 5, rem = L & 31;
      int lane, j;
      if (u < rem * (per + 1)) {
        lane = u / (per + 1);
        j = u - lane * (per + 1);
      } else {
        const int u2 = u - rem * (per + 1);
        lane = rem + u2 / per;
        j = u2 - (lane - rem) * per;
      }
      const int slot = off[w] + 32 * j + lane;
      const int pos = (int)__ldg(pos2 + s + t);
      row16[o + slot] = (unsigned short)(__ldg(key2 + s + t) & 0xffffu);
      const unsigned c = __ldg(skey + s + pos) & cmask;
      const int sp = round_vperm(pos);
      packed[o + sp] = ((c - (unsigned)base) << DB) | (unsigned)slot;
      val[o + sp] = __uint_as_float(__ldg(sval + s + pos));
    } else {
      // padding: the unused slots [len, E), column offset 0, value 0
      const int sp = round_vperm(t);
      packed[o + sp] = (unsigned)t;
      val[o + sp] = 0.f;
      row16[o + t] = 0;
    }
  }
}

int bits_for(long long v) {  // bits to hold values in [0, v)
  int b = 1;
  while (b < 62 && (1LL << b) < v) ++b;
  return b;
}

template <bool GATED>
static void round_set_smem(size_t smem) {
  cudaFuncSetAttribute(round_spmv_kernel<GATED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

static long long round_static_smem() {
  cudaFuncAttributes a = {};
  if (cudaFuncGetAttributes(&a, round_spmv_kernel<true>) != cudaSuccess) {
    cudaGetLastError();
    return 1024;
  }
  return (long long)a.sharedSizeBytes + 16;
}

}  // namespace
}  // namespace spmx

using namespace spmx;

extern "C" int spmx_round_postprocess(spmx_handle_t h) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  RoundTables* t = rtab(h);
  if (!t) return SPMX_SUCCESS;
  dfree(t->rb_row);
  dfree(t->cta_round);
  dfree(t->packed);
  dfree(t->val);
  dfree(t->row16);
  dfree(t->rbase);
  dfree(t->roff);
  delete t;
  h->round = nullptr;
  return SPMX_SUCCESS;
}

extern "C" int spmx_round_preprocess(spmx_handle_t h, int rb_rows) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  if (!h->has_csr || (!h->val && h->nnz > 0))
    return set_error(SPMX_ERR_NOT_READY, "round SpMV needs the CSR input with values");
  if (rb_rows < 0) return set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: rb_rows must be >= 0");
  constexpr int NW = kRoundNW, E = kRoundE;
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  const long long fixed = (long long)round_smem_fixed() + round_static_smem();
  long long rcap = ((long long)optin - fixed) / 4;
  rcap = std::min<long long>(rcap & ~3LL, 65532);
  if (rb_rows > 0) rcap = std::min<long long>(rcap, std::max(4, (rb_rows + 3) & ~3));
  if (rcap < 4) return set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: no shared memory left for y");
  spmx_round_postprocess(h);
  const int m = h->m, n = h->n, nnz = h->nnz;
  cudaStream_t st = h->stream;
  std::vector<int> rp((size_t)m + 1, 0);
  if (m > 0 &&
      cudaMemcpyAsync(rp.data(), h->rowptr, 4 * ((size_t)m + 1), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return set_error(SPMX_ERR_CUDA, "round SpMV: row pointer copy");
  cudaStreamSynchronize(st);
  // row blocks: one wave of 2-CTA clusters when the rows fit, about equal
  // nonzero counts, boundaries on multiples of 4, at most rcap rows each
  const long long need = std::max<long long>(1, (m + rcap - 1) / rcap);
  int nrb = (int)std::max<long long>(need, std::min<long long>(h->num_sms / kRoundCS, std::max(1, m / 4)));
  nrb = std::max(1, nrb);
  const int cbits = bits_for((long long)std::max(n, 1));
  const int bbits = bits_for((long long)nrb + 1);
  if (cbits + bbits > 32)
    return set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: row blocks x columns exceed a 32-bit sort key");
  std::vector<int> rbr((size_t)nrb + 1, 0);
  rbr[nrb] = m;
  for (int k = 1; k < nrb; ++k) {
    const long long want_nz = (long long)nnz * k / nrb;
    long long r = std::lower_bound(rp.begin(), rp.end(), (int)want_nz) - rp.begin();
    r = (r + 2) & ~3LL;
    const long long lo = std::max<long long>(rbr[k - 1], (long long)m - (long long)(nrb - k) * rcap);
    const long long hi = std::min<long long>((long long)rbr[k - 1] + rcap, m);
    r = std::max(r, (lo + 3) & ~3LL);
    r = std::min(r, hi & ~3LL);
    r = std::max<long long>(r, rbr[k - 1]);
    rbr[k] = (int)r;
  }
  int rmax = 4;
  for (int k = 0; k < nrb; ++k) rmax = std::max(rmax, rbr[k + 1] - rbr[k]);
  if (rmax > rcap) return set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: row blocks do not fit shared memory");
  rmax = (rmax + 3) & ~3;
  // warp row splits inside each row block (about equal nonzeros)
  std::vector<int> wsp((size_t)nrb * (NW + 1), 0);
  for (int k = 0; k < nrb; ++k) {
    const int a = rbr[k], b = rbr[k + 1];
    const long long z0 = rp[a], z1 = rp[b];
    for (int w = 0; w <= NW; ++w) {
      int r;
      if (w == 0) r = a;
      else if (w == NW) r = b;
      else
        r = (int)(std::lower_bound(rp.begin() + a, rp.begin() + b, (int)(z0 + (z1 - z0) * w / NW)) - rp.begin());
      wsp[(size_t)k * (NW + 1) + w] = std::max(r - a, w ? wsp[(size_t)k * (NW + 1) + w - 1] : 0);
    }
  }
  RoundTables* t = new RoundTables();
  h->round = t;
  t->nrb = nrb;
  t->grid = nrb * kRoundCS;
  t->rmax = rmax;
  t->smem = round_smem_fixed() + 4 * (size_t)rmax;
  round_set_smem<false>(t->smem);
  round_set_smem<true>(t->smem);

  const size_t b4 = 4 * (size_t)std::max(nnz, 1);
  unsigned *k0 = nullptr, *k1 = nullptr, *a0 = nullptr, *a1 = nullptr, *v0 = nullptr, *v1 = nullptr;
  unsigned *q0 = nullptr, *q1 = nullptr;
  int *hist = nullptr, *hoff = nullptr, *d_wsp = nullptr, *flags = nullptr, *d_bounds = nullptr;
  const size_t hn = radix_hist_ints(std::max(nnz, 1));
  int rc = SPMX_SUCCESS;
  rc = rc ? rc : dalloc((void**)&k0, b4, "round keys");
  rc = rc ? rc : dalloc((void**)&k1, b4, "round keys alt");
  rc = rc ? rc : dalloc((void**)&a0, b4, "round rows");
  rc = rc ? rc : dalloc((void**)&a1, b4, "round rows alt");
  rc = rc ? rc : dalloc((void**)&v0, b4, "round values");
  rc = rc ? rc : dalloc((void**)&v1, b4, "round values alt");
  rc = rc ? rc : dalloc((void**)&q0, b4, "round row keys");
  rc = rc ? rc : dalloc((void**)&q1, b4, "round row keys alt");
  rc = rc ? rc : dalloc((void**)&hist, 4 * hn, "round hist");
  rc = rc ? rc : dalloc((void**)&hoff, 4 * hn, "round hist off");
  rc = rc ? rc : dalloc((void**)&d_wsp, 4 * wsp.size(), "round warp splits");
  rc = rc ? rc : dalloc((void**)&flags, 4 * sizeof(int), "round flags");
  rc = rc ? rc : dalloc((void**)&d_bounds, 4 * ((size_t)nrb + 1), "round block bounds");
  rc = rc ? rc : dalloc((void**)&t->rb_row, 4 * ((size_t)nrb + 1), "round row blocks");
  std::vector<int> bounds((size_t)nrb + 1, 0);
  unsigned *skey = nullptr, *slrow = nullptr, *sval = nullptr;
  if (!rc) {
    cudaMemcpyAsync(t->rb_row, rbr.data(), 4 * ((size_t)nrb + 1), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_wsp, wsp.data(), 4 * wsp.size(), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(flags, 0, 4 * sizeof(int), st);
  }
  if (!rc && nnz > 0) {
    note_launch();
    round_keys_kernel<<<(unsigned)(((long long)m * 32 + 255) / 256), 256, 0, st>>>(
        m, n, h->rowptr, h->col, h->val, t->rb_row, nrb, cbits, k0, a0, v0, flags);
    RadixBuffers rbuf{k0, k1, a0, a1, v0, v1, hist, hoff, false};
    if (radix_sort_pairs(rbuf, nnz, cbits + bbits, h->ls, h->d_err, st))
      rc = set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: sort capacity");
    if (!rc) {
      skey = rbuf.result_in_alt ? k1 : k0;
      slrow = rbuf.result_in_alt ? a1 : a0;
      sval = rbuf.result_in_alt ? v1 : v0;
      note_launch();
      round_bounds_kernel<<<(nrb + 1 + 255) / 256, 256, 0, st>>>(nnz, skey, nrb, cbits, d_bounds);
      if (cudaMemcpyAsync(bounds.data(), d_bounds, 4 * ((size_t)nrb + 1), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess)
        rc = set_error(SPMX_ERR_CUDA, "round SpMV: block bounds");
    }
  }
  cudaError_t se = cudaStreamSynchronize(st);
  if (!rc && se != cudaSuccess) rc = set_error(SPMX_ERR_CUDA, std::string("round SpMV: ") + cudaGetErrorString(se));
  // rounds (host): each row block's sorted nonzeros split in two halves of
  // whole rounds, one per CTA of the cluster, each cut into rounds of E
  std::vector<int> rstart, rlen, rrb, cta((size_t)t->grid + 1, 0);
  if (!rc) {
    for (int k = 0; k < nrb; ++k) {
      const int s = bounds[k], e = bounds[k + 1];
      const long long cnt = e - s;
      const long long nr = (cnt + E - 1) / E;
      const int mid = s + (int)std::min<long long>(cnt, ((nr + 1) / 2) * E);
      const int part[3] = {s, mid, e};
      for (int c = 0; c < kRoundCS; ++c) {
        cta[(size_t)k * kRoundCS + c] = (int)rstart.size();
        for (int p = part[c]; p < part[c + 1]; p += E) {
          rstart.push_back(p);
          rlen.push_back(std::min(E, part[c + 1] - p));
          rrb.push_back(k);
        }
      }
    }
    cta[(size_t)t->grid] = (int)rstart.size();
    if (rstart.size() >= 65536) rc = set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: too many rounds");
  }
  const int nrounds = (int)rstart.size();
  t->nrounds = nrounds;
  int *d_rstart = nullptr, *d_rlen = nullptr, *d_rrb = nullptr;
  const size_t qn = (size_t)std::max(nrounds, 1);
  rc = rc ? rc : dalloc((void**)&t->cta_round, 4 * cta.size(), "round CTA runs");
  rc = rc ? rc : dalloc((void**)&t->packed, 4 * qn * E, "round stream words");
  rc = rc ? rc : dalloc((void**)&t->val, 4 * qn * E, "round values");
  rc = rc ? rc : dalloc((void**)&t->row16, 2 * qn * E, "round rows");
  rc = rc ? rc : dalloc((void**)&t->rbase, 4 * qn, "round first columns");
  rc = rc ? rc : dalloc((void**)&t->roff, 4 * qn * (NW + 1), "round warp offsets");
  rc = rc ? rc : dalloc((void**)&d_rstart, 4 * qn, "round starts");
  rc = rc ? rc : dalloc((void**)&d_rlen, 4 * qn, "round lengths");
  rc = rc ? rc : dalloc((void**)&d_rrb, 4 * qn, "round blocks");
  if (!rc) {
    cudaMemcpyAsync(t->cta_round, cta.data(), 4 * cta.size(), cudaMemcpyHostToDevice, st);
    if (nrounds > 0) {
      cudaMemcpyAsync(d_rstart, rstart.data(), 4 * (size_t)nrounds, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(d_rlen, rlen.data(), 4 * (size_t)nrounds, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(d_rrb, rrb.data(), 4 * (size_t)nrounds, cudaMemcpyHostToDevice, st);
      const unsigned cmask = (unsigned)((1ULL << cbits) - 1);
      const int nvalid = bounds[nrb];
      note_launch();
      round_key2_kernel<<<nrounds, 256, 0, st>>>(d_rstart, d_rlen, skey, slrow, cmask, q0, a1 == slrow ? a0 : a1,
                                                 t->rbase, flags);
      // second stable sort: by (round, local row), payload the column-order position
      unsigned* pos_in = a1 == slrow ? a0 : a1;
      unsigned* pos_alt = k1 == skey ? k0 : k1;
      RadixBuffers r2{q0, q1, pos_in, pos_alt, nullptr, nullptr, hist, hoff, false};
      if (radix_sort_pairs(r2, nvalid, 16 + bits_for((long long)nrounds), h->ls, h->d_err, st))
        rc = set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: sort capacity");
      if (!rc) {
        const unsigned* key2 = r2.result_in_alt ? q1 : q0;
        const unsigned* pos2 = r2.result_in_alt ? pos_alt : pos_in;
        note_launch();
        round_layout_kernel<<<nrounds, 256, 0, st>>>(d_rstart, d_rlen, d_rrb, d_wsp, skey, sval, cmask, key2, pos2,
                                                    t->rbase, t->packed, t->val, t->row16, t->roff);
      }
    }
    int hflags[4] = {0, 0, 0, 0};
    if (cudaMemcpyAsync(hflags, flags, sizeof(hflags), cudaMemcpyDeviceToHost, st) != cudaSuccess)
      rc = rc ? rc : set_error(SPMX_ERR_CUDA, "round SpMV: flags");
    se = cudaStreamSynchronize(st);
    if (!rc && se != cudaSuccess) rc = set_error(SPMX_ERR_CUDA, std::string("round SpMV: ") + cudaGetErrorString(se));
    if (!rc && (hflags[0] & 1)) rc = set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: column index out of range");
    if (!rc && (hflags[0] & 2))
      rc = set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: a round spans too many columns (matrix too sparse)");
  }
  dfree(k0); dfree(k1); dfree(a0); dfree(a1); dfree(v0); dfree(v1); dfree(q0); dfree(q1);
  dfree(hist); dfree(hoff); dfree(d_wsp); dfree(flags); dfree(d_bounds);
  dfree(d_rstart); dfree(d_rlen); dfree(d_rrb);
  if (rc) {
    spmx_round_postprocess(h);
    return rc;
  }
  return SPMX_SUCCESS;
}

template <bool GATED>
static cudaError_t round_launch(spmx_handle_t h, RoundTables* t, float alpha, float* y, const unsigned* bits) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(t->grid);
  cfg.blockDim = dim3(kRoundNW * 32);
  cfg.dynamicSmemBytes = t->smem;
  cfg.stream = h->stream;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = kRoundCS;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 2;
  return cudaLaunchKernelEx(&cfg, round_spmv_kernel<GATED>, (const int*)t->rb_row, (const int*)t->cta_round,
                            (const unsigned*)t->packed, (const float*)t->val, (const unsigned short*)t->row16,
                            (const int*)t->rbase, (const int*)t->roff, (const float*)h->x_dense, bits, alpha, y,
                            h->d_err);
}

int round_spmv_impl(spmx_handle_t h, float alpha, float* y, bool gated) {
  RoundTables* t = rtab(h);
  if (!t) return set_error(SPMX_ERR_NOT_READY, "call spmx_round_preprocess first");
  if (!h->x_dense) return set_error(SPMX_VEC_FORMAT_ERR, "round SpMV needs the dense x");
  if (gated && !h->bitvec) return set_error(SPMX_VEC_FORMAT_ERR, "round SpMSpV needs the bitarray");
  if (!y && h->m > 0) return set_error(SPMX_ERR_INVALID_VALUE, "y is NULL");
  if (h->m == 0) return SPMX_SUCCESS;
  note_launch();
  const cudaError_t e = gated ? round_launch<true>(h, t, alpha, y, (const unsigned*)h->bitvec)
                              : round_launch<false>(h, t, alpha, y, nullptr);
  if (e != cudaSuccess) return set_error(SPMX_ERR_CUDA, std::string("round spmv: ") + cudaGetErrorString(e));
  return SPMX_SUCCESS;
}

extern "C" int spmx_round_info(spmx_handle_t h, int* info) {
  if (!h || !info) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle or info");
  RoundTables* t = rtab(h);
  if (!t) return set_error(SPMX_ERR_NOT_READY, "call spmx_round_preprocess first");
  info[0] = t->nrb;
  info[1] = kRoundCS;
  info[2] = t->nrounds;
  info[3] = kRoundE;
  info[4] = kRoundNW;
  info[5] = t->rmax;
  info[6] = (int)t->smem;
  info[7] = t->grid;
  return SPMX_SUCCESS;
}

extern "C" int spmx_roundspmv(spmx_handle_t h, float alpha, float* d_y) {
  SPMX_CHECK_HANDLE(h);
  return round_spmv_impl(h, alpha, d_y, false);
}

extern "C" int spmx_roundspmspv(spmx_handle_t h, float alpha, float* d_y) {
  SPMX_CHECK_HANDLE(h);
  return round_spmv_impl(h, alpha, d_y, true);
}
