// Round SpMV / bitmap-gated SpMSpV (y = alpha * A * x): a fourth
// load-balanced back-end beside Hola, CSR5 and the tiled SpMV (spmv_type 3;
// no reference counterpart).
//
// Why: a row-ordered SpMV gathers x one cache line per nonzero (about one
// line per cycle per SM on B200), and the tiled back-end, which stages x
// windows in shared memory, pays a producer/consumer handshake per (row
// block, x window) tile.  Here the nonzeros of a row block are streamed in
// COLUMN order, so the 32 lanes of a warp gather x from a few neighbouring
// cache lines, and the accumulation into y needs neither atomics nor a
// reduction pass:
//
//   - rows are cut into row blocks; a row block is processed by a cluster of
//     2 CTAs, each taking one half (in column order) of the block's
//     nonzeros, sorted by (column, row) and cut into rounds of E = 4096;
//   - every row owns as many shared-memory accumulators ("slots") as it has
//     nonzeros in any single round; the k-th nonzero of a row inside a round
//     (column order) adds into the row's k-th slot.  Within a round every
//     nonzero therefore has its own slot, so each lane adds v * x[c] into
//     its slot with a plain read-modify-write, and one CTA barrier per round
//     separates the rounds.  A row of a few nonzeros has one slot; a hub row
//     has one per nonzero it has in its densest round;
//   - each of the 32 warps takes 128 consecutive nonzeros of a round (16-byte
//     loads of the stream, interleaved so that consecutive lanes hold
//     consecutive nonzeros); the gathers of round k + 1 are issued before the
//     additions of round k, so their latency overlaps the round's barrier,
//     and the stream is loaded two rounds ahead;
//   - at the end each CTA sums every row's slots in slot order, and the 2
//     CTAs of a cluster add their row sums in rank order through distributed
//     shared memory; each row is stored once.  Every addition has a fixed
//     order: the result is deterministic.
//
// Stream per nonzero: a 32-bit word (slot << 16 | column offset from the
// first column of its 128-nonzero chunk) and the value: 8 bytes, as CSR, plus
// one chunk base column per 128 nonzeros.
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

constexpr int kRoundE = 4096;     // nonzeros per round
constexpr int kRoundChunk = 128;  // nonzeros per chunk (one base column each)
constexpr int kRoundNW = 32;      // warps per CTA
constexpr int kRoundCS = 2;       // CTAs per cluster (per row block)
constexpr int kRoundCPW = kRoundE / kRoundChunk / kRoundNW;  // chunks per warp per round
constexpr int kRoundDummy = 32;   // padding slots after the real ones (one per lane)
static_assert(kRoundCPW >= 1, "round geometry");

// the per-CTA round runs and row-block bounds of a launch of at most
// kRoundParamCtas CTAs, passed by value so that a CTA reads them without a
// memory round trip (use = 0: read them from the device arrays instead)
constexpr int kRoundParamCtas = 296;
struct RoundGeom {
  int use;
  int cta_round[kRoundParamCtas + 1];
  int rb_row[kRoundParamCtas + 1];
};

struct RoundTables {
  int nrb = 0, grid = 0, rmax = 0, nrounds = 0, nslots = 0;
  int parts = kRoundCS;           // CTAs per row block: one, one cluster, or two (then psum / pcnt)
  bool inplace = false;           // row sums folded into each row's first slot
  float* psum = nullptr;          // parts > 2: each cluster's row sums, [parts / 2][m]
  unsigned* pcnt = nullptr;       // parts > 2: arrivals per (row block, row slice)
  RoundGeom geom = {};
  size_t smem = 0;
  int* rb_row = nullptr;          // nrb + 1 row block boundaries
  int* cta_round = nullptr;       // grid + 1: rounds of CTA c are [cta_round[c], cta_round[c + 1])
  unsigned* packed = nullptr;     // nrounds * E stream words (chunk-interleaved)
  float* val = nullptr;           // nrounds * E values (same order)
  int* cbase = nullptr;           // nrounds * E / 128 chunk base columns
  int* vbg = nullptr;             // m + 1 slot prefix over all rows
};

static RoundTables* rtab(spmx_handle_t h) { return reinterpret_cast<RoundTables*>(h->round); }

namespace {

// shared memory: nslots accumulators (rounded to 4), then (unless the row
// sums are folded into the slots) rmax row sums
size_t round_smem(int nslots, int rmax, bool inplace) {
  return 4 * (size_t)(((nslots + 3) & ~3) + (inplace ? 0 : rmax));
}

// The slot sums (in slot order) of the rows [0, rows) of a row block that
// starts at row0, a multiple of 4: a thread takes groups of 4 consecutive
// rows, one 16-byte load of their slot bounds plus the next row's, VG groups
// per pass with their loads issued together; then the ragged end one row at a
// time.  store4(r, t) receives rows r .. r + 3, store1(r, v) one row.
template <class Store4, class Store1>
__device__ __forceinline__ void round_fold4(int rows, int row0, const int* __restrict__ vbg, int base0,
                                            const float* ys, Store4 store4, Store1 store1) {
  constexpr int VG = 4;
  const int full = rows & ~3;
  for (int rb = 0; rb < full; rb += 4 * VG * (int)blockDim.x) {
    int4 lo[VG];
    int hi[VG];
#pragma unroll
    for (int j = 0; j < VG; ++j) {
      const int r = rb + 4 * (j * (int)blockDim.x + (int)threadIdx.x);
      lo[j] = r < full ? __ldg(reinterpret_cast<const int4*>(vbg + row0 + r)) : make_int4(0, 0, 0, 0);
      hi[j] = r < full ? __ldg(vbg + row0 + r + 4) : 0;
    }
#pragma unroll
    for (int j = 0; j < VG; ++j) {
      const int r = rb + 4 * (j * (int)blockDim.x + (int)threadIdx.x);
      if (r >= full) continue;
      const int b[5] = {lo[j].x - base0, lo[j].y - base0, lo[j].z - base0, lo[j].w - base0, hi[j] - base0};
      float t[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float acc = 0.f;
        for (int s = b[q]; s < b[q + 1]; ++s) acc += ys[s];
        t[q] = acc;
      }
      store4(r, t);
    }
  }
  for (int r = full + (int)threadIdx.x; r < rows; r += blockDim.x) {
    float acc = 0.f;
    for (int s = __ldg(vbg + row0 + r) - base0; s < __ldg(vbg + row0 + r + 1) - base0; ++s) acc += ys[s];
    store1(r, acc);
  }
}

// parts CTAs per row block: one CTA, whose row sums are y (no cluster); or
// clusters of 2, with parts = 4 two of them, in which case each cluster adds
// its two CTAs' row sums and the two clusters meet in psum: the second to
// arrive at a row slice writes y (no waiting, a fixed order of addition).
template <bool GATED, bool INPLACE>
__global__ void __launch_bounds__(kRoundNW * 32, 1)
round_spmv_kernel(const __grid_constant__ RoundGeom geom, int nslots, int parts, const int* __restrict__ rb_row,
                  const int* __restrict__ cta_round,
                  const uint4* __restrict__ packed, const float4* __restrict__ val,
                  const int* __restrict__ cbase, const int* __restrict__ vbg, const float* __restrict__ x,
                  const unsigned* __restrict__ xbits, float alpha, float* __restrict__ y, int m,
                  float* __restrict__ psum, unsigned* __restrict__ pcnt) {
  constexpr int E = kRoundE, CPW = kRoundCPW;
  extern __shared__ __align__(16) float ys[];
  float* F = ys + ((nslots + 3) & ~3);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rb = blockIdx.x / parts;
  const int row0 = geom.use ? geom.rb_row[rb] : __ldg(rb_row + rb);
  const int rows = (geom.use ? geom.rb_row[rb + 1] : __ldg(rb_row + rb + 1)) - row0;
  const int k0 = geom.use ? geom.cta_round[blockIdx.x] : __ldg(cta_round + blockIdx.x);
  const int k1 = geom.use ? geom.cta_round[blockIdx.x + 1] : __ldg(cta_round + blockIdx.x + 1);
  for (int r = threadIdx.x; r < nslots; r += blockDim.x) ys[r] = 0.f;
  // the row block's slot prefix is read by the epilogue: bring it into L2 now
  if (threadIdx.x == 0 && rows > 0) {
    const size_t a0 = ((size_t)(vbg + row0)) & ~(size_t)15;
    const size_t a1 = ((size_t)(vbg + row0 + rows + 1) + 15) & ~(size_t)15;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a0), "r"((unsigned)(a1 - a0)) : "memory");
  }
  // two register sets, used alternately: a round's stream words, values,
  // chunk bases and gathered x
  uint4 pa[CPW], pb[CPW];
  float4 va[CPW], vb[CPW];
  int ba[CPW], bb[CPW];
  float xa[CPW][4], xb[CPW][4];
  auto load = [&](int q, uint4 (&p)[CPW], float4 (&v)[CPW], int (&b)[CPW]) {
#pragma unroll
    for (int u = 0; u < CPW; ++u) {
      const size_t c = (size_t)q * (E / kRoundChunk) + warp * CPW + u;
      p[u] = __ldcs(packed + c * 32 + lane);
      v[u] = __ldcs(val + c * 32 + lane);
      b[u] = __ldg(cbase + c);
    }
  };
  auto gather = [&](const uint4 (&p)[CPW], const int (&b)[CPW], float (&xv)[CPW][4]) {
#pragma unroll
    for (int u = 0; u < CPW; ++u) {
      const unsigned w[4] = {p[u].x, p[u].y, p[u].z, p[u].w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = b[u] + (int)(w[j] & 0xffffu);
        float xx = __ldg(x + c);
        if (GATED && !((__ldg(xbits + (c >> 5)) >> (c & 31)) & 1u)) xx = 0.f;
        xv[u][j] = xx;
      }
    }
  };
  // the stream does not depend on the grid this one is launched after
  if (k0 < k1) load(k0, pa, va, ba);
  if (k0 + 1 < k1) load(k0 + 1, pb, vb, bb);
  // launched as a programmatic dependent of the grid that writes x: nothing
  // above touches x or y
  asm volatile("griddepcontrol.wait;" ::: "memory");
  // (no griddepcontrol.launch_dependents here: with it the kernel took 48.0
  // instead of 46.1 us on the 1M-row Zipf matrix, followed by no dependent)
  if (k0 < k1) gather(pa, ba, xa);
  __syncthreads();
  // one round: issue the next round's gathers, add this round into its
  // slots, load the stream two rounds ahead into this round's registers
  auto step = [&](int k, uint4 (&pc)[CPW], float4 (&vc)[CPW], int (&bc)[CPW], float (&xc)[CPW][4],
                  const uint4 (&pn)[CPW], const int (&bn)[CPW], float (&xn)[CPW][4]) {
    if (k + 1 < k1) gather(pn, bn, xn);
#pragma unroll
    for (int u = 0; u < CPW; ++u) {
      const unsigned w[4] = {pc[u].x, pc[u].y, pc[u].z, pc[u].w};
      const float vv[4] = {vc[u].x, vc[u].y, vc[u].z, vc[u].w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int s = (int)(w[j] >> 16);
        ys[s] = fmaf(vv[j], xc[u][j], ys[s]);
      }
    }
    if (k + 2 < k1) load(k + 2, pc, vc, bc);
    __syncthreads();
  };
  for (int k = k0; k < k1; k += 2) {
    step(k, pa, va, ba, xa, pb, bb, xb);
    if (k + 1 < k1) step(k + 1, pb, vb, bb, xb, pa, ba, xa);
  }
  // each row's slots, summed in slot order, into F[r] or (INPLACE) into the
  // row's first slot; a row without slots has the sum 0
  const int base0 = __ldg(vbg + row0);
  if (parts == 1) {
    // one CTA per row block: each row's slot sum is y (16-byte stores where
    // y allows them)
    const bool y16 = (((uintptr_t)(y + row0)) & 15u) == 0;
    round_fold4(
        rows, row0, vbg, base0, ys,
        [&](int r, const float (&t)[4]) {
          if (y16) {
            *reinterpret_cast<float4*>(y + row0 + r) = make_float4(alpha * t[0], alpha * t[1], alpha * t[2], alpha * t[3]);
          } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) y[row0 + r + q] = alpha * t[q];
          }
        },
        [&](int r, float v) { y[row0 + r] = alpha * v; });
    return;
  }
  if (!INPLACE && parts == kRoundCS) {
    // one 2-CTA cluster per row block: the slot sums into F, then each CTA
    // adds a slice of the rows (a multiple of 4) from both CTAs' F in rank
    // order, 16 bytes at a time through distributed shared memory
    round_fold4(
        rows, row0, vbg, base0, ys,
        [&](int r, const float (&t)[4]) { *reinterpret_cast<float4*>(F + r) = make_float4(t[0], t[1], t[2], t[3]); },
        [&](int r, float v) { F[r] = v; });
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    const int rank = (int)cl.block_rank();
    const int slice = ((rows + 7) / 8) * 4;
    const int r0 = rank * slice, r1 = min(rows, r0 + slice);
    const float* F0 = cl.map_shared_rank(F, 0);
    const float* F1 = cl.map_shared_rank(F, 1);
    const bool y16 = (((uintptr_t)(y + row0)) & 15u) == 0;
    const int g1 = r0 + ((max(0, r1 - r0)) & ~3);  // the slice's groups of 4 end here
    constexpr int CG = 2;  // groups of 4 rows per thread per pass: their peer reads are issued together
    for (int rc = r0; rc < g1; rc += 4 * CG * (int)blockDim.x) {
      float4 a[CG], c[CG];
#pragma unroll
      for (int j = 0; j < CG; ++j) {
        const int r = rc + 4 * (j * (int)blockDim.x + (int)threadIdx.x);
        a[j] = r < g1 ? *reinterpret_cast<const float4*>(F0 + r) : make_float4(0.f, 0.f, 0.f, 0.f);
        c[j] = r < g1 ? *reinterpret_cast<const float4*>(F1 + r) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int j = 0; j < CG; ++j) {
        const int r = rc + 4 * (j * (int)blockDim.x + (int)threadIdx.x);
        if (r >= g1) continue;
        float t[4] = {0.f, 0.f, 0.f, 0.f};
        t[0] += a[j].x; t[1] += a[j].y; t[2] += a[j].z; t[3] += a[j].w;
        t[0] += c[j].x; t[1] += c[j].y; t[2] += c[j].z; t[3] += c[j].w;
        if (y16) {
          *reinterpret_cast<float4*>(y + row0 + r) =
              make_float4(alpha * t[0], alpha * t[1], alpha * t[2], alpha * t[3]);
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q) y[row0 + r + q] = alpha * t[q];
        }
      }
    }
    for (int r = g1 + (int)threadIdx.x; r < r1; r += blockDim.x) {  // the slice's ragged end
      float acc = 0.f;
      acc += F0[r];
      acc += F1[r];
      y[row0 + r] = alpha * acc;
    }
    cl.sync();  // the peer reads this CTA's F until here
    return;
  }
  constexpr int FU = 8;  // rows per thread per pass: their slot bounds are loaded together
  for (int rb4 = 0; rb4 < rows; rb4 += FU * (int)blockDim.x) {
    int lo[FU], hi[FU];
#pragma unroll
    for (int j = 0; j < FU; ++j) {
      const int r = rb4 + j * (int)blockDim.x + (int)threadIdx.x;
      lo[j] = r < rows ? __ldg(vbg + row0 + r) : 0;
      hi[j] = r < rows ? __ldg(vbg + row0 + r + 1) : 0;
    }
#pragma unroll
    for (int j = 0; j < FU; ++j) {
      const int r = rb4 + j * (int)blockDim.x + (int)threadIdx.x;
      if (r < rows) {
        float acc = 0.f;
        for (int s = lo[j] - base0; s < hi[j] - base0; ++s) acc += ys[s];
        if (!INPLACE) F[r] = acc;
        else if (hi[j] > lo[j]) ys[lo[j] - base0] = acc;  // rows own disjoint slots
      }
    }
  }
  // the cluster's row sums, added in rank order; each CTA takes a slice
  cg::cluster_group cl = cg::this_cluster();
  cl.sync();
  const int rank = (int)cl.block_rank();
  const int slice = (rows + kRoundCS - 1) / kRoundCS;
  const int r0 = rank * slice, r1 = min(rows, r0 + slice);
  const int nclu = parts / kRoundCS;  // clusters per row block
  float* mine = nclu > 1 ? psum + (size_t)((blockIdx.x % parts) / kRoundCS) * m + row0 : nullptr;
  constexpr int CU = 4;  // rows per thread per pass: their peer reads are issued together
  for (int rc = r0; rc < r1; rc += CU * (int)blockDim.x) {
    float acc[CU];
    int at[CU];  // where the row's sum lives: F[r], or its first slot (-1: no slots)
#pragma unroll
    for (int j = 0; j < CU; ++j) {
      const int r = rc + j * (int)blockDim.x + (int)threadIdx.x;
      at[j] = r;
      if (INPLACE && r < r1) {
        const int lo = __ldg(vbg + row0 + r);
        at[j] = __ldg(vbg + row0 + r + 1) > lo ? lo - base0 : -1;
      }
    }
#pragma unroll
    for (int j = 0; j < CU; ++j) {
      const int r = rc + j * (int)blockDim.x + (int)threadIdx.x;
      acc[j] = 0.f;
      if (r < r1 && at[j] >= 0) {
        float* src = INPLACE ? ys + at[j] : F + r;
#pragma unroll
        for (int q = 0; q < kRoundCS; ++q) acc[j] += *cl.map_shared_rank(src, q);
      }
    }
#pragma unroll
    for (int j = 0; j < CU; ++j) {
      const int r = rc + j * (int)blockDim.x + (int)threadIdx.x;
      if (r < r1) {
        if (nclu == 1) y[row0 + r] = alpha * acc[j];
        else mine[r] = acc[j];
      }
    }
  }
  if (nclu > 1) {
    // the last cluster to finish this row slice adds the clusters' sums in
    // cluster order and stores y; its ticket is reset for the next launch
    __shared__ int s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned* t = pcnt + (size_t)rb * kRoundCS + rank;
      s_last = atomicAdd(t, 1u) == (unsigned)(nclu - 1);
      if (s_last) atomicExch(t, 0u);
    }
    __syncthreads();
    if (s_last) {
      __threadfence();
      for (int r = r0 + (int)threadIdx.x; r < r1; r += blockDim.x) {
        float acc = 0.f;
        for (int c = 0; c < nclu; ++c) acc += __ldcg(psum + (size_t)c * m + row0 + r);
        y[row0 + r] = alpha * acc;
      }
    }
  }
  cl.sync();  // peers read this CTA's row sums until here
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

// *out = 1 when some run of up to 128 consecutive sorted entries of one row
// block spans 2^16 columns or more.  The layout's chunks are such runs (they
// start at multiples of 128 from their row block's first entry), so without
// a flag no chunk needs the padded layout.  Valid entries end at bounds[nrb].
__global__ void round_span_kernel(int nnz, const unsigned* __restrict__ skey, int nrb, int cbits,
                                  const int* __restrict__ bounds, int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnz || i >= __ldg(bounds + nrb)) return;
  const unsigned cmask = (1u << cbits) - 1u;
  const unsigned ki = __ldg(skey + i);
  const int b = (int)(ki >> cbits);
  const int j = min(i + 127, __ldg(bounds + b + 1) - 1);
  if ((__ldg(skey + j) & cmask) - (ki & cmask) >= 65536u) *out = 1;
}

// out[t] = first sorted position with key >= (rb << cbits) | (seg << 16),
// t = rb * nseg + seg in [0, nrb * nseg]: where each 2^16-column segment of
// each row block starts (t = nrb * nseg gives the end of the last block)
__global__ void round_seg_bounds_kernel(int nnz, const unsigned* __restrict__ skey, int nrb, int nseg,
                                        int cbits, int* __restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t > (long long)nrb * nseg) return;
  const unsigned rb = (unsigned)(t / nseg), seg = (unsigned)(t % nseg);
  const unsigned want = (rb << cbits) | (seg << 16);
  int lo = 0, hi = nnz;
  while (lo < hi) {
    const int mid = (int)(((long long)lo + hi) >> 1);
    if (__ldg(skey + mid) < want) lo = mid + 1;
    else hi = mid;
  }
  out[t] = lo;
}

// stream position of every sorted nonzero within its CTA's half when each
// 2^16-column segment starts a new 128-entry chunk: half h (real entries
// [half_lo[h], half_lo[h + 1])) places segment j at padded offset
// pad_off[h * nseg + j]; its first real entry is seg_real[h * nseg + j]
__global__ void round_ppos_kernel(int nvalid, const unsigned* __restrict__ skey, unsigned cmask, int nhalf,
                                  const int* __restrict__ half_lo, int nseg, const int* __restrict__ seg_real,
                                  const int* __restrict__ pad_off, int* __restrict__ ppos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nvalid) return;
  int lo = 0, hi = nhalf;  // the last half with half_lo <= i
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(half_lo + mid) <= i) lo = mid;
    else hi = mid;
  }
  const int j = (int)((__ldg(skey + i) & cmask) >> 16);
  const long long hj = (long long)lo * nseg + j;
  ppos[i] = __ldg(pad_off + hj) + (i - __ldg(seg_real + hj));
}

// one CTA per round: the second sort's keys (round << 16 | local row, stable
// over the round's column order) and the column-order positions
__global__ void round_key2_kernel(const int* __restrict__ rstart, const int* __restrict__ rlen,
                                  const unsigned* __restrict__ slrow, unsigned* __restrict__ key2,
                                  unsigned* __restrict__ pos2) {
  const int q = blockIdx.x;
  const int s = __ldg(rstart + q), len = __ldg(rlen + q);
  for (int i = threadIdx.x; i < len; i += blockDim.x) {
    key2[s + i] = ((unsigned)q << 16) | __ldg(slrow + s + i);
    pos2[s + i] = (unsigned)i;
  }
}

// one CTA per round: the occurrence of every nonzero among its row's
// nonzeros in the round (column order), stored by column-order position, and
// the row's slot count (the largest occurrence + 1 over all rounds)
__global__ void round_occurrence_kernel(const int* __restrict__ rstart, const int* __restrict__ rlen,
                                        const int* __restrict__ rrb, const int* __restrict__ rb_row,
                                        const unsigned* __restrict__ key2, const unsigned* __restrict__ pos2,
                                        int* __restrict__ occ, int* __restrict__ slots_per_row) {
  const int q = blockIdx.x;
  const int s = __ldg(rstart + q), len = __ldg(rlen + q);
  const int row0 = __ldg(rb_row + __ldg(rrb + q));
  for (int t = threadIdx.x; t < len; t += blockDim.x) {
    const unsigned k = __ldg(key2 + s + t);
    int lo = 0, hi = t;  // first entry of the round with this key
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(key2 + s + mid) < k) lo = mid + 1;
      else hi = mid;
    }
    const int o = t - lo;
    occ[s + (int)__ldg(pos2 + s + t)] = o;
    atomicMax(slots_per_row + row0 + (int)(k & 0xffffu), o + 1);
  }
}

// storage position of chunk-local position p: a lane's 16-byte word holds
// entries l, l + 32, l + 64, l + 96 of the chunk
__device__ __forceinline__ int round_vperm(int p) {
  const int blk = p >> 7, c = (p >> 5) & 3, l = p & 31;
  return (blk << 7) + 4 * l + c;
}

// one CTA per round: stream words (slot << 16 | column offset from the
// chunk's first column), values and chunk bases.  Every position starts as
// padding (a lane's own dummy slot, the chunk's base column, value 0); real
// entry t of the round then goes to position t, or, with ppos, to its padded
// position ppos[i] - rpad0[q] (chunks then never cross a 2^16-column segment).
// A chunk's real entries are contiguous from its first position, which holds
// its base column.  An offset of 2^16 columns or more sets flags bit 1.
__global__ void __launch_bounds__(256)
round_layout_kernel(const int* __restrict__ rstart, const int* __restrict__ rlen, const int* __restrict__ rpad0,
                    const int* __restrict__ rrb, const int* __restrict__ rb_row, const int* __restrict__ vbg,
                    const unsigned* __restrict__ skey, const unsigned* __restrict__ slrow,
                    const unsigned* __restrict__ sval, unsigned cmask, const int* __restrict__ occ,
                    const int* __restrict__ ppos, int dummy, unsigned* __restrict__ packed,
                    float* __restrict__ val, int* __restrict__ cbase, int* __restrict__ flags) {
  constexpr int E = kRoundE;
  const int q = blockIdx.x;
  const int s = __ldg(rstart + q), len = __ldg(rlen + q);
  const int p0 = ppos ? __ldg(rpad0 + q) : 0;
  const int row0 = __ldg(rb_row + __ldg(rrb + q));
  const int vb0 = __ldg(vbg + row0);
  const size_t o = (size_t)q * E;
  for (int p = threadIdx.x; p < E; p += blockDim.x) {
    packed[o + round_vperm(p)] = (unsigned)(dummy + (p & 31)) << 16;
    val[o + round_vperm(p)] = 0.f;
    if ((p & (kRoundChunk - 1)) == 0) cbase[o / kRoundChunk + p / kRoundChunk] = 0;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < len; t += blockDim.x) {
    const int i = s + t;
    const int pp = ppos ? __ldg(ppos + i) - p0 : t;
    if ((unsigned)pp >= (unsigned)E) {
      atomicOr(flags, 4);
      continue;
    }
    const int first = pp & ~(kRoundChunk - 1);
    const unsigned cb = __ldg(skey + i - (pp - first)) & cmask;
    const unsigned c = __ldg(skey + i) & cmask;
    const int slot = __ldg(vbg + row0 + (int)__ldg(slrow + i)) - vb0 + __ldg(occ + i);
    if (c - cb >= 65536u) atomicOr(flags, 2);
    packed[o + round_vperm(pp)] = ((unsigned)slot << 16) | ((c - cb) & 0xffffu);
    val[o + round_vperm(pp)] = __uint_as_float(__ldg(sval + i));
    if (pp == first) cbase[o / kRoundChunk + pp / kRoundChunk] = (int)cb;
  }
}

// slots of each row block: out[b] = vbg[rb_row[b + 1]] - vbg[rb_row[b]]
__global__ void round_block_slots_kernel(int nrb, const int* __restrict__ rb_row, const int* __restrict__ vbg,
                                         int* __restrict__ out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nrb) out[b] = __ldg(vbg + __ldg(rb_row + b + 1)) - __ldg(vbg + __ldg(rb_row + b));
}

int bits_for(long long v) {  // bits to hold values in [0, v)
  int b = 1;
  while (b < 62 && (1LL << b) < v) ++b;
  return b;
}

template <bool GATED, bool INPLACE>
static void round_set_smem(size_t smem) {
  kernel_smem_limit((const void*)round_spmv_kernel<GATED, INPLACE>, smem);
}

static long long round_static_smem() {
  cudaFuncAttributes a = {};
  if (cudaFuncGetAttributes(&a, round_spmv_kernel<true, false>) != cudaSuccess) {
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
  dfree(t->cbase);
  dfree(t->vbg);
  dfree(t->psum);
  dfree(t->pcnt);
  delete t;
  h->round = nullptr;
  return SPMX_SUCCESS;
}

// Temporaries carved from one device allocation: plan() the total (each piece
// rounded up to 256 bytes), alloc() once, take() the pieces in order,
// release() once.
struct Arena {
  char* base = nullptr;
  size_t cap = 0, used = 0;
  void plan(size_t bytes_and_pieces) { cap = bytes_and_pieces + 256 * 32; }
  int alloc(const char* what) { return dalloc((void**)&base, cap, what); }
  template <class T>
  T* take(size_t bytes) {
    const size_t o = (used + 255) & ~(size_t)255;
    used = o + bytes;
    return used <= cap ? reinterpret_cast<T*>(base + o) : nullptr;
  }
  void release() {
    dfree(base);
    base = nullptr;
  }
};

// builds the round format with row blocks of at most rcap rows; *overflow is
// set when a row block needs more accumulator slots than shared memory holds,
// *span when 128 consecutive nonzeros of a row block span 2^16 columns or more
// (then a build with pad = true starts a new chunk at every 2^16-column
// segment, which bounds every chunk's span)
static int round_build(spmx_handle_t h, long long rcap, long long avail, int parts, bool inplace, bool pad,
                       int waves, bool* overflow, bool* span) {
  constexpr int E = kRoundE;
  spmx_round_postprocess(h);
  const int m = h->m, n = h->n, nnz = h->nnz;
  cudaStream_t st = h->stream;
  std::vector<int> rp((size_t)m + 1, 0);
  if (m > 0 &&
      cudaMemcpyAsync(rp.data(), h->rowptr, 4 * ((size_t)m + 1), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return set_error(SPMX_ERR_CUDA, "round SpMV: row pointer copy");
  cudaStreamSynchronize(st);
  // row blocks: one wave of CTAs (times `waves`) when the rows fit,
  // about equal nonzero counts, boundaries on multiples of 4, at most rcap rows
  // each.  Where the row cap makes some blocks take far more nonzeros than
  // others (a power-law matrix: its many short rows fill blocks by rows, so
  // the hub rows crowd into the first blocks), the block count doubles (more
  // waves) until the largest block holds at most 1.5 times the mean, or until
  // its CTAs' share is at most 3/4 of what one SM takes of the whole matrix
  // (then it no longer sets the time).  A doubling that leaves the largest
  // block above 2/3 of its size (a single hub row fills it) is undone: a
  // second wave costs more than the imbalance it removes.
  const long long need = std::max<long long>(1, (m + rcap - 1) / rcap);
  const long long max_blocks = std::max(1, m / 4);
  int nrb = (int)std::max<long long>(need, std::min<long long>((long long)(h->num_sms / parts) * waves, max_blocks));
  nrb = std::max(1, nrb);
  std::vector<int> rbr, prev_rbr;
  long long prev_big = -1;
  for (;;) {
    rbr.assign((size_t)nrb + 1, 0);
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
    long long big = 0;
    for (int k = 0; k < nrb; ++k) big = std::max<long long>(big, (long long)rp[rbr[k + 1]] - rp[rbr[k]]);
    const double mean = (double)nnz / nrb;
    if (prev_big >= 0 && 3 * big > 2 * prev_big) {
      // doubling left the largest block above 2/3 of its size (one hub row
      // fills it): the extra wave would only cost, keep the previous count
      rbr.swap(prev_rbr);
      nrb /= 2;
      break;
    }
    if (nnz == 0 || (double)big <= 1.5 * mean || (double)big / parts <= 0.75 * (double)nnz / h->num_sms ||
        2LL * nrb > max_blocks || nrb >= 16 * (h->num_sms / parts))
      break;
    prev_big = big;
    prev_rbr = rbr;
    nrb *= 2;
  }
  const int cbits = bits_for((long long)std::max(n, 1));
  const int bbits = bits_for((long long)nrb + 1);
  if (cbits + bbits > 32)
    return set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: row blocks x columns exceed a 32-bit sort key");
  int rmax = 4;
  for (int k = 0; k < nrb; ++k) rmax = std::max(rmax, rbr[k + 1] - rbr[k]);
  if (rmax > rcap) return set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: row blocks do not fit shared memory");
  rmax = (rmax + 3) & ~3;
  RoundTables* t = new RoundTables();
  h->round = t;
  t->nrb = nrb;
  t->grid = nrb * parts;
  t->rmax = rmax;
  t->parts = parts;
  t->inplace = inplace;

  const size_t b4 = 4 * (size_t)std::max(nnz, 1);
  unsigned *k0 = nullptr, *k1 = nullptr, *a0 = nullptr, *a1 = nullptr, *v0 = nullptr, *v1 = nullptr;
  unsigned *q0 = nullptr, *q1 = nullptr;
  int *hist = nullptr, *hoff = nullptr, *flags = nullptr, *d_bounds = nullptr, *spr = nullptr;
  const size_t hn = radix_hist_ints(std::max(nnz, 1));
  int rc = SPMX_SUCCESS;
  // the build's temporaries whose sizes are known now, carved from one
  // allocation (one cudaMalloc and one cudaFree per build instead of one per
  // array: the build took 31 ms of host time around 3.7 ms of kernels)
  int *occ = nullptr, *ppos = nullptr, *d_bslots = nullptr, *d_segb = nullptr;
  Arena tmp;
  tmp.plan(8 * b4 + 2 * 4 * hn + 16 + 4 * ((size_t)nrb + 1) + 4 * ((size_t)m + 1) + b4 + 4 * ((size_t)nrb + 1));
  rc = rc ? rc : tmp.alloc("round build scratch");
  if (!rc) {
    k0 = tmp.take<unsigned>(b4); k1 = tmp.take<unsigned>(b4);
    a0 = tmp.take<unsigned>(b4); a1 = tmp.take<unsigned>(b4);
    v0 = tmp.take<unsigned>(b4); v1 = tmp.take<unsigned>(b4);
    q0 = tmp.take<unsigned>(b4); q1 = tmp.take<unsigned>(b4);
    hist = tmp.take<int>(4 * hn); hoff = tmp.take<int>(4 * hn);
    flags = tmp.take<int>(16);
    d_bounds = tmp.take<int>(4 * ((size_t)nrb + 1));
    spr = tmp.take<int>(4 * ((size_t)m + 1));
    occ = tmp.take<int>(b4);
    d_bslots = tmp.take<int>(4 * ((size_t)nrb + 1));
  }
  rc = rc ? rc : dalloc((void**)&t->rb_row, 4 * ((size_t)nrb + 1), "round row blocks");
  rc = rc ? rc : dalloc((void**)&t->vbg, 4 * ((size_t)m + 1), "round slot prefix");
  std::vector<int> bounds((size_t)nrb + 1, 0);
  unsigned *skey = nullptr, *slrow = nullptr, *sval = nullptr;
  if (!rc) {
    cudaMemcpyAsync(t->rb_row, rbr.data(), 4 * ((size_t)nrb + 1), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(flags, 0, 4 * sizeof(int), st);
    cudaMemsetAsync(spr, 0, 4 * ((size_t)m + 1), st);
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
    // a wide column span switches the padded layout on here, so the sort is
    // not repeated (the layout kernel still checks every chunk)
    if (!rc && !pad) {
      int wide = 0;
      note_launch();
      round_span_kernel<<<(unsigned)(((long long)nnz + 255) / 256), 256, 0, st>>>(nnz, skey, nrb, cbits, d_bounds,
                                                                                 flags + 1);
      if (cudaMemcpyAsync(&wide, flags + 1, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        rc = set_error(SPMX_ERR_CUDA, "round SpMV: span check");
      if (!rc && wide) pad = true;
    }
  }
  // with pad: where each 2^16-column segment of each row block starts
  const int nseg = pad ? (int)(((long long)std::max(n, 1) + 65535) / 65536) : 1;
  std::vector<int> segb;
  if (!rc && pad && nnz > 0) {
    const long long nt = (long long)nrb * nseg + 1;
    segb.assign((size_t)nt, 0);
    rc = dalloc((void**)&d_segb, 4 * (size_t)nt, "round segment bounds");
    if (!rc) {
      note_launch();
      round_seg_bounds_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(nnz, skey, nrb, nseg, cbits, d_segb);
      if (cudaMemcpyAsync(segb.data(), d_segb, 4 * (size_t)nt, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        rc = set_error(SPMX_ERR_CUDA, "round SpMV: segment bounds");
    }
  }
  cudaError_t se = cudaStreamSynchronize(st);
  if (!rc && se != cudaSuccess) rc = set_error(SPMX_ERR_CUDA, std::string("round SpMV: ") + cudaGetErrorString(se));
  // rounds (host): each row block's sorted nonzeros split in `parts` runs of
  // whole rounds, one per CTA of the row block, each cut into rounds of E
  // stream positions.  With pad, a half's stream places every segment at a
  // multiple of the chunk length (a segment's last chunk is padded), and the
  // rounds are cut on that padded stream; a round then holds the real entries
  // whose padded positions fall in it, a contiguous run of the sorted order.
  std::vector<int> rstart, rlen, rpad0, rrb, cta((size_t)t->grid + 1, 0);
  std::vector<int> half_lo, seg_real, pad_off;  // per half (pad only)
  if (!rc) {
    for (int k = 0; k < nrb; ++k) {
      const int s = bounds[k], e = bounds[k + 1];
      const long long cnt = e - s;
      const long long nr = (cnt + E - 1) / E;
      // part q takes nr / parts whole rounds, the first nr % parts one more
      std::vector<int> part((size_t)parts + 1, e);
      long long acc_r = 0;
      for (int q = 0; q <= parts; ++q) {
        part[q] = s + (int)std::min<long long>(cnt, acc_r * E);
        if (q < parts) acc_r += nr / parts + (q < nr % parts ? 1 : 0);
      }
      for (int c = 0; c < parts; ++c) {
        cta[(size_t)k * parts + c] = (int)rstart.size();
        const int lo = part[c], hi = part[c + 1];
        if (!pad) {
          for (int p = lo; p < hi; p += E) {
            rstart.push_back(p);
            rlen.push_back(std::min(E, hi - p));
            rpad0.push_back(0);
            rrb.push_back(k);
          }
          continue;
        }
        half_lo.push_back(lo);
        std::vector<long long> off((size_t)nseg + 1, 0);
        std::vector<int> st0((size_t)nseg, lo), cnts((size_t)nseg, 0);
        for (int j = 0; j < nseg; ++j) {
          const int a = std::max(lo, segb[(size_t)k * nseg + j]);
          const int b = std::min(hi, segb[(size_t)k * nseg + j + 1]);
          st0[j] = a;
          cnts[j] = std::max(0, b - a);
          off[j + 1] = off[j] + ((cnts[j] + kRoundChunk - 1) / kRoundChunk) * kRoundChunk;
          seg_real.push_back(a);
          pad_off.push_back((int)off[j]);
        }
        const long long L = off[nseg];
        // the real index at padded position P (a chunk start, or L)
        auto real_at = [&](long long P) -> int {
          if (P >= L) return hi;
          const int j = (int)(std::upper_bound(off.begin(), off.end(), P) - off.begin()) - 1;
          return st0[j] + (int)std::min<long long>(P - off[j], cnts[j]);
        };
        for (long long P = 0; P < L; P += E) {
          const int a = real_at(P), b = real_at(std::min(L, P + E));
          rstart.push_back(a);
          rlen.push_back(b - a);
          rpad0.push_back((int)P);
          rrb.push_back(k);
        }
      }
    }
    cta[(size_t)t->grid] = (int)rstart.size();
    if (rstart.size() >= 65536) rc = set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: too many rounds");
    if (pad && (long long)half_lo.size() * nseg > (1LL << 26))
      rc = set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: too many column segments");
  }
  const int nrounds = (int)rstart.size();
  t->nrounds = nrounds;
  int *d_rstart = nullptr, *d_rlen = nullptr, *d_rrb = nullptr;
  int *d_rpad0 = nullptr, *d_half_lo = nullptr, *d_seg_real = nullptr, *d_pad_off = nullptr;
  const size_t qn = (size_t)std::max(nrounds, 1);
  rc = rc ? rc : dalloc((void**)&t->cta_round, 4 * cta.size(), "round CTA runs");
  rc = rc ? rc : dalloc((void**)&t->packed, 4 * qn * E, "round stream words");
  rc = rc ? rc : dalloc((void**)&t->val, 4 * qn * E, "round values");
  rc = rc ? rc : dalloc((void**)&t->cbase, 4 * qn * (E / kRoundChunk), "round chunk bases");
  // the per-round tables, sized by the round cut: a second carved allocation
  const size_t hs = std::max<size_t>(half_lo.size(), 1), ss = std::max<size_t>(seg_real.size(), 1);
  Arena tmp2;
  tmp2.plan(3 * 4 * qn + (pad ? 4 * qn + 4 * hs + 2 * 4 * ss + b4 : 0));
  rc = rc ? rc : tmp2.alloc("round build tables");
  if (!rc) {
    d_rstart = tmp2.take<int>(4 * qn);
    d_rlen = tmp2.take<int>(4 * qn);
    d_rrb = tmp2.take<int>(4 * qn);
    if (pad) {
      d_rpad0 = tmp2.take<int>(4 * qn);
      d_half_lo = tmp2.take<int>(4 * hs);
      d_seg_real = tmp2.take<int>(4 * ss);
      d_pad_off = tmp2.take<int>(4 * ss);
      ppos = tmp2.take<int>(b4);
    }
  }
  const unsigned cmask = (unsigned)((1ULL << cbits) - 1);
  int nslots_real = 0;
  if (!rc) {
    cudaMemcpyAsync(t->cta_round, cta.data(), 4 * cta.size(), cudaMemcpyHostToDevice, st);
    if (nrounds > 0) {
      cudaMemcpyAsync(d_rstart, rstart.data(), 4 * (size_t)nrounds, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(d_rlen, rlen.data(), 4 * (size_t)nrounds, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(d_rrb, rrb.data(), 4 * (size_t)nrounds, cudaMemcpyHostToDevice, st);
      const int nvalid = bounds[nrb];
      if (pad && nvalid > 0) {
        cudaMemcpyAsync(d_rpad0, rpad0.data(), 4 * (size_t)nrounds, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_half_lo, half_lo.data(), 4 * half_lo.size(), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_seg_real, seg_real.data(), 4 * seg_real.size(), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_pad_off, pad_off.data(), 4 * pad_off.size(), cudaMemcpyHostToDevice, st);
        note_launch();
        round_ppos_kernel<<<(nvalid + 255) / 256, 256, 0, st>>>(nvalid, skey, cmask, (int)half_lo.size(), d_half_lo,
                                                                nseg, d_seg_real, d_pad_off, ppos);
      }
      unsigned* pos_in = a1 == slrow ? a0 : a1;
      unsigned* pos_alt = k1 == skey ? k0 : k1;
      note_launch();
      round_key2_kernel<<<nrounds, 256, 0, st>>>(d_rstart, d_rlen, slrow, q0, pos_in);
      // second stable sort: by (round, local row), payload the column-order position
      RadixBuffers r2{q0, q1, pos_in, pos_alt, nullptr, nullptr, hist, hoff, false};
      if (radix_sort_pairs(r2, nvalid, 16 + bits_for((long long)nrounds), h->ls, h->d_err, st))
        rc = set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: sort capacity");
      if (!rc) {
        const unsigned* key2 = r2.result_in_alt ? q1 : q0;
        const unsigned* pos2 = r2.result_in_alt ? pos_alt : pos_in;
        note_launch();
        round_occurrence_kernel<<<nrounds, 256, 0, st>>>(d_rstart, d_rlen, d_rrb, t->rb_row, key2, pos2, occ, spr);
      }
    }
    // slot prefix over all rows; slots of the largest row block
    if (!rc && m > 0 && launch_scan_exclusive(spr, t->vbg, m, t->vbg + m, h->ls, h->d_err, st))
      rc = set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: scan capacity");
    if (!rc && m == 0) cudaMemsetAsync(t->vbg, 0, 4, st);
    std::vector<int> bslots((size_t)nrb, 0);
    if (!rc) {
      note_launch();
      round_block_slots_kernel<<<(nrb + 255) / 256, 256, 0, st>>>(nrb, t->rb_row, t->vbg, d_bslots);
      cudaMemcpyAsync(bslots.data(), d_bslots, 4 * (size_t)nrb, cudaMemcpyDeviceToHost, st);
      se = cudaStreamSynchronize(st);
      if (se != cudaSuccess) rc = set_error(SPMX_ERR_CUDA, std::string("round SpMV: ") + cudaGetErrorString(se));
    }
    if (!rc) {
      for (int k = 0; k < nrb; ++k) nslots_real = std::max(nslots_real, bslots[k]);
      t->nslots = nslots_real + kRoundDummy;
      t->smem = round_smem(t->nslots, rmax, inplace || parts == 1);
      if (t->nslots >= 65536 || (long long)t->smem > avail) {
        *overflow = true;
        rc = set_error(SPMX_ERR_INVALID_VALUE,
                       "round SpMV: a row block needs more accumulator slots than shared memory holds");
      }
    }
    if (!rc && nrounds > 0) {
      note_launch();
      round_layout_kernel<<<nrounds, 256, 0, st>>>(d_rstart, d_rlen, d_rpad0, d_rrb, t->rb_row, t->vbg, skey,
                                                  slrow, sval, cmask, occ, pad ? ppos : nullptr, nslots_real,
                                                  t->packed, t->val, t->cbase, flags);
    }
    int hflags[4] = {0, 0, 0, 0};
    if (cudaMemcpyAsync(hflags, flags, sizeof(hflags), cudaMemcpyDeviceToHost, st) != cudaSuccess)
      rc = rc ? rc : set_error(SPMX_ERR_CUDA, "round SpMV: flags");
    se = cudaStreamSynchronize(st);
    if (!rc && se != cudaSuccess) rc = set_error(SPMX_ERR_CUDA, std::string("round SpMV: ") + cudaGetErrorString(se));
    if (!rc && (hflags[0] & 1)) rc = set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: column index out of range");
    if (!rc && (hflags[0] & 4)) rc = set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: internal layout error");
    if (!rc && (hflags[0] & 2)) {
      *span = true;
      rc = set_error(SPMX_ERR_INVALID_VALUE,
                     "round SpMV: 128 consecutive nonzeros of a row block span 2^16 columns");
    }
  }
  tmp.release();
  tmp2.release();
  dfree(d_segb);
  if (!rc && parts > kRoundCS) {
    rc = dalloc((void**)&t->psum, 4 * (size_t)(parts / kRoundCS) * (size_t)std::max(m, 1), "round cluster sums");
    rc = rc ? rc : dalloc((void**)&t->pcnt, 4 * (size_t)nrb * kRoundCS, "round cluster tickets");
    if (!rc && cudaMemsetAsync(t->pcnt, 0, 4 * (size_t)nrb * kRoundCS, st) != cudaSuccess)
      rc = set_error(SPMX_ERR_CUDA, "round SpMV: ticket reset");
    if (!rc && cudaStreamSynchronize(st) != cudaSuccess) rc = set_error(SPMX_ERR_CUDA, "round SpMV: ticket reset");
  }
  if (rc) {
    spmx_round_postprocess(h);
    return rc;
  }
  if (inplace) {
    round_set_smem<false, true>(t->smem);
    round_set_smem<true, true>(t->smem);
  } else {
    round_set_smem<false, false>(t->smem);
    round_set_smem<true, false>(t->smem);
  }
  t->geom.use = t->grid <= kRoundParamCtas ? 1 : 0;
  if (t->geom.use) {
    std::copy(cta.begin(), cta.end(), t->geom.cta_round);
    std::copy(rbr.begin(), rbr.end(), t->geom.rb_row);
  }
  return SPMX_SUCCESS;
}

// parts = 1: one CTA per row block (no cluster), its row sums stored as y
// straight from the slots (rows <= avail / 4);
// parts = 2: one 2-CTA cluster per row block, row sums in their own shared
// array (rows <= avail / 8), row blocks halved while the slots overflow;
// parts = 4: two clusters per row block over twice as many rows, the row sums
// folded into the slots (rows <= avail / 4), row blocks shrunk by 15% while
// the slots overflow.  Either way a matrix whose 128 consecutive nonzeros
// (in a row block's column order) span 2^16 columns or more is rebuilt with
// every 2^16-column segment starting a new chunk.
static int round_preprocess(spmx_handle_t h, int rb_rows, int parts) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  if (!h->has_csr || (!h->val && h->nnz > 0))
    return set_error(SPMX_ERR_NOT_READY, "round SpMV needs the CSR input with values");
  if (rb_rows < 0) return set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: rb_rows must be >= 0");
  if (parts != 1 && parts != 2 && parts != 4)
    return set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: parts must be 1, 2 or 4");
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  const long long avail = (long long)optin - round_static_smem();
  const bool inplace = parts > 2;
  // every nonempty row needs a slot (and, unless folded or stored as y, a row sum)
  long long rcap = std::min<long long>((avail / (inplace || parts == 1 ? 4 : 8)) & ~3LL, 65532);
  if (rb_rows > 0) rcap = std::min<long long>(rcap, std::max(4, (rb_rows + 3) & ~3));
  if (rcap < 4) return set_error(SPMX_ERR_INVALID_VALUE, "round SpMV: no shared memory left for y");
  // When the slots of some row block overflow, first take twice as many row
  // blocks (shorter in nonzeros, so fewer slots each; up to 4 times the
  // blocks), then shrink the row cap.
  bool pad = false;
  int waves = 1;
  for (int attempt = 0;; ++attempt) {
    bool overflow = false, span = false;
    const int rc = round_build(h, rcap, avail, parts, inplace, pad, waves, &overflow, &span);
    if (rc == SPMX_SUCCESS) return rc;
    if (span && !pad) {
      pad = true;
      continue;
    }
    if (!overflow || attempt >= (inplace || parts == 1 ? 14 : 8) || rcap <= 64) return rc;
    if (waves < 4) {
      waves *= 2;
      continue;
    }
    rcap = std::max<long long>(64, (inplace || parts == 1 ? rcap * 85 / 100 : rcap / 2) & ~3LL);
  }
}

extern "C" int spmx_round_preprocess(spmx_handle_t h, int rb_rows) { return round_preprocess(h, rb_rows, 1); }

extern "C" int spmx_round_preprocess_parts(spmx_handle_t h, int rb_rows, int parts) {
  return round_preprocess(h, rb_rows, parts);
}

template <bool GATED, bool INPLACE>
static cudaError_t round_launch(spmx_handle_t h, RoundTables* t, float alpha, float* y, const unsigned* bits) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(t->grid);
  cfg.blockDim = dim3(kRoundNW * 32);
  cfg.dynamicSmemBytes = t->smem;
  cfg.stream = h->stream;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = t->parts == 1 ? 1 : kRoundCS;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 2;
  // another handle's build may have set this kernel's limit for its own size
  const cudaError_t e = kernel_smem_limit((const void*)round_spmv_kernel<GATED, INPLACE>, t->smem);
  if (e != cudaSuccess) return e;
  return cudaLaunchKernelEx(&cfg, round_spmv_kernel<GATED, INPLACE>, t->geom, t->nslots, t->parts,
                            (const int*)t->rb_row, (const int*)t->cta_round, (const uint4*)t->packed,
                            (const float4*)t->val, (const int*)t->cbase, (const int*)t->vbg,
                            (const float*)h->x_dense, bits, alpha, y, h->m, t->psum, t->pcnt);
}

int round_spmv_impl(spmx_handle_t h, float alpha, float* y, bool gated) {
  RoundTables* t = rtab(h);
  if (!t) return set_error(SPMX_ERR_NOT_READY, "call spmx_round_preprocess first");
  if (!h->x_dense) return set_error(SPMX_VEC_FORMAT_ERR, "round SpMV needs the dense x");
  if (gated && !h->bitvec) return set_error(SPMX_VEC_FORMAT_ERR, "round SpMSpV needs the bitarray");
  if (!y && h->m > 0) return set_error(SPMX_ERR_INVALID_VALUE, "y is NULL");
  if (h->m == 0) return SPMX_SUCCESS;
  note_launch();
  const unsigned* bits = (const unsigned*)h->bitvec;
  const cudaError_t e = t->inplace ? (gated ? round_launch<true, true>(h, t, alpha, y, bits)
                                            : round_launch<false, true>(h, t, alpha, y, nullptr))
                                   : (gated ? round_launch<true, false>(h, t, alpha, y, bits)
                                            : round_launch<false, false>(h, t, alpha, y, nullptr));
  if (e != cudaSuccess) return set_error(SPMX_ERR_CUDA, std::string("round spmv: ") + cudaGetErrorString(e));
  return SPMX_SUCCESS;
}

extern "C" int spmx_round_info(spmx_handle_t h, int* info) {
  if (!h || !info) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle or info");
  RoundTables* t = rtab(h);
  if (!t) return set_error(SPMX_ERR_NOT_READY, "call spmx_round_preprocess first");
  info[0] = t->nrb;
  info[1] = t->parts;
  info[2] = t->nrounds;
  info[3] = kRoundE;
  info[4] = t->nslots;
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
