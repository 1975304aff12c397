// Tiled SpMV / bitmap-gated SpMSpV (y = alpha * A * x): a third load-balanced
// back-end beside Hola and CSR5 (spmv_type 2; no reference counterpart).
//
// Why: with uniformly random columns every nonzero of a row-ordered SpMV
// gathers x through L1/L2 one cache line at a time.  On B200 the L1 tag stage
// handles about one distinct line per cycle per SM, which caps a 1M-column,
// 16.8M-nonzero SpMV near 68 us (measured with a bare gather loop), about a
// third of HBM bandwidth.  Reading x from shared memory instead costs a few
// bank wavefronts per warp, so this back-end stages x in shared memory:
//
//   - rows are cut into row blocks whose y fits in shared memory (up to about
//     20K rows with the default window), columns into windows of `win`
//     entries of x (8192 by default);
//     a tile is the set of nonzeros of one row block inside one window, in
//     CSR order (sorted by row), cut into stages of at most `chunk` entries;
//   - a row block is processed by a cluster of `cs` CTAs (cs chosen so that
//     the grid is one wave of one CTA per SM); each CTA owns a contiguous run
//     of the block's stages;
//   - in each CTA one producer warp streams every stage (x window, bitmap
//     window, packed (row, column) words, values) into a ring of shared
//     memory buffers with cp.async.bulk, completion tracked by mbarriers;
//   - consumer warps each own a fixed range of the block's rows (equal
//     nonzero counts).  A warp's slice of a stage is cut into 32 contiguous
//     lane ranges, stored lane-interleaved; each lane gathers x from the
//     shared window, sums its runs of equal rows in registers and adds them
//     into the shared y with a plain read-modify-write; a run that crosses
//     into the next lane is joined with shuffles and added once.  No two
//     warps ever touch a row, and a warp updates a row in stage order, so
//     the result is deterministic;
//   - at the end the cluster's partial y vectors are added in CTA-rank order
//     through distributed shared memory and each row is stored once.
//
// HBM traffic per call is the staged copy of the matrix (8 bytes per nonzero
// plus at most 3 padding entries per tile), x once and y once; x windows are
// re-read from L2 once per row block.  Every wait is bounded: a timeout sets
// the device error word and the kernel drains its copies and returns.
#include <algorithm>
#include <cooperative_groups.h>
#include <string>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "feat.h"
#include "kernels.h"
#include "sort.h"

namespace cg = cooperative_groups;

namespace spmx {

constexpr int kTileBuf = 3;                  // stages in flight per CTA
constexpr unsigned kPadEntry = 0xffffffffu;  // packed word of a padding entry
constexpr int kTilePrefetch = 12;            // stages between L2 prefetch and bulk copy

struct TileStage {
  int window;  // column window of the stage
  int e0;      // first entry in the staged arrays (multiple of 4)
  int len;     // entries (multiple of 4, padding included)
  int rb;      // row block
};

struct TileGeom {
  int win;    // columns per window (multiple of 128)
  int chunk;  // entry capacity of a stage buffer (multiple of 4)
  int rmax;   // shared y entries (multiple of 4)
};

// Shared memory layout (dynamic): full[NB] and empty[NB] barriers, then per
// buffer the x window (win floats), the bitmap window (win/32 words), packed
// words and values (chunk each), then y (rmax floats).
template <int NW>
struct TileSmem {
  static constexpr int kBufBase = ((2 * kTileBuf * 8) + 127) & ~127;
  __host__ __device__ static int buf_bytes(const TileGeom& g) { return 4 * g.win + g.win / 8 + 8 * g.chunk; }
  __host__ __device__ static int total(const TileGeom& g) {
    return kBufBase + kTileBuf * buf_bytes(g) + 4 * g.rmax;
  }
};

// A warp adds its slice [lo, hi) of one stage into the shared y.  The slice
// holds len = hi - lo entries sorted by row, cut into 32 contiguous lane
// ranges of equal length (the first len % 32 lanes get one more).  The
// preprocessing stores the slice lane-interleaved: entry j of lane l's range
// sits at lo + 32 * j + l, so every load below is one conflict-free
// wavefront.  A lane walks its range in groups of G entries (all loads
// first), keeps the running sum of the current row in a register and adds
// every run that starts and ends inside its range to ys with a plain
// read-modify-write.  Only a run that continues into a neighbouring lane is
// added with shared atomics, piece by piece.  No other warp owns these rows.
template <int G, bool GATED>
__device__ __forceinline__ void tile_warp_slice(int lo, int hi, const unsigned* __restrict__ P,
                                                const float* __restrict__ V, const float* __restrict__ X,
                                                const unsigned* __restrict__ B, float* __restrict__ ys) {
  const int lane = threadIdx.x & 31;
  const int len = hi - lo;
  if (len <= 0) return;  // warp-uniform
  const int per = len >> 5, rem = len & 31;
  const int cnt = per + (lane < rem ? 1 : 0);
  const unsigned* Pl = P + lo + lane;
  const float* Vl = V + lo + lane;
  int hk = -1, cur = -1;  // head run row, current run row
  float hs = 0.f, acc = 0.f;
  bool head_open = true;  // still inside the first run of the range
  for (int j0 = 0; j0 < cnt; j0 += G) {
    const int ng = min(G, cnt - j0);
    unsigned w[G];
    float pr[G];
#pragma unroll
    for (int j = 0; j < G; ++j) w[j] = j < ng ? Pl[32 * (j0 + j)] : 0u;
#pragma unroll
    for (int j = 0; j < G; ++j) {
      const int c = (int)(w[j] & 0xffffu);
      float v = 0.f;
      if (j < ng) {
        v = Vl[32 * (j0 + j)] * X[c];
        if (GATED && !((B[c >> 5] >> (c & 31)) & 1u)) v = 0.f;
      }
      pr[j] = v;
    }
    int fr[G];
    float fs[G];
#pragma unroll
    for (int j = 0; j < G; ++j) {
      fr[j] = -1;
      fs[j] = 0.f;
      if (j < ng) {
        const int r = (int)(w[j] >> 16);
        if (cur < 0) {
          cur = r;
          hk = r;
          acc = pr[j];
        } else if (r != cur) {
          if (head_open) {
            hs = acc;  // the first run is added after the loop
            head_open = false;
          } else {
            fr[j] = cur;
            fs[j] = acc;
          }
          cur = r;
          acc = pr[j];
        } else {
          acc += pr[j];
        }
      }
    }
    float old[G];
#pragma unroll
    for (int j = 0; j < G; ++j) old[j] = fr[j] >= 0 ? ys[fr[j]] : 0.f;
#pragma unroll
    for (int j = 0; j < G; ++j)
      if (fr[j] >= 0) ys[fr[j]] = old[j] + fs[j];
  }
  // lane summary: head run (hk, hs) and tail run (cur, acc); one run if the
  // head never closed.  Every run that crosses a lane boundary is added once,
  // with a plain store, by the lane where it ends.
  const bool single = head_open;
  if (single) hs = acc;
  const int ptail = __shfl_up_sync(0xffffffffu, cur, 1);  // row ending the previous lane's range
  const bool cont = lane > 0 && cnt > 0 && ptail == hk;
  const bool ncont = __shfl_down_sync(0xffffffffu, cont, 1) && lane < 31;
  const float pacc = __shfl_up_sync(0xffffffffu, acc, 1);  // the previous lane's tail sum
  if (!__any_sync(0xffffffffu, single && cont && ncont)) {
    // common case: a crossing run spans two lanes; the second adds the first's part
    if (cont) ys[single ? cur : hk] += (single ? acc : hs) + pacc;
    else if (!single && hk >= 0) ys[hk] += hs;
    if (cur >= 0 && !ncont && !(single && cont)) ys[cur] += acc;
  } else {
    // a lane inside a longer run: chain the tail sums with a segmented scan
    float S = acc;
    bool F = !(single && cont);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const float oS = __shfl_up_sync(0xffffffffu, S, d);
      const bool oF = __shfl_up_sync(0xffffffffu, F, d);
      if (lane >= d && !F) {
        S += oS;
        F = oF;
      }
    }
    const float PS = __shfl_up_sync(0xffffffffu, S, 1);  // chain sum ending at lane - 1
    if (!single && hk >= 0) ys[hk] += hs + (cont ? PS : 0.f);
    if ((lane == 31 || !ncont) && cur >= 0) ys[cur] += S;
  }
  __syncwarp();
}

template <int NW, bool GATED>
__global__ void __launch_bounds__((NW + 1) * 32, 1)
tiled_spmv_kernel(int n, TileGeom g, int cs, const int* __restrict__ rb_row,
                  const int* __restrict__ cta_stage, const TileStage* __restrict__ stages,
                  const int* __restrict__ offsets, const unsigned* __restrict__ packed,
                  const float* __restrict__ val, const float* __restrict__ x,
                  const unsigned* __restrict__ xbits, int x_aligned, float alpha, float* __restrict__ y,
                  int* err) {
  using L = TileSmem<NW>;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ volatile int s_abort;
  unsigned long long* full = reinterpret_cast<unsigned long long*>(smem);
  unsigned long long* empty = full + kTileBuf;
  unsigned char* bufs = smem + L::kBufBase;
  const int bb = L::buf_bytes(g);
  float* ys = reinterpret_cast<float*>(bufs + kTileBuf * bb);
  auto xs_of = [&](int b) { return reinterpret_cast<float*>(bufs + b * bb); };
  auto bits_of = [&](int b) { return reinterpret_cast<unsigned*>(bufs + b * bb + 4 * g.win); };
  auto pk_of = [&](int b) { return reinterpret_cast<unsigned*>(bufs + b * bb + 4 * g.win + g.win / 8); };
  auto vv_of = [&](int b) {
    return reinterpret_cast<float*>(bufs + b * bb + 4 * g.win + g.win / 8 + 4 * g.chunk);
  };

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rb = blockIdx.x / cs;
  const int s0 = __ldg(cta_stage + blockIdx.x), s1 = __ldg(cta_stage + blockIdx.x + 1);
  const int cnt = s1 - s0;
  const int row0 = __ldg(rb_row + rb), rows = __ldg(rb_row + rb + 1) - row0;

  for (int r = threadIdx.x; r < g.rmax; r += blockDim.x) ys[r] = 0.f;
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int b = 0; b < kTileBuf; ++b) {
      bar_init(full + b, 1);
      bar_init(empty + b, NW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // launched as a programmatic dependent of the grid that writes x: nothing
  // above touches x or y
  asm volatile("griddepcontrol.wait;" ::: "memory");

  if (warp == NW) {
    // producer warp.  Lane l keeps the descriptor of stage (batch * 32 + l) in
    // registers, fetched one batch of 32 stages ahead, and that lane issues
    // the stage: it waits for the free buffer, arms the full barrier and
    // starts the bulk copies.  Only the window index is broadcast (the whole
    // warp copies an unaligned x tail), so a stage costs the producer a few
    // instructions and no global load.
    int4 cur_d = make_int4(0, 0, 0, 0), nxt_d = make_int4(0, 0, 0, 0);
    auto fetch = [&](int first, int4& d) {
      const int s = first + lane;
      if (s < cnt) d = __ldg(reinterpret_cast<const int4*>(stages) + s0 + s);
    };
    fetch(0, cur_d);
    fetch(32, nxt_d);
    if (lane < kTilePrefetch && lane < cnt && cur_d.z > 0) {
      l2_prefetch(packed + cur_d.y, 4u * cur_d.z);
      l2_prefetch(val + cur_d.y, 4u * cur_d.z);
    }
    int issued = 0;
    for (int i = 0; i < cnt; ++i) {
      const int b = i % kTileBuf;
      if (i > 0 && (i & 31) == 0) {
        cur_d = nxt_d;
        fetch(i + 32, nxt_d);
      }
      // L2 prefetch of the nonzeros of stage i + kTilePrefetch, by its lane
      {
        const int j = i + kTilePrefetch;
        if (j < cnt && lane == (j & 31)) {
          const int4 d = (j >> 5) == (i >> 5) ? cur_d : nxt_d;
          if (d.z > 0) {
            l2_prefetch(packed + d.y, 4u * d.z);
            l2_prefetch(val + d.y, 4u * d.z);
          }
        }
      }
      const int owner = i & 31;
      bool ok = true;
      if (lane == owner && i >= kTileBuf) ok = bar_wait(empty + b, ((i / kTileBuf) - 1) & 1, &s_abort);
      ok = __shfl_sync(0xffffffffu, ok, owner);
      if (!ok) {
        if (lane == owner) {
          flag_error(err, kDevErrTimeout);
          s_abort = 1;
        }
        break;
      }
      const int window = __shfl_sync(0xffffffffu, cur_d.x, owner);
      const int cbase = window * g.win;
      const int xw = min(g.win, n - cbase);
      float* xs = xs_of(b);
      unsigned* bits = bits_of(b);
      // x window: bulk copy of the 16-byte part, plain copy of the rest
      const int xb = x_aligned ? ((xw * 4) & ~15) : 0;
      for (int q = xb / 4 + lane; q < xw; q += 32) xs[q] = __ldg(x + cbase + q);
      int wb = 0;
      if (GATED) {
        const int nwd = (xw + 31) >> 5;
        wb = x_aligned ? ((nwd * 4) & ~15) : 0;
        for (int q = wb / 4 + lane; q < nwd; q += 32) bits[q] = __ldg(xbits + (cbase >> 5) + q);
      }
      __syncwarp();
      if (lane == owner) {
        const int e0 = cur_d.y, len = cur_d.z;
        bar_arrive_tx(full + b, (unsigned)(xb + wb + 8 * len));
        if (xb) bulk_load(xs, x + cbase, (unsigned)xb, full + b);
        if (wb) bulk_load(bits, xbits + (cbase >> 5), (unsigned)wb, full + b);
        if (len) {
          bulk_load(pk_of(b), packed + e0, 4u * len, full + b);
          bulk_load(vv_of(b), val + e0, 4u * len, full + b);
        }
      }
      issued = i + 1;
    }
    // no copy may still be in flight when the CTA leaves
    if (lane == 0) {
      volatile int never = 0;
      for (int i = max(0, issued - kTileBuf); i < issued; ++i)
        if (!bar_wait(full + (i % kTileBuf), (i / kTileBuf) & 1, &never)) flag_error(err, kDevErrTimeout);
    }
  } else {
    // consumer warps.  Lane l keeps this warp's entry range in stage
    // (batch * 32 + l), fetched one batch of 32 stages ahead.
    int2 cur_r = make_int2(0, 0), nxt_r = make_int2(0, 0);
    auto fetch = [&](int first, int2& r) {
      const int s = first + lane;
      if (s < cnt) {
        const int* o = offsets + (size_t)(s0 + s) * (NW + 1) + warp;
        r = make_int2(__ldg(o), __ldg(o + 1));
      }
    };
    fetch(0, cur_r);
    fetch(32, nxt_r);
    for (int i = 0; i < cnt; ++i) {
      const int b = i % kTileBuf;
      if (i > 0 && (i & 31) == 0) {
        cur_r = nxt_r;
        fetch(i + 32, nxt_r);
      }
      const int lo = __shfl_sync(0xffffffffu, cur_r.x, i & 31);
      const int hi = __shfl_sync(0xffffffffu, cur_r.y, i & 31);
      bool ok = true;
      if (lane == 0) ok = bar_wait(full + b, (i / kTileBuf) & 1, &s_abort);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) {
          flag_error(err, kDevErrTimeout);
          s_abort = 1;
        }
        break;
      }
      tile_warp_slice<(NW <= 4 ? 16 : 8), GATED>(lo, hi, pk_of(b), vv_of(b), xs_of(b), bits_of(b), ys);
      if (lane == 0) bar_arrive(empty + b);
    }
  }
  __syncthreads();

  // add the cluster's partial y vectors in rank order; each CTA stores a slice
  cg::cluster_group cl = cg::this_cluster();
  cl.sync();
  const int rank = (int)cl.block_rank();
  const int slice = (((rows + cs - 1) / cs) + 3) & ~3;
  const int r0 = rank * slice, r1 = min(rows, r0 + slice);
  for (int r = r0 + 4 * (int)threadIdx.x; r < r1; r += 4 * (int)blockDim.x) {
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int k = 0; k < cs; ++k) {
      const float4 v = *reinterpret_cast<const float4*>(cl.map_shared_rank(ys + r, k));
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

// tile key, local coordinates and value of every nonzero (CSR order)
__global__ void tile_keys_kernel(int m, int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                                 const float* __restrict__ val, const int* __restrict__ rb_row, int nrb,
                                 int win, int nwin, unsigned dump_key, unsigned* __restrict__ key,
                                 unsigned* __restrict__ packed, float* __restrict__ v_out, int* err) {
  // one warp per row
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= m) return;
  const int r = (int)gw;
  int lo = 0, hi = nrb;  // row block: the last rb with rb_row[rb] <= r
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
      flag_error(err, kDevErrOob);
      key[k] = dump_key;
      packed[k] = kPadEntry;
      v_out[k] = 0.f;
      continue;
    }
    const int w = c / win;
    key[k] = (unsigned)lo * (unsigned)nwin + (unsigned)w;
    packed[k] = (lr << 16) | (unsigned)(c - w * win);
    v_out[k] = __ldg(val + k);
  }
}

// tptr[t] = first position of key t in the sorted keys, t in [0, nkeys]
__global__ void tile_bounds_kernel(int nnz, const unsigned* __restrict__ skey, long long nkeys,
                                   int* __restrict__ tptr) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t > nkeys) return;
  int lo = 0, hi = nnz;
  while (lo < hi) {
    const int mid = (int)(((long long)lo + hi) >> 1);
    if ((long long)__ldg(skey + mid) < t) lo = mid + 1;
    else hi = mid;
  }
  tptr[t] = lo;
}

// move sorted entries to their padded slots (tile t starts at pad_start[t]);
// entries of the dump key (invalid columns) are dropped
__global__ void tile_scatter_kernel(int nvalid, const unsigned* __restrict__ skey,
                                    const unsigned* __restrict__ spk, const float* __restrict__ sval,
                                    const int* __restrict__ tptr, const long long* __restrict__ pad_start,
                                    unsigned* __restrict__ packed, float* __restrict__ vals) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nvalid; i += gridDim.x * blockDim.x) {
    const unsigned t = skey[i];
    const long long d = pad_start[t] + (i - __ldg(tptr + t));
    packed[d] = spk[i];
    vals[d] = sval[i];
  }
}

// per stage: where each consumer warp's rows begin inside the stage
__global__ void tile_offsets_kernel(int nstages, int nw, const TileStage* __restrict__ stages,
                                    const int* __restrict__ wsplit, const unsigned* __restrict__ packed,
                                    int* __restrict__ offsets) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nstages * (nw + 1)) return;
  const int s = (int)(t / (nw + 1)), k = (int)(t % (nw + 1));
  const TileStage sd = stages[s];
  int res;
  if (k == 0) {
    res = 0;
  } else {
    // first entry whose row >= split; padding entries (row 0xffff) belong to
    // no warp, so the last slice ends at the first of them
    const unsigned split = k == nw ? 0xffffu : (unsigned)__ldg(wsplit + sd.rb * (nw + 1) + k);
    int lo = 0, hi = sd.len;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if ((packed[sd.e0 + mid] >> 16) < split) lo = mid + 1;
      else hi = mid;
    }
    res = lo;
  }
  offsets[t] = res;
}

// Reorder every warp slice of every stage lane-interleaved (entry j of lane
// l's range to lo + 32 j + l, ranges as in tile_warp_slice); one CTA per
// stage, out-of-place.  Padding entries past the last slice keep their place.
__global__ void tile_interleave_kernel(int nw, const TileStage* __restrict__ stages,
                                       const int* __restrict__ offsets, const unsigned* __restrict__ pin,
                                       const float* __restrict__ vin, unsigned* __restrict__ pout,
                                       float* __restrict__ vout) {
  const TileStage sd = stages[blockIdx.x];
  const int* off = offsets + (size_t)blockIdx.x * (nw + 1);
  for (int t = threadIdx.x; t < sd.len; t += blockDim.x) {
    int dst = t;
    if (t < off[nw]) {
      int k = 0;  // warp slice holding t
      while (k + 1 < nw && off[k + 1] <= t) ++k;
      const int lo = off[k], len = off[k + 1] - lo;
      const int per = len >> 5, rem = len & 31;
      const int u = t - lo;
      int l, j;
      if (u < rem * (per + 1)) {
        l = u / (per + 1);
        j = u % (per + 1);
      } else {
        l = rem + (u - rem * (per + 1)) / per;
        j = (u - rem * (per + 1)) % per;
      }
      dst = lo + 32 * j + l;
    }
    pout[sd.e0 + dst] = pin[sd.e0 + t];
    vout[sd.e0 + dst] = vin[sd.e0 + t];
  }
}

}  // namespace spmx

using namespace spmx;

struct TiledTables {
  TileGeom g{8192, 2048, 4};
  int nw = 8, cs = 1, nrb = 0, grid = 0, nstages = 0;
  size_t smem = 0;
  unsigned* packed = nullptr;
  float* val = nullptr;
  TileStage* stages = nullptr;
  int* offsets = nullptr;
  int* cta_stage = nullptr;
  int* rb_row = nullptr;
};

static TiledTables* ttab(spmx_handle_t h) { return reinterpret_cast<TiledTables*>(h->tiled); }

static int log2_ceil(long long v) {
  int b = 0;
  while ((1LL << b) < v) ++b;
  return b;
}

extern "C" int spmx_tiled_postprocess(spmx_handle_t h) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  TiledTables* t = ttab(h);
  if (t) {
    cudaStreamSynchronize(h->stream);
    dfree(t->packed);
    dfree(t->val);
    dfree(t->stages);
    dfree(t->offsets);
    dfree(t->cta_stage);
    dfree(t->rb_row);
    delete t;
    h->tiled = nullptr;
  }
  return SPMX_SUCCESS;
}

template <int NW>
static void tiled_set_smem(size_t smem) {
  kernel_smem_limit((const void*)tiled_spmv_kernel<NW, false>, smem);
  kernel_smem_limit((const void*)tiled_spmv_kernel<NW, true>, smem);
}

// clusters of `cs` CTAs that can be resident at once (0 if unknown)
template <int NW>
static int tiled_max_clusters(int cs, size_t smem) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cs * 64);
  cfg.blockDim = dim3((NW + 1) * 32);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cs;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int nc = 0;
  if (cudaOccupancyMaxActiveClusters(&nc, (void*)tiled_spmv_kernel<NW, false>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nc;
}

// static shared memory of the kernel (barriers' abort flag and friends)
static long long tiled_static_smem(int nw) {
  cudaFuncAttributes a = {};
  cudaError_t e;
  if (nw == 16) e = cudaFuncGetAttributes(&a, tiled_spmv_kernel<16, true>);
  else if (nw == 4) e = cudaFuncGetAttributes(&a, tiled_spmv_kernel<4, true>);
  else e = cudaFuncGetAttributes(&a, tiled_spmv_kernel<8, true>);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 1024;
  }
  return (long long)a.sharedSizeBytes + 16;
}

static size_t tiled_smem_total(int nw, const TileGeom& g) {
  if (nw == 16) return (size_t)TileSmem<16>::total(g);
  if (nw == 4) return (size_t)TileSmem<4>::total(g);
  return (size_t)TileSmem<8>::total(g);
}

static void tiled_set_smem_nw(int nw, size_t smem) {
  if (nw == 16) tiled_set_smem<16>(smem);
  else if (nw == 4) tiled_set_smem<4>(smem);
  else tiled_set_smem<8>(smem);
}

static int tiled_max_clusters_nw(int nw, int cs, size_t smem) {
  if (nw == 16) return tiled_max_clusters<16>(cs, smem);
  if (nw == 4) return tiled_max_clusters<4>(cs, smem);
  return tiled_max_clusters<8>(cs, smem);
}

extern "C" int spmx_tiled_preprocess(spmx_handle_t h, int rb_rows, int win, int chunk, int warps) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  if (!h->has_csr || (!h->val && h->nnz > 0))
    return set_error(SPMX_ERR_NOT_READY, "tiled SpMV needs the CSR input with values");
  if (win <= 0) win = 8192;
  if (chunk <= 0) chunk = 2048;
  chunk = (chunk + 3) & ~3;
  if (warps <= 0) warps = 8;
  if (rb_rows < 0 || win % 128 || win > 65536 || chunk < 4 || chunk > (1 << 16) ||
      (warps != 4 && warps != 8 && warps != 16))
    return set_error(SPMX_ERR_INVALID_VALUE,
                     "tiled SpMV: win must be a multiple of 128 (<= 65536), chunk in [4, 65536], warps 4, 8 or 16");
  const int NW = warps;
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  TileGeom g{win, chunk, 4};
  const long long fixed = (long long)tiled_smem_total(NW, g) - 4 * g.rmax + tiled_static_smem(NW);
  long long rcap = ((long long)optin - fixed) / 4;
  rcap = std::min<long long>(rcap & ~3LL, 65532);
  if (rb_rows > 0) rcap = std::min<long long>(rcap, std::max(4, (rb_rows + 3) & ~3));
  if (rcap < 4) return set_error(SPMX_ERR_INVALID_VALUE, "tiled SpMV: win/chunk leave no shared memory for y");
  spmx_tiled_postprocess(h);
  TiledTables* t = new TiledTables();
  h->tiled = t;
  t->nw = NW;
  const int m = h->m, n = h->n, nnz = h->nnz;
  cudaStream_t st = h->stream;
  // row pointer on the host for the block and warp splits
  std::vector<int> rp((size_t)m + 1, 0);
  if (m > 0 &&
      cudaMemcpyAsync(rp.data(), h->rowptr, 4 * ((size_t)m + 1), cudaMemcpyDeviceToHost, st) != cudaSuccess) {
    spmx_tiled_postprocess(h);
    return set_error(SPMX_ERR_CUDA, "tiled SpMV: row pointer copy");
  }
  cudaStreamSynchronize(st);
  // cluster size and row block count: the largest cluster (4, 3 or 2 CTAs)
  // whose grid of one CTA per SM covers the rows in one wave (every cluster
  // resident at once); fewer row blocks mean fewer passes over x.  Otherwise
  // single CTAs over as many row blocks as needed.
  const int sms = h->num_sms;
  const long long need = std::max<long long>(1, (m + rcap - 1) / rcap);
  int cs = 1, nrb = (int)std::max<long long>(need, std::min(sms, std::max(1, m / 4)));
  for (int c = 4; c >= 2; --c) {
    const int nb = sms / c;
    if (nb < need || nb > std::max(1, m / 4)) continue;
    TileGeom gc = g;
    gc.rmax = (int)std::min<long long>(rcap, ((((long long)m + nb - 1) / nb) + 64 + 3) & ~3LL);
    const size_t sm_c = tiled_smem_total(NW, gc);
    tiled_set_smem_nw(NW, sm_c);
    if (tiled_max_clusters_nw(NW, c, sm_c) < nb) continue;
    cs = c;
    nrb = nb;
    break;
  }
  nrb = std::max(1, std::min(nrb, (m + 3) / 4));
  // row blocks: about equal nonzero counts, boundaries on multiples of 4, at
  // most rcap rows each
  std::vector<int> rbr(nrb + 1, 0);
  rbr[nrb] = m;
  for (int k = 1; k < nrb; ++k) {
    const long long want_nz = (long long)nnz * k / nrb;
    long long r = std::lower_bound(rp.begin(), rp.end(), (int)want_nz) - rp.begin();
    r = (r + 2) & ~3LL;
    const long long lo = std::max<long long>(rbr[k - 1], (long long)m - (long long)(nrb - k) * rcap);
    const long long hi = std::min<long long>((long long)rbr[k - 1] + rcap, m);
    r = std::max(r, (lo + 3) & ~3LL);
    r = std::min(r, hi & ~3LL);
    if (r < rbr[k - 1]) r = rbr[k - 1];
    rbr[k] = (int)r;
  }
  int rmax = 4;
  for (int k = 0; k < nrb; ++k) rmax = std::max(rmax, rbr[k + 1] - rbr[k]);
  if (rmax > rcap) {
    spmx_tiled_postprocess(h);
    return set_error(SPMX_ERR_INVALID_VALUE, "tiled SpMV: row blocks do not fit shared memory");
  }
  g.rmax = (rmax + 3) & ~3;
  t->g = g;
  t->cs = cs;
  t->nrb = nrb;
  t->smem = tiled_smem_total(NW, g);
  tiled_set_smem_nw(NW, t->smem);
  // consumer-warp row splits inside each row block (about equal nonzeros)
  std::vector<int> wsp((size_t)nrb * (NW + 1), 0);
  for (int k = 0; k < nrb; ++k) {
    const int a = rbr[k], b = rbr[k + 1];
    const long long z0 = rp[a], z1 = rp[b];
    for (int w = 0; w <= NW; ++w) {
      int r;
      if (w == 0) r = a;
      else if (w == NW) r = b;
      else
        r = (int)(std::lower_bound(rp.begin() + a, rp.begin() + b, (int)(z0 + (z1 - z0) * w / NW)) -
                  rp.begin());
      wsp[(size_t)k * (NW + 1) + w] = std::max(r - a, w ? wsp[(size_t)k * (NW + 1) + w - 1] : 0);
    }
  }
  const int nwin = std::max(1, (n + win - 1) / win);
  const long long ntiles = (long long)nrb * nwin;
  if (ntiles + 1 > (1LL << 30)) {
    spmx_tiled_postprocess(h);
    return set_error(SPMX_ERR_INVALID_VALUE, "tiled SpMV: too many tiles");
  }
  const size_t b = 4 * (size_t)std::max(nnz, 1);
  unsigned *k0 = nullptr, *k1 = nullptr, *p0 = nullptr, *p1 = nullptr, *v0 = nullptr, *v1 = nullptr;
  int *hist = nullptr, *hoff = nullptr, *tptr = nullptr, *d_wsp = nullptr;
  long long* d_pad = nullptr;
  const size_t hn = radix_hist_ints(std::max(nnz, 1));
  int rc = SPMX_SUCCESS;
  rc = rc ? rc : dalloc((void**)&k0, b, "tiled keys");
  rc = rc ? rc : dalloc((void**)&k1, b, "tiled keys alt");
  rc = rc ? rc : dalloc((void**)&p0, b, "tiled packed");
  rc = rc ? rc : dalloc((void**)&p1, b, "tiled packed alt");
  rc = rc ? rc : dalloc((void**)&v0, b, "tiled vals");
  rc = rc ? rc : dalloc((void**)&v1, b, "tiled vals alt");
  rc = rc ? rc : dalloc((void**)&hist, 4 * hn, "tiled hist");
  rc = rc ? rc : dalloc((void**)&hoff, 4 * hn, "tiled hist off");
  rc = rc ? rc : dalloc((void**)&tptr, 4 * (size_t)(ntiles + 2), "tiled pointers");
  rc = rc ? rc : dalloc((void**)&t->rb_row, 4 * (size_t)(nrb + 1), "tiled row blocks");
  rc = rc ? rc : dalloc((void**)&d_wsp, 4 * wsp.size(), "tiled warp splits");
  rc = rc ? rc : dalloc((void**)&d_pad, 8 * (size_t)ntiles, "tiled padded starts");
  if (!rc) {
    cudaMemcpyAsync(t->rb_row, rbr.data(), 4 * (size_t)(nrb + 1), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_wsp, wsp.data(), 4 * wsp.size(), cudaMemcpyHostToDevice, st);
  }
  std::vector<int> htp((size_t)ntiles + 2, 0);
  unsigned* spk = nullptr;
  float* sval = nullptr;
  unsigned* skey = nullptr;
  if (!rc && nnz > 0) {
    note_launch();
    tile_keys_kernel<<<(unsigned)(((long long)m * 32 + 255) / 256), 256, 0, st>>>(
        m, n, h->rowptr, h->col, h->val, t->rb_row, nrb, win, nwin, (unsigned)ntiles, k0, p0, (float*)v0,
        h->d_err);
    RadixBuffers rbuf{k0, k1, p0, p1, v0, v1, hist, hoff, false};
    if (radix_sort_pairs(rbuf, nnz, std::max(1, log2_ceil(ntiles + 1)), h->ls, h->d_err, st))
      rc = set_error(SPMX_ERR_INVALID_VALUE, "tiled SpMV: sort capacity");
    if (!rc) {
      skey = rbuf.result_in_alt ? k1 : k0;
      spk = rbuf.result_in_alt ? p1 : p0;
      sval = (float*)(rbuf.result_in_alt ? v1 : v0);
      // tile pointers by binary search in the sorted keys (the dump key of
      // invalid entries is ntiles, so tptr[ntiles] ends the valid entries)
      note_launch();
      tile_bounds_kernel<<<(unsigned)((ntiles + 1 + 256) / 256), 256, 0, st>>>(nnz, skey, ntiles + 1, tptr);
      if (!rc && cudaMemcpyAsync(htp.data(), tptr, 4 * (size_t)(ntiles + 2), cudaMemcpyDeviceToHost, st) !=
                     cudaSuccess)
        rc = set_error(SPMX_ERR_CUDA, "tiled SpMV: tile pointers");
    }
  }
  cudaError_t se = cudaStreamSynchronize(st);
  if (!rc && se != cudaSuccess) rc = set_error(SPMX_ERR_CUDA, cudaGetErrorString(se));
  // padded layout, stages and the per-CTA stage runs (host)
  std::vector<long long> pad((size_t)ntiles, 0);
  std::vector<TileStage> stg;
  std::vector<int> cta((size_t)nrb * cs + 1, 0);
  long long total = 0;
  if (!rc) {
    for (long long tt = 0; tt < ntiles; ++tt) {
      pad[tt] = total;
      total += ((long long)(htp[tt + 1] - htp[tt]) + 3) & ~3LL;
    }
    if (total >= (1LL << 31) - chunk) rc = set_error(SPMX_ERR_INVALID_VALUE, "tiled SpMV: too many entries");
  }
  if (!rc) {
    for (int k = 0; k < nrb; ++k) {
      const size_t first = stg.size();
      long long nz_rb = 0;
      for (int w = 0; w < nwin; ++w) {
        const long long tt = (long long)k * nwin + w;
        const int c = htp[tt + 1] - htp[tt];
        const int padded = (c + 3) & ~3;
        for (int o = 0; o < padded; o += chunk) {
          stg.push_back(TileStage{w, (int)(pad[tt] + o), std::min(chunk, padded - o), k});
          nz_rb += std::min(chunk, padded - o);
        }
      }
      // split the block's stages into cs runs of about equal entries
      long long acc = 0;
      int c = 1;
      cta[(size_t)k * cs] = (int)first;
      for (size_t s = first; s < stg.size() && c < cs; ++s) {
        acc += stg[s].len;
        while (c < cs && acc * cs >= nz_rb * c) cta[(size_t)k * cs + c++] = (int)s + 1;
      }
      while (c < cs) cta[(size_t)k * cs + c++] = (int)stg.size();
    }
    cta[(size_t)nrb * cs] = (int)stg.size();
  }
  t->nstages = (int)stg.size();
  t->grid = nrb * cs;
  const size_t words = 4 * (size_t)std::max<long long>(total, 4);
  rc = rc ? rc : dalloc((void**)&t->packed, words, "tiled staged words");
  rc = rc ? rc : dalloc((void**)&t->val, words, "tiled staged values");
  rc = rc ? rc : dalloc((void**)&t->stages, sizeof(TileStage) * std::max<size_t>(stg.size(), 1), "tiled stages");
  rc = rc ? rc : dalloc((void**)&t->offsets, 4 * (size_t)(NW + 1) * std::max<size_t>(stg.size(), 1), "tiled offsets");
  rc = rc ? rc : dalloc((void**)&t->cta_stage, 4 * cta.size(), "tiled CTA runs");
  if (!rc) {
    cudaMemsetAsync(t->packed, 0xff, words, st);
    cudaMemsetAsync(t->val, 0, words, st);
    cudaMemcpyAsync(d_pad, pad.data(), 8 * pad.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(t->cta_stage, cta.data(), 4 * cta.size(), cudaMemcpyHostToDevice, st);
    if (!stg.empty())
      cudaMemcpyAsync(t->stages, stg.data(), sizeof(TileStage) * stg.size(), cudaMemcpyHostToDevice, st);
    const int nvalid = htp[ntiles];
    if (nvalid > 0) {
      note_launch();
      tile_scatter_kernel<<<std::min((nvalid + 255) / 256, h->num_sms * 16), 256, 0, st>>>(
          nvalid, skey, spk, sval, tptr, d_pad, t->packed, t->val);
    }
    if (!stg.empty()) {
      const long long nt = (long long)stg.size() * (NW + 1);
      note_launch();
      tile_offsets_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>((int)stg.size(), NW, t->stages, d_wsp,
                                                                     t->packed, t->offsets);
      // lane-interleave the warp slices (out of place, then back)
      unsigned* tp2 = nullptr;
      float* tv2 = nullptr;
      rc = dalloc((void**)&tp2, words, "tiled interleave words");
      rc = rc ? rc : dalloc((void**)&tv2, words, "tiled interleave values");
      if (!rc) {
        note_launch();
        tile_interleave_kernel<<<(unsigned)stg.size(), 256, 0, st>>>(NW, t->stages, t->offsets, t->packed,
                                                                     t->val, tp2, tv2);
        cudaMemcpyAsync(t->packed, tp2, 4 * (size_t)total, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(t->val, tv2, 4 * (size_t)total, cudaMemcpyDeviceToDevice, st);
        cudaStreamSynchronize(st);
      }
      dfree(tp2);
      dfree(tv2);
    }
  }
  se = cudaStreamSynchronize(st);
  if (!rc && se != cudaSuccess) rc = set_error(SPMX_ERR_CUDA, cudaGetErrorString(se));
  dfree(k0); dfree(k1); dfree(p0); dfree(p1); dfree(v0); dfree(v1);
  dfree(hist); dfree(hoff); dfree(tptr); dfree(d_wsp); dfree(d_pad);
  if (rc) {
    spmx_tiled_postprocess(h);
    return rc;
  }
  return SPMX_SUCCESS;
}

template <int NW, bool GATED>
static cudaError_t tiled_launch(spmx_handle_t h, TiledTables* t, float alpha, float* y, const unsigned* bits,
                                int aligned) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(t->grid);
  cfg.blockDim = dim3((NW + 1) * 32);
  cfg.dynamicSmemBytes = t->smem;
  cfg.stream = h->stream;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = t->cs;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 2;
  // another handle's build may have set this kernel's limit for its own size
  const cudaError_t e = kernel_smem_limit((const void*)tiled_spmv_kernel<NW, GATED>, t->smem);
  if (e != cudaSuccess) return e;
  return cudaLaunchKernelEx(&cfg, tiled_spmv_kernel<NW, GATED>, h->n, t->g, t->cs, (const int*)t->rb_row,
                            (const int*)t->cta_stage, (const TileStage*)t->stages, (const int*)t->offsets,
                            (const unsigned*)t->packed, (const float*)t->val, (const float*)h->x_dense, bits,
                            aligned, alpha, y, h->d_err);
}

int tiled_spmv_impl(spmx_handle_t h, float alpha, float* y, bool gated) {
  TiledTables* t = ttab(h);
  if (!t) return set_error(SPMX_ERR_NOT_READY, "call spmx_tiled_preprocess first");
  if (!h->x_dense) return set_error(SPMX_VEC_FORMAT_ERR, "tiled SpMV needs the dense x");
  if (gated && !h->bitvec) return set_error(SPMX_VEC_FORMAT_ERR, "tiled SpMSpV needs the bitarray");
  if (!y && h->m > 0) return set_error(SPMX_ERR_INVALID_VALUE, "y is NULL");
  if (h->m == 0) return SPMX_SUCCESS;
  const unsigned* bits = gated ? (const unsigned*)h->bitvec : nullptr;
  const int aligned = ((((uintptr_t)h->x_dense) | (uintptr_t)bits) & 15u) == 0;
  note_launch();
  cudaError_t e;
  if (t->nw == 16)
    e = gated ? tiled_launch<16, true>(h, t, alpha, y, bits, aligned)
              : tiled_launch<16, false>(h, t, alpha, y, bits, aligned);
  else if (t->nw == 4)
    e = gated ? tiled_launch<4, true>(h, t, alpha, y, bits, aligned)
              : tiled_launch<4, false>(h, t, alpha, y, bits, aligned);
  else
    e = gated ? tiled_launch<8, true>(h, t, alpha, y, bits, aligned)
              : tiled_launch<8, false>(h, t, alpha, y, bits, aligned);
  if (e != cudaSuccess) return set_error(SPMX_ERR_CUDA, std::string("tiled spmv: ") + cudaGetErrorString(e));
  return SPMX_SUCCESS;
}

extern "C" int spmx_tiled_info(spmx_handle_t h, int* info) {
  if (!h || !info) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle or info");
  TiledTables* t = ttab(h);
  if (!t) return set_error(SPMX_ERR_NOT_READY, "call spmx_tiled_preprocess first");
  info[0] = t->nrb;
  info[1] = t->cs;
  info[2] = t->nstages;
  info[3] = t->g.win;
  info[4] = t->g.chunk;
  info[5] = t->g.rmax;
  info[6] = (int)t->smem;
  info[7] = t->nw;
  return SPMX_SUCCESS;
}

extern "C" int spmx_tiledspmv(spmx_handle_t h, float alpha, float* y) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  return tiled_spmv_impl(h, alpha, y, false);
}

extern "C" int spmx_tiledspmspv(spmx_handle_t h, float alpha, float* y) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  return tiled_spmv_impl(h, alpha, y, true);
}
