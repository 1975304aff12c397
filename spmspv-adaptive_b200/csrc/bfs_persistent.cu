// Persistent BFS kernels: every level of a traversal inside ONE cooperative
// launch (all CTAs co-resident), levels separated by bounded grid barriers, the
// push/pull choice made on the device from frontier counters.  No host round
// trip per level.
//
// bfs_persistent_kernel: one source; levels as in the level-stepped kernels
//   of bfs.cu (push = Boolean CSC SpMSpV masked by the visited set, pull =
//   bitmap-gated CSR SpMSpV).
// msbfs_persistent_kernel: up to 64 sources at once, one bit per source in a
//   64-bit word per vertex (visited / frontier / next).  A frontier vertex
//   pushes its whole word to every neighbour (one 64-bit atomicOr), or an
//   unvisited vertex pulls the OR of its neighbours' frontier words and stops
//   once every source has reached it.  Levels are written vertex-major,
//   levels[v * ns + s], so each finished vertex is one contiguous store.
#include <algorithm>

#include "bfs.h"
#include "common.cuh"
#include "kernels.h"

namespace spmx {

__device__ __forceinline__ bool tbit(const unsigned* bits, int v) {
  return (bits[v >> 5] >> (v & 31)) & 1u;
}

__device__ __forceinline__ unsigned long long warp_or64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void warp_append2(bool want, int v, int deg, int* q, int* q_count,
                                             unsigned long long* edge_count) {
  const unsigned mask = __ballot_sync(0xffffffffu, want);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(q_count, __popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (want) q[base + __popc(mask & lanemask_lt())] = v;
  unsigned long long d = want ? (unsigned long long)deg : 0ull;
  d = warp_sum(d);
  if (lane == leader) atomicAdd(edge_count, d);
}

__global__ void __launch_bounds__(256)
bfs_persistent_kernel(int n, long long total_edges, const int* __restrict__ rowptr,
                      const int* __restrict__ col, int* __restrict__ levels,
                      unsigned* visited, unsigned* fb0, unsigned* fb1, unsigned* fb2, int* q0, int* q1,
                      BfsCtrl* ctrl, double alpha_b, double beta_b, int src, int* err) {
  const GridBarrier bar{&ctrl->bar_count, &ctrl->bar_gen, &ctrl->abort_flag};
  const int lane = threadIdx.x & 31;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nthreads = (long long)gridDim.x * blockDim.x;
  const long long gwarp = gtid >> 5, nwarps = nthreads >> 5;
  const long long words = (n + 31) >> 5;
  // initial state: every write goes to a distinct place, so one barrier suffices
  for (long long i = gtid; i < n; i += nthreads) levels[i] = i == src ? 0 : -1;
  for (long long w = gtid; w < words; w += nthreads) {
    const unsigned sb = w == (src >> 5) ? 1u << (src & 31) : 0u;
    visited[w] = sb;
    fb0[w] = sb;
    fb1[w] = 0u;
    fb2[w] = 0u;
  }
  if (gtid == 0) {
    q0[0] = src;
    for (int k = 0; k < 3; ++k) {
      ctrl->cnt[k] = 0;
      ctrl->edges[k] = 0ull;
    }
  }
  if (!grid_sync(bar, err)) return;
  const int src_deg = __ldg(rowptr + src + 1) - __ldg(rowptr + src);
  long long nf = 1, mf = src_deg, mu = total_edges - src_deg;
  bool pull = false;
  int L = 0, cur = 0;
  unsigned* fbs[3] = {fb0, fb1, fb2};
  while (true) {
    if (!pull && (double)mf > (double)mu / alpha_b) pull = true;
    else if (pull && (double)nf < (double)n / beta_b) pull = false;
    const int nxt = cur ^ 1;
    const int slot = (L + 1) % 3;
    int* qn = nxt ? q1 : q0;
    const int* qc = cur ? q1 : q0;
    // frontier bitmaps rotate over three buffers: this level reads fbs[L % 3],
    // writes fbs[(L + 1) % 3], and clears fbs[(L + 2) % 3] (the frontier of
    // the previous level, read by nobody now) for the next level; the counter
    // slot of the next level is cleared the same way.  One barrier per level.
    const unsigned* fbc = fbs[L % 3];
    unsigned* fbn = fbs[(L + 1) % 3];
    unsigned* fbr = fbs[(L + 2) % 3];
    if (L > 0)
      for (long long w = gtid; w < words; w += nthreads) fbr[w] = 0u;
    if (gtid == 0) {
      ctrl->cnt[(L + 2) % 3] = 0;
      ctrl->edges[(L + 2) % 3] = 0ull;
    }
    if (pull) {
      for (long long vb = gwarp * 32; vb < n; vb += nwarps * 32) {
        const int v = (int)(vb + lane);
        bool found = false;
        int deg = 0, a = 0, b = 0;
        const bool open = v < n && !tbit(visited, v);
        if (open) {
          a = __ldg(rowptr + v);
          b = __ldg(rowptr + v + 1);
          deg = b - a;
        }
        const bool heavy = open && deg > 32;
        if (open && !heavy) {
          for (int k = a; k < b; ++k) {
            const int u = __ldg(col + k);
            if ((unsigned)u >= (unsigned)n) { flag_error(err, kDevErrOob); continue; }
            if (tbit(fbc, u)) { found = true; break; }
          }
        }
        // vertices of degree > 32: the whole warp looks for a frontier neighbour
        unsigned hm = __ballot_sync(0xffffffffu, heavy);
        while (hm) {
          const int sl = __ffs(hm) - 1;
          hm &= hm - 1;
          const int ha = __shfl_sync(0xffffffffu, a, sl), hb = __shfl_sync(0xffffffffu, b, sl);
          bool any = false;
          for (int kb = ha; kb < hb && !any; kb += 32) {
            const int k = kb + lane;
            bool hit = false;
            if (k < hb) {
              const int u = __ldg(col + k);
              if ((unsigned)u >= (unsigned)n) flag_error(err, kDevErrOob);
              else hit = tbit(fbc, u);
            }
            any = __any_sync(0xffffffffu, hit);
          }
          if (lane == sl) found = any;
        }
        if (found) {
          levels[v] = L + 1;
          atomicOr(visited + (v >> 5), 1u << (v & 31));
          atomicOr(fbn + (v >> 5), 1u << (v & 31));
        }
        warp_append2(found, v, deg, qn, &ctrl->cnt[slot], &ctrl->edges[slot]);
      }
    } else {
      // a small frontier gets several warps per vertex (equal slices of its
      // adjacency), so a hub vertex does not serialise on one warp
      const long long g = nf < nwarps ? nwarps / nf : 1;
      for (long long wi = gwarp; wi < nf * g; wi += nwarps) {
        const long long f = wi / g;
        const long long part = wi - f * g;
        const int u = qc[f];
        const int a0 = __ldg(rowptr + u), b0 = __ldg(rowptr + u + 1);
        const int a = a0 + (int)(((long long)(b0 - a0) * part) / g);
        const int b = a0 + (int)(((long long)(b0 - a0) * (part + 1)) / g);
        for (int kb = a; kb < b; kb += 32) {
          const int k = kb + lane;
          bool win = false;
          int v = 0, deg = 0;
          if (k < b) {
            v = __ldg(col + k);
            if ((unsigned)v >= (unsigned)n) {
              flag_error(err, kDevErrOob);
            } else if (!tbit(visited, v)) {
              const unsigned bit = 1u << (v & 31);
              const unsigned old = atomicOr(visited + (v >> 5), bit);
              if (!(old & bit)) {
                win = true;
                levels[v] = L + 1;
                atomicOr(fbn + (v >> 5), bit);
                deg = __ldg(rowptr + v + 1) - __ldg(rowptr + v);
              }
            }
          }
          warp_append2(win, v, deg, qn, &ctrl->cnt[slot], &ctrl->edges[slot]);
        }
      }
    }
    if (!grid_sync(bar, err)) return;
    nf = *(volatile int*)&ctrl->cnt[slot];
    const long long me = (long long)*(volatile unsigned long long*)&ctrl->edges[slot];
    mf = me;
    mu -= me;
    if (nf == 0) break;
    cur = nxt;
    ++L;
  }
  if (gtid == 0) ctrl->depth = L + 1;
}


// ---------------------------------------------------------------------------
// multi-source BFS, up to 64 sources
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
msbfs_persistent_kernel(int n, int ns, long long total_edges, double alpha_ms,
                        const int* __restrict__ rowptr, const int* __restrict__ col,
                        int* __restrict__ levels, unsigned long long* visit,
                        unsigned long long* front0, unsigned long long* front1,
                        unsigned long long* next, int* q0, int* q1, BfsCtrl* ctrl,
                        HubChunks hub, int* err) {
  const GridBarrier bar{&ctrl->bar_count, &ctrl->bar_gen, &ctrl->abort_flag};
  const unsigned long long FULL = ns >= 64 ? ~0ull : ((1ull << ns) - 1ull);
  const int lane = threadIdx.x & 31;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nthreads = (long long)gridDim.x * blockDim.x;
  const long long gwarp = gtid >> 5, nwarps = nthreads >> 5;
  // the first frontier (written by msbfs_init_kernel into slot 0)
  long long nq = *(volatile int*)&ctrl->cnt[0];
  long long mf = (long long)*(volatile unsigned long long*)&ctrl->edges[0];
  int L = 0, cur = 0;
  while (true) {
    const bool pull = (double)mf > (double)total_edges / alpha_ms;
    const int nxt = cur ^ 1;
    const int slot = (L + 1) % 3;
    int* qn = nxt ? q1 : q0;
    const int* qc = cur ? q1 : q0;
    const unsigned long long* fc = cur ? front1 : front0;
    unsigned long long* fn = nxt ? front1 : front0;
    if (pull) {
      for (long long vb = gwarp * 32; vb < n; vb += nwarps * 32) {
        const int v = (int)(vb + lane);
        bool add = false;
        int deg = 0, a = 0, b = 0;
        unsigned long long vis = FULL;
        if (v < n) {
          vis = visit[v];
          a = __ldg(rowptr + v);
          b = __ldg(rowptr + v + 1);
          deg = b - a;
        }
        // hubs (degree > hub.deg) are pulled chunk by chunk below
        const bool open = v < n && vis != FULL && deg <= hub.deg;
        const bool heavy = open && deg > 32;
        unsigned long long nv = 0ull;
        if (open && !heavy) {
          unsigned long long acc = 0ull;
          for (int k = a; k < b; ++k) {
            const int u = __ldg(col + k);
            if ((unsigned)u >= (unsigned)n) { flag_error(err, kDevErrOob); continue; }
            acc |= fc[u];
            if ((acc | vis) == FULL) break;
          }
          nv = acc & ~vis;
        }
        // vertices of degree > 32: the whole warp pulls, one vertex at a time,
        // and stops once every source has reached the vertex
        unsigned hm = __ballot_sync(0xffffffffu, heavy);
        while (hm) {
          const int sl = __ffs(hm) - 1;
          hm &= hm - 1;
          const int ha = __shfl_sync(0xffffffffu, a, sl), hb = __shfl_sync(0xffffffffu, b, sl);
          const unsigned long long hvis = __shfl_sync(0xffffffffu, vis, sl);
          unsigned long long acc = 0ull;
          for (int kb = ha; kb < hb; kb += 32) {
            const int k = kb + lane;
            if (k < hb) {
              const int u = __ldg(col + k);
              if ((unsigned)u >= (unsigned)n) flag_error(err, kDevErrOob);
              else acc |= fc[u];
            }
            acc = warp_or64(acc);
            if ((acc | hvis) == FULL) break;
          }
          if (lane == sl) nv = acc & ~vis;
        }
        if (nv) {
          next[v] = nv;
          add = true;
        }
        warp_append2(add, v, deg, qn, &ctrl->cnt[slot], &ctrl->edges[slot]);
      }
      // hub chunks, spread over all warps: each ORs its slice of a hub's
      // neighbours into the hub's accumulator; the warp that retires the
      // hub's last chunk (a counter, no waiting) finishes the hub
      for (long long c = gwarp; c < hub.nchunks; c += nwarps) {
        const int4 ch = hub.chunk[c];  // {vertex, first edge, end edge, hub index}
        const unsigned long long hvis = visit[ch.x];
        unsigned long long acc = 0ull;
        if (hvis != FULL) {
          for (int kb = ch.y; kb < ch.z; kb += 32) {
            const int k = kb + lane;
            if (k < ch.z) {
              const int u = __ldg(col + k);
              if ((unsigned)u >= (unsigned)n) flag_error(err, kDevErrOob);
              else acc |= fc[u];
            }
          }
          acc = warp_or64(acc);
        }
        bool add = false;
        int deg = 0;
        if (lane == 0) {
          if (acc) atomicOr(hub.acc + ch.w, acc);
          __threadfence();
          if (atomicSub(hub.left + ch.w, 1) == 1) {
            __threadfence();
            const unsigned long long nv = atomicOr(hub.acc + ch.w, 0ull) & ~hvis;
            if (nv) {
              next[ch.x] = nv;
              add = true;
              deg = __ldg(rowptr + ch.x + 1) - __ldg(rowptr + ch.x);
            }
          }
        }
        warp_append2(add, ch.x, deg, qn, &ctrl->cnt[slot], &ctrl->edges[slot]);
      }
    } else {
      const long long g = nq < nwarps ? nwarps / nq : 1;  // warps per frontier vertex
      for (long long wi = gwarp; wi < nq * g; wi += nwarps) {
        const long long f = wi / g;
        const long long part = wi - f * g;
        const int u = qc[f];
        const unsigned long long fu = fc[u];
        const int a0 = __ldg(rowptr + u), b0 = __ldg(rowptr + u + 1);
        const int a = a0 + (int)(((long long)(b0 - a0) * part) / g);
        const int b = a0 + (int)(((long long)(b0 - a0) * (part + 1)) / g);
        for (int kb = a; kb < b; kb += 32) {
          const int k = kb + lane;
          bool add = false;
          int v = 0, deg = 0;
          if (k < b) {
            v = __ldg(col + k);
            if ((unsigned)v >= (unsigned)n) {
              flag_error(err, kDevErrOob);
            } else {
              const unsigned long long nv = fu & ~visit[v];
              if (nv) {
                const unsigned long long old = atomicOr(next + v, nv);
                if (old == 0ull) {
                  add = true;
                  deg = __ldg(rowptr + v + 1) - __ldg(rowptr + v);
                }
              }
            }
          }
          warp_append2(add, v, deg, qn, &ctrl->cnt[slot], &ctrl->edges[slot]);
        }
      }
    }
    if (!grid_sync(bar, err)) return;
    const long long nn = *(volatile int*)&ctrl->cnt[slot];
    const long long me = (long long)*(volatile unsigned long long*)&ctrl->edges[slot];
    // retire the current frontier
    for (long long f = gtid; f < nq; f += nthreads) ((unsigned long long*)fc)[qc[f]] = 0ull;
    // finalize the next frontier: one warp per vertex, levels stored vertex-major
    for (long long f = gwarp; f < nn; f += nwarps) {
      const int v = qn[f];
      unsigned long long nv = 0ull;
      if (lane == 0) {
        nv = next[v] & ~visit[v];
        visit[v] |= nv;
        fn[v] = nv;
        next[v] = 0ull;
      }
      nv = __shfl_sync(0xffffffffu, nv, 0);
      for (int s = lane; s < ns; s += 32)
        if ((nv >> s) & 1ull) levels[(long long)v * ns + s] = L + 1;
    }
    // hub accumulators for the next level
    for (long long i = gtid; i < hub.nhubs; i += nthreads) {
      hub.acc[i] = 0ull;
      hub.left[i] = hub.nchunk_of[i];
    }
    if (gtid == 0) {
      ctrl->cnt[(L + 2) % 3] = 0;
      ctrl->edges[(L + 2) % 3] = 0ull;
    }
    if (!grid_sync(bar, err)) return;
    nq = nn;
    mf = me;
    if (nq == 0) break;
    cur = nxt;
    ++L;
  }
  if (gtid == 0) ctrl->depth = L + 1;
}

// sources: distinct vertices enter the first frontier once, a vertex shared by
// several sources carries all their bits
__global__ void msbfs_init_kernel(int n, int ns, const int* __restrict__ srcs,
                                  const int* __restrict__ rowptr, int* levels,
                                  unsigned long long* visit, unsigned long long* front0,
                                  int* q0, BfsCtrl* ctrl) {
  int nq = 0;
  long long mf = 0;
  for (int s = 0; s < ns; ++s) {
    const int v = srcs[s];
    if ((unsigned)v >= (unsigned)n) continue;
    if (front0[v] == 0ull) {
      q0[nq++] = v;
      mf += rowptr[v + 1] - rowptr[v];
    }
    front0[v] |= 1ull << s;
    visit[v] |= 1ull << s;
    levels[(long long)v * ns + s] = 0;
  }
  ctrl->cnt[0] = nq;
  ctrl->edges[0] = (unsigned long long)mf;
}

__global__ void levels_transpose_kernel(int n, int ns, const int* __restrict__ vmajor,
                                        int* __restrict__ smajor) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)n * ns) return;
  const int s = (int)(i / n), v = (int)(i % n);
  smajor[i] = vmajor[(long long)v * ns + s];
}

// --------------------------------------------------------------------------
// Co-resident grid for a cooperative launch, scaled to the work: every CTA
// joins every grid barrier, so a small graph gets few CTAs (one per SM down
// to 1024 vertices per CTA) and a large one the whole resident capacity.
template <class K>
static int coop_grid(K kernel, int num_sms, int min_ctas, long long work_items) {
  // the occupancy query costs host time on every launch otherwise; one value
  // per kernel (the same on every GPU of a node)
  static int per = -1;
  if (per < 0) {
    int p = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, kernel, 256, 0) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    per = p;
  }
  const long long cap = (long long)per * num_sms;
  long long want = (work_items + 255) / 256;
  if (want < min_ctas) want = min_ctas;
  if (want > cap) want = cap;
  return (int)want;
}

int launch_bfs_persistent(const BfsPersistentArgs& a, cudaStream_t st) {
  // small graphs get few CTAs: the level barriers then cost less
  const int grid = coop_grid(bfs_persistent_kernel, a.num_sms, 16, a.n);
  if (grid <= 0) return -1;
  cudaMemsetAsync(a.ctrl, 0, sizeof(BfsCtrl), st);
  note_launch();
  int n = a.n;
  long long te = a.total_edges;
  const int* rp = a.rowptr;
  const int* cl = a.col;
  int* lv = a.levels;
  unsigned* vis = a.visited;
  unsigned* f0 = a.fb0;
  unsigned* f1 = a.fb1;
  unsigned* f2 = a.fb2;
  int* q0 = a.q0;
  int* q1 = a.q1;
  BfsCtrl* ctrl = a.ctrl;
  double al = a.alpha, be = a.beta;
  int src = a.src;
  int* err = a.err;
  void* args[] = {&n, &te, &rp, &cl, &lv, &vis, &f0, &f1, &f2, &q0, &q1, &ctrl, &al, &be, &src, &err};
  cudaError_t e = cudaLaunchCooperativeKernel((void*)bfs_persistent_kernel, grid, 256, args, 0, st);
  return e == cudaSuccess ? 0 : -2;
}

// chunks of hub.deg edges of every vertex of degree > hub.deg
__global__ void hub_chunks_kernel(int n, const int* __restrict__ rowptr, int deg_cut, int4* chunk,
                                  int* nchunk_of, int* counters, int max_hubs, int max_chunks) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const int a = __ldg(rowptr + v), b = __ldg(rowptr + v + 1);
    if (b - a <= deg_cut) continue;
    const int nch = (b - a + deg_cut - 1) / deg_cut;
    const int hi = atomicAdd(counters, 1);
    const int base = atomicAdd(counters + 1, nch);
    if (hi >= max_hubs || base + nch > max_chunks) continue;  // cannot happen by the bounds
    nchunk_of[hi] = nch;
    for (int j = 0; j < nch; ++j)
      chunk[base + j] = make_int4(v, a + j * deg_cut, min(b, a + (j + 1) * deg_cut), hi);
  }
}

int launch_hub_chunks(int n, const int* rowptr, int deg_cut, int4* chunk, int* nchunk_of,
                      int* counters, int max_hubs, int max_chunks, cudaStream_t st) {
  if (n <= 0) return 0;
  note_launch();
  hub_chunks_kernel<<<std::min((n + 255) / 256, 148 * 8), 256, 0, st>>>(n, rowptr, deg_cut, chunk, nchunk_of,
                                                                       counters, max_hubs, max_chunks);
  return 0;
}

int launch_msbfs_persistent(const MsBfsArgs& a, cudaStream_t st) {
  const int grid = coop_grid(msbfs_persistent_kernel, a.num_sms, a.num_sms, a.n);
  if (grid <= 0) return -1;
  cudaMemsetAsync(a.ctrl, 0, sizeof(BfsCtrl), st);
  note_launch(2);
  msbfs_init_kernel<<<1, 1, 0, st>>>(a.n, a.ns, a.srcs, a.rowptr, a.levels, a.visit,
                                     a.front0, a.q0, a.ctrl);
  int n = a.n, ns = a.ns;
  long long te = a.total_edges;
  double al = a.alpha;
  const int* rp = a.rowptr;
  const int* cl = a.col;
  int* lv = a.levels;
  unsigned long long* vis = a.visit;
  unsigned long long* f0 = a.front0;
  unsigned long long* f1 = a.front1;
  unsigned long long* nx = a.next;
  int* q0 = a.q0;
  int* q1 = a.q1;
  BfsCtrl* ctrl = a.ctrl;
  HubChunks hub = a.hub;
  int* err = a.err;
  void* args[] = {&n, &ns, &te, &al, &rp, &cl, &lv, &vis, &f0, &f1, &nx, &q0, &q1, &ctrl, &hub, &err};
  cudaError_t e = cudaLaunchCooperativeKernel((void*)msbfs_persistent_kernel, grid, 256, args, 0, st);
  return e == cudaSuccess ? 0 : -2;
}

int launch_levels_transpose(int n, int ns, const int* vmajor, int* smajor, cudaStream_t st) {
  const long long tot = (long long)n * ns;
  if (tot <= 0) return 0;
  note_launch();
  levels_transpose_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(n, ns, vmajor, smajor);
  return 0;
}

}  // namespace spmx
