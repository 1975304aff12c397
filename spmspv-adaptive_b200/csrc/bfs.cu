// BFS on the Boolean (OR-AND) semiring, driven by sparse matrix-vector steps.
//
// The reference has no BFS: its "application" drivers replay recorded frontier
// patterns through the SpMSpV kernels (TEST/test_application.cu:207-261,
// TEST/new_test_app.cu:226-300).  Here each level is one Boolean SpMSpV:
//   push = CSC SpMSpV with the frontier as the sparse x, masked by the
//          visited set (each newly reached vertex claims its bit with one
//          atomicOr; winners are appended to the next frontier with a
//          warp-aggregated ballot/popc reservation);
//   pull = CSR SpMSpV gated by the frontier bitmap (bottom-up: every
//          unvisited vertex scans its row and stops at the first parent).
// The choice between them is the adaptive selector's CSC-vs-CSR decision,
// made per level from the frontier size and edge counts (direction-optimising
// BFS).
#include "kernels.h"
#include "bfs.h"
#include "common.cuh"

namespace spmx {

__device__ __forceinline__ bool test_bit(const unsigned* bits, int v) {
  return (bits[v >> 5] >> (v & 31)) & 1u;
}

// warp-aggregated append of `want` lanes' vertices to q; returns nothing
__device__ __forceinline__ void warp_append(bool want, int v, int deg, int* q,
                                            int* q_count,
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

// one warp per frontier vertex
__global__ void __launch_bounds__(256)
bfs_push_kernel(int nf, const int* __restrict__ queue, int n,
                const int* __restrict__ rowptr, const int* __restrict__ col,
                unsigned* visited, int* __restrict__ levels, int next_level,
                int* q_next, int* q_next_count, unsigned long long* next_edges,
                int* err) {
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long f = gw; f < nf; f += nwarps) {
    const int u = __ldg(queue + f);
    const int a = __ldg(rowptr + u), b = __ldg(rowptr + u + 1);
    for (int kb = a; kb < b; kb += 32) {
      const int k = kb + lane;
      bool win = false;
      int v = 0, deg = 0;
      if (k < b) {
        v = __ldg(col + k);
        if ((unsigned)v >= (unsigned)n) {
          flag_error(err, kDevErrOob);
        } else if (!test_bit(visited, v)) {
          const unsigned bit = 1u << (v & 31);
          const unsigned old = atomicOr(visited + (v >> 5), bit);
          if (!(old & bit)) {
            win = true;
            levels[v] = next_level;
            deg = __ldg(rowptr + v + 1) - __ldg(rowptr + v);
          }
        }
      }
      warp_append(win, v, deg, q_next, q_next_count, next_edges);
    }
  }
}

// one thread per vertex, grid-stride; warps stay converged for the append
__global__ void __launch_bounds__(256)
bfs_pull_kernel(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                unsigned* visited, const unsigned* __restrict__ front,
                int* __restrict__ levels, int next_level, int* q_next,
                int* q_next_count, unsigned long long* next_edges, int* err) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  // vb is the first vertex of this warp's 32; uniform across the warp
  for (long long vb = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
       vb < n; vb += stride) {
    const int v = (int)(vb + (threadIdx.x & 31));
    bool found = false;
    int deg = 0;
    if (v < n && !test_bit(visited, v)) {
      const int a = __ldg(rowptr + v), b = __ldg(rowptr + v + 1);
      deg = b - a;
      for (int k = a; k < b; ++k) {
        const int u = __ldg(col + k);
        if ((unsigned)u >= (unsigned)n) { flag_error(err, kDevErrOob); continue; }
        if (test_bit(front, u)) { found = true; break; }
      }
      if (found) {
        levels[v] = next_level;
        atomicOr(visited + (v >> 5), 1u << (v & 31));
      }
    }
    warp_append(found, v, deg, q_next, q_next_count, next_edges);
  }
}

__global__ void bfs_init_kernel(int src, int* levels, unsigned* visited, int* q,
                                int* q_count) {
  levels[src] = 0;
  visited[src >> 5] |= 1u << (src & 31);
  q[0] = src;
  *q_count = 1;
}

int launch_bfs_init(int src, int* levels, unsigned* visited, int* q,
                    int* q_count, cudaStream_t st) {
  note_launch();
  bfs_init_kernel<<<1, 1, 0, st>>>(src, levels, visited, q, q_count);
  return 0;
}

int launch_bfs_push(int nf, const int* queue, int n, const int* rowptr,
                    const int* col, unsigned* visited, int* levels,
                    int next_level, int* q_next, int* q_next_count,
                    unsigned long long* next_edges, int* err, int max_grid,
                    cudaStream_t st) {
  if (nf <= 0) return 0;
  long long warps = nf;
  long long blocks = (warps * 32 + 255) / 256;
  if (blocks > max_grid) blocks = max_grid;
  note_launch();
  bfs_push_kernel<<<(unsigned)blocks, 256, 0, st>>>(nf, queue, n, rowptr, col, visited,
                                                   levels, next_level, q_next,
                                                   q_next_count, next_edges, err);
  return 0;
}

int launch_bfs_pull(int n, const int* rowptr, const int* col, unsigned* visited,
                    const unsigned* front, int* levels, int next_level,
                    int* q_next, int* q_next_count,
                    unsigned long long* next_edges, int* err, int max_grid,
                    cudaStream_t st) {
  long long blocks = ((long long)n + 255) / 256;
  if (blocks > max_grid) blocks = max_grid;
  if (blocks < 1) blocks = 1;
  note_launch();
  bfs_pull_kernel<<<(unsigned)blocks, 256, 0, st>>>(n, rowptr, col, visited, front, levels,
                                                   next_level, q_next, q_next_count,
                                                   next_edges, err);
  return 0;
}

}  // namespace spmx
