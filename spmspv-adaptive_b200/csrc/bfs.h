// BFS launchers (bfs.cu).
#pragma once
#include <cuda_runtime.h>

namespace spmx {

// device control block of the persistent BFS kernels (zeroed before a launch)
struct BfsCtrl {
  int cnt[3];                    // next-frontier sizes, by level % 3
  int depth;                     // number of levels, written at the end
  unsigned long long edges[3];   // sum of degrees of the next frontier
  unsigned bar_count, bar_gen;   // grid barrier
  int abort_flag;
  int pad;
};

struct BfsPersistentArgs {
  int n, src, num_sms;
  long long total_edges;
  const int* rowptr;
  const int* col;
  int* levels;
  unsigned* visited;
  unsigned* fb0;
  unsigned* fb1;
  unsigned* fb2;
  int* q0;
  int* q1;
  BfsCtrl* ctrl;
  double alpha, beta;  // direction switch: push->pull when m_f > m_u/alpha,
                       // pull->push when n_f < n/beta
  int* err;
};

// Hubs for the multi-source pull: every vertex of degree > deg is cut into
// chunks of deg edges that all warps share; acc / left are per-hub OR
// accumulators and outstanding-chunk counters, reset to 0 / nchunk_of each
// level.
struct HubChunks {
  const int4* chunk;     // {vertex, first edge, end edge, hub index}
  long long nchunks;
  const int* nchunk_of;  // chunks per hub
  unsigned long long* acc;
  int* left;
  int nhubs;
  int deg;
};

struct MsBfsArgs {
  int n, ns, num_sms;
  long long total_edges;
  double alpha;        // pull when the frontier's edges exceed total/alpha
  const int* srcs;     // device [ns]
  const int* rowptr;
  const int* col;
  int* levels;         // device [n * ns], vertex-major
  unsigned long long* visit;
  unsigned long long* front0;
  unsigned long long* front1;
  unsigned long long* next;
  int* q0;
  int* q1;
  BfsCtrl* ctrl;
  HubChunks hub;
  int* err;
};

int launch_hub_chunks(int n, const int* rowptr, int deg_cut, int4* chunk, int* nchunk_of,
                      int* counters, int max_hubs, int max_chunks, cudaStream_t st);
int launch_bfs_persistent(const BfsPersistentArgs& a, cudaStream_t st);
int launch_msbfs_persistent(const MsBfsArgs& a, cudaStream_t st);
int launch_levels_transpose(int n, int ns, const int* vmajor, int* smajor, cudaStream_t st);

int launch_bfs_init(int src, int* levels, unsigned* visited, int* q,
                    int* q_count, cudaStream_t st);
int launch_bfs_push(int nf, const int* queue, int n, const int* rowptr,
                    const int* col, unsigned* visited, int* levels,
                    int next_level, int* q_next, int* q_next_count,
                    unsigned long long* next_edges, int* err, int max_grid,
                    cudaStream_t st);
int launch_bfs_pull(int n, const int* rowptr, const int* col, unsigned* visited,
                    const unsigned* front, int* levels, int next_level,
                    int* q_next, int* q_next_count,
                    unsigned long long* next_edges, int* err, int max_grid,
                    cudaStream_t st);

}  // namespace spmx
