// BFS launchers (bfs.cu).
#pragma once
#include <cuda_runtime.h>

namespace spmx {

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
