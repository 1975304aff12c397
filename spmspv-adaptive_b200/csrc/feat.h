// Feature-extraction and utility launchers (features.cu).
#pragma once
#include <cuda_runtime.h>

namespace spmx {

int launch_mat_features(int m, const int* rowptr, int nnz, double avg,
                        double avg_int, double* acc, int* iacc,
                        cudaStream_t st);
int launch_degree_hist(int m, const int* rowptr, int* hist, cudaStream_t st);
int launch_gini_sum(int maxdeg, const int* hist, const int* pref,
                    unsigned long long* out, cudaStream_t st);
int launch_vec_features(int x_nnz, int n, const int* x_key, const int* colptr,
                        unsigned long long* out64, int* out32, int* err,
                        cudaStream_t st);
int launch_expand_rows(int m, const int* rowptr, unsigned* rows, cudaStream_t st);
int launch_count_keys(int nnz, int n, const int* keys, int* cnt, int* err,
                      cudaStream_t st);
int launch_set_int(int* p, int v, cudaStream_t st);

}  // namespace spmx
