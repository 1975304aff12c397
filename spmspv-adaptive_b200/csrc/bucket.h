// Bucket-based CSC SpMSpV launcher (bucket.cu).
#pragma once
#include "kernels.h"

namespace spmx {

constexpr int kBucketMax = 16384;  // buckets per call (shared-memory histogram)

struct BucketScratch {
  int* gcount;   // [kBucketMax]
  int* boff;     // [kBucketMax + 1]
  int* cursor;   // [kBucketMax]
  int* prow;     // pair rows   [cap]
  float* pval;   // pair values [cap]
  int cap;
};

// rows per bucket = 1 << rshift (256 .. 8192); returns -1 if m needs more
// than kBucketMax buckets
int bucket_geometry(int m, int buckets, int* rshift, int* nb);
int launch_bucket_spmspv(const CscArgs& a, const CscScratch& s, const BucketScratch& bs,
                         int variant, int rshift, int nb, float* y, int* ykey,
                         float* yval, int* d_count, ScanScratch& ls, int grid,
                         cudaStream_t st);

}  // namespace spmx
