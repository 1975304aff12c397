// Radix sort / scan / reduce_by_key launchers (sort.cu).
#pragma once
#include "kernels.h"

namespace spmx {

struct RadixBuffers {
  unsigned* keys;      // input keys; result here unless result_in_alt
  unsigned* keys_alt;
  unsigned* p1;        // optional payloads (NULL when absent)
  unsigned* p1_alt;
  unsigned* p2;
  unsigned* p2_alt;
  int* hist;           // radix_hist_ints(n) ints
  int* hist_off;       // same size
  bool result_in_alt;  // set by radix_sort_pairs
};

size_t radix_hist_ints(int n);
int radix_sort_pairs(RadixBuffers& b, int n, int key_bits, ScanScratch& ls,
                     int* err, cudaStream_t st);
int launch_scan_exclusive(const int* in, int* out, int n, int* total_out,
                          ScanScratch& ls, int* err, cudaStream_t st);
int reduce_by_key_sorted(const unsigned* keys, const float* vals, int n,
                         int* slot_scratch, int* out_key, float* out_val,
                         int* d_count, ScanScratch& ls, int* err,
                         cudaStream_t st);

}  // namespace spmx
