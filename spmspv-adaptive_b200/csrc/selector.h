// Kernel selector over the reference's 23-feature schema
// (model/1-test_dtree.py:63).  spmx_select_kernel returns one of SPMX_K_*.
//
// The reference trains three decision trees offline (solution, workload,
// write-back; model/[123]-test_dtree.py) and deploys them as generated C
// if/else code (model/1-test_dtree.py:93-112, get_code).  selector_tree.inc
// holds such generated code when a tree has been trained on this hardware
// (spmspv-adaptive_b200/spmx/train_selector.py writes it); without it the
// analytic traffic model below decides.
#pragma once
#include <math.h>
#include "spmx.h"

#if defined(__CUDACC__)
#define SPMX_HD __host__ __device__
#else
#define SPMX_HD
#endif

namespace spmx {

// Analytic model: bytes moved at the measured B200 copy bandwidth plus a
// fixed cost per dependent launch.  Feature indices follow SPMX_NUM_FEATURES.
SPMX_HD inline int select_by_traffic_model(const double* f) {
  const double m = f[0], n = f[1], nnz = f[2];
  const double max_row = f[3], avg_row = f[5] > 0 ? f[5] : 1.0;
  const double x = f[10], bin = f[11];
  const double bw = 6.5e6;     // bytes per microsecond (6.5 TB/s)
  const double launch = 2.5;   // microseconds per dependent launch
  const bool skewed = max_row > 8.0 * avg_row + 32.0;
  // CSC SpMSpV, atomic write-back: y memset, scan, gather + atomics
  const double csc_lb = 3 * launch + (4 * m + 16 * x + 8 * bin + 8 * bin) / bw;
  // f[12] holds the longest column of x (or an upper bound of it): one
  // group per column serialises on it
  const double avg_col = n > 0 ? nnz / n : 1.0;
  const double max_col = f[12] > 0 ? f[12] : avg_col;
  const bool col_skewed = max_col > 8.0 * avg_col + 64.0;
  const double csc_naive = 2 * launch + (4 * m + 12 * x + 16 * bin) / bw;
  // sort write-back: scan, read-back, pairs, radix passes, reduce
  const double passes = ceil(log2(m > 2 ? m : 2) / 8.0);
  const double csc_sort = (6 + 3 * passes) * launch + 10.0 +
                          (16 * x + 16 * bin + passes * 32 * bin) / bw;
  // CSR SpMSpV gated by the bitarray: s2a (2 memsets + scatter) + row pass
  const double s2a = 3 * launch + (4 * n + n / 8 + 8 * x) / bw;
  const double csr_spmspv = s2a + launch + (4 * (m + 1) + 4 * nnz + 8 * bin + 4 * m) / bw;
  // SpMV: s2d (memset + scatter) + row pass
  const double s2d = 2 * launch + (4 * n + 8 * x) / bw;
  const double spmv = s2d + launch + (4 * (m + 1) + 8 * nnz + 4 * n + 4 * m) / bw;
  double best = csc_lb;
  int k = SPMX_K_CSC_LB_ATOMIC;
  if (!col_skewed && csc_naive < best) { best = csc_naive; k = SPMX_K_CSC_NAIVE_ATOMIC; }
  if (csc_sort < best) { best = csc_sort; k = SPMX_K_CSC_LB_SORT; }
  if (csr_spmspv < best) { best = csr_spmspv; k = skewed ? SPMX_K_CSR_LB_SPMSPV : SPMX_K_CSR_NAIVE_SPMSPV; }
  if (spmv < best) { best = spmv; k = skewed ? SPMX_K_LB_SPMV : SPMX_K_NAIVE_SPMV; }
  return k;
}

}  // namespace spmx

#if __has_include("selector_tree.inc")
#include "selector_tree.inc"  // defines spmx::select_by_tree(const double*)
#define SPMX_HAVE_TREE 1
#endif

SPMX_HD inline int spmx_select_kernel(const double* f) {
#ifdef SPMX_HAVE_TREE
  return spmx::select_by_tree(f);
#else
  return spmx::select_by_traffic_model(f);
#endif
}
