// Matrix / vector feature extraction on the device and small utility kernels.
//
// Matrix features restate computeMatFeture_serial (H:2275-2335) and the
// parallel stdRow of extractMatFeatureParallel (H:921-976, whose mean is
// truncated to int, H:929): max/min row length, mean, relative range,
// standard deviation, normalised row-length entropy ("edge equality") and the
// Gini coefficient of sorted row lengths.  The Gini sums are formed exactly
// from a row-length histogram (no sort, no float accumulation).
//
// Vector features restate computeVecFeture_serial (H:2338-2361) and
// computeBinlenVer2 (H:2703-2723) without copying colptr to the host.
#include "kernels.h"
#include "feat.h"
#include "common.cuh"

namespace spmx {

// acc layout (doubles): [0] sum (d-avg)^2, [1] sum (d-avg_int)^2, [2] entropy
// ints (separate array): [0] max, [1] min_inv (INT_MAX-min), [2] zero rows
__global__ void mat_features_kernel(int m, const int* __restrict__ rowptr,
                                    double nnz, double avg, double avg_int,
                                    double* acc, int* iacc) {
  double s0 = 0, s1 = 0, s2 = 0;
  int mx = 0, mn = INT_MAX, zeros = 0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += gridDim.x * blockDim.x) {
    const int d = __ldg(rowptr + r + 1) - __ldg(rowptr + r);
    const double dd = (double)d;
    s0 += (dd - avg) * (dd - avg);
    s1 += (dd - avg_int) * (dd - avg_int);
    if (d != 0) { const double p = dd / nnz; s2 += -p * log(p); }
    mx = max(mx, d);
    mn = min(mn, d);
    zeros += (d == 0);
  }
  s0 = warp_sum(s0); s1 = warp_sum(s1); s2 = warp_sum(s2);
  mx = warp_max(mx);
  int mninv = warp_max(INT_MAX - mn);
  zeros = warp_sum(zeros);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(acc + 0, s0);
    atomicAdd(acc + 1, s1);
    atomicAdd(acc + 2, s2);
    atomicMax(iacc + 0, mx);
    atomicMax(iacc + 1, mninv);
    atomicAdd(iacc + 2, zeros);
  }
}

__global__ void degree_hist_kernel(int m, const int* __restrict__ rowptr,
                                   int* __restrict__ hist) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += gridDim.x * blockDim.x) {
    const int d = __ldg(rowptr + r + 1) - __ldg(rowptr + r);
    atomicAdd(hist + d, 1);
  }
}

// sum over degree values v of v * (h_v * P_v + h_v*(h_v-1)/2): the sum of
// j * d_(j) over sorted positions j, with P_v = rows of degree < v.
__global__ void gini_sum_kernel(int maxdeg, const int* __restrict__ hist,
                                const int* __restrict__ pref,
                                unsigned long long* out) {
  unsigned long long s = 0;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v <= maxdeg;
       v += gridDim.x * blockDim.x) {
    const unsigned long long h = (unsigned)__ldg(hist + v);
    if (h) {
      const unsigned long long P = (unsigned)__ldg(pref + v);
      s += (unsigned long long)v * (h * P + h * (h - 1) / 2);
    }
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// vector features: sum / max / min of the column lengths of x's keys.
// out64[0] = bin_len; out32[0] = max, out32[1] = INT_MAX - min (both max-reduced
// from zero-initialised words).
__global__ void vec_features_kernel(int x_nnz, int n, const int* __restrict__ x_key,
                                    const int* __restrict__ colptr,
                                    unsigned long long* out64, int* out32,
                                    int* err) {
  unsigned long long s = 0;
  int mx = 0, mninv = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < x_nnz;
       i += gridDim.x * blockDim.x) {
    const int k = __ldg(x_key + i);
    if ((unsigned)k >= (unsigned)n) { flag_error(err, kDevErrOob); continue; }
    const int len = __ldg(colptr + k + 1) - __ldg(colptr + k);
    s += (unsigned)len;
    mx = max(mx, len);
    mninv = max(mninv, INT_MAX - len);
  }
  s = warp_sum(s);
  mx = warp_max(mx);
  mninv = warp_max(mninv);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out64, s);
    atomicMax(out32 + 0, mx);
    atomicMax(out32 + 1, mninv);
  }
}

// ---- utility kernels -------------------------------------------------------
__global__ void expand_rows_kernel(int m, const int* __restrict__ rowptr,
                                   unsigned* __restrict__ rows) {
  // one warp per row
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= m) return;
  const int r = (int)gw;
  const int a = __ldg(rowptr + r), b = __ldg(rowptr + r + 1);
  for (int k = a + lane; k < b; k += 32) rows[k] = (unsigned)r;
}

__global__ void count_keys_kernel(int nnz, int n, const int* __restrict__ keys,
                                  int* __restrict__ cnt, int* err) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
       i += gridDim.x * blockDim.x) {
    const int k = __ldg(keys + i);
    if ((unsigned)k < (unsigned)n) atomicAdd(cnt + k, 1);
    else flag_error(err, kDevErrOob);
  }
}

__global__ void set_int_kernel(int* p, int v) { *p = v; }

static int grid_for(long long work, int nt, int cap) {
  long long g = (work + nt - 1) / nt;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

int launch_mat_features(int m, const int* rowptr, int nnz, double avg,
                        double avg_int, double* acc, int* iacc,
                        cudaStream_t st) {
  if (m <= 0) return 0;
  note_launch();
  mat_features_kernel<<<grid_for(m, 256, 148 * 8), 256, 0, st>>>(
      m, rowptr, (double)(nnz > 0 ? nnz : 1), avg, avg_int, acc, iacc);
  return 0;
}

int launch_degree_hist(int m, const int* rowptr, int* hist, cudaStream_t st) {
  if (m <= 0) return 0;
  note_launch();
  degree_hist_kernel<<<grid_for(m, 256, 148 * 8), 256, 0, st>>>(m, rowptr, hist);
  return 0;
}

int launch_gini_sum(int maxdeg, const int* hist, const int* pref,
                    unsigned long long* out, cudaStream_t st) {
  note_launch();
  gini_sum_kernel<<<grid_for(maxdeg + 1, 256, 148 * 4), 256, 0, st>>>(maxdeg, hist, pref, out);
  return 0;
}

int launch_vec_features(int x_nnz, int n, const int* x_key, const int* colptr,
                        unsigned long long* out64, int* out32, int* err,
                        cudaStream_t st) {
  if (x_nnz <= 0) return 0;
  note_launch();
  vec_features_kernel<<<grid_for(x_nnz, 256, 148 * 8), 256, 0, st>>>(
      x_nnz, n, x_key, colptr, out64, out32, err);
  return 0;
}

int launch_expand_rows(int m, const int* rowptr, unsigned* rows, cudaStream_t st) {
  if (m <= 0) return 0;
  const long long threads = (long long)m * 32;
  note_launch();
  expand_rows_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(m, rowptr, rows);
  return 0;
}

int launch_count_keys(int nnz, int n, const int* keys, int* cnt, int* err,
                      cudaStream_t st) {
  if (nnz <= 0) return 0;
  note_launch();
  count_keys_kernel<<<grid_for(nnz, 256, 148 * 16), 256, 0, st>>>(nnz, n, keys, cnt, err);
  return 0;
}

int launch_set_int(int* p, int v, cudaStream_t st) {
  note_launch();
  set_int_kernel<<<1, 1, 0, st>>>(p, v);
  return 0;
}

}  // namespace spmx
