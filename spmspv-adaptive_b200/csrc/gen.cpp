// Deterministic synthetic inputs (host only).  Every random draw is a pure
// function of (seed, stream, counter) through a splitmix64-style hash, so the
// result does not depend on the OpenMP thread count.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <unordered_set>
#include <vector>

#include "spmx.h"

namespace {

inline uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
inline uint64_t rng(uint64_t seed, uint64_t stream, uint64_t ctr) {
  return mix64(mix64(seed * 0x632be59bd9b4e019ULL + stream) ^ (ctr * 0xd1b54a32d192ed03ULL));
}
// uniform in [0, 1)
inline double u01(uint64_t seed, uint64_t stream, uint64_t ctr) {
  return (double)(rng(seed, stream, ctr) >> 11) * (1.0 / 9007199254740992.0);
}
inline double normal(uint64_t seed, uint64_t stream, uint64_t ctr) {
  double u1 = u01(seed, stream, 2 * ctr), u2 = u01(seed, stream, 2 * ctr + 1);
  if (u1 < 1e-300) u1 = 1e-300;
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

enum Stream : uint64_t {
  kRmat = 1, kZipfLen = 2, kZipfRound = 3, kZipfFix = 4, kZipfCol = 5, kZipfVal = 6,
  kClEdge = 7, kClVal = 8, kLapVal = 9, kVecPos = 10, kVecVal = 11
};

// Build a symmetric CSR (sorted, deduplicated, no self-loops) from an edge
// list.  rowptr/col are malloc'ed and returned.
int build_symmetric_csr(int n, const std::vector<int>& eu, const std::vector<int>& ev,
                        long long* nnz_out, int** rowptr_out, int** col_out) {
  const long long E = (long long)eu.size();
  std::vector<long long> deg(n + 1, 0);
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < E; ++e) {
    if (eu[e] == ev[e]) continue;
#pragma omp atomic
    deg[eu[e]]++;
#pragma omp atomic
    deg[ev[e]]++;
  }
  std::vector<long long> off(n + 1, 0);
  for (int i = 0; i < n; ++i) off[i + 1] = off[i] + deg[i];
  std::vector<int> tmp((size_t)off[n]);
  std::vector<long long> cur(off.begin(), off.end() - 1);
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < E; ++e) {
    const int u = eu[e], v = ev[e];
    if (u == v) continue;
    long long pu, pv;
#pragma omp atomic capture
    pu = cur[u]++;
#pragma omp atomic capture
    pv = cur[v]++;
    tmp[pu] = v;
    tmp[pv] = u;
  }
  std::vector<int> ulen(n, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int i = 0; i < n; ++i) {
    int* b = tmp.data() + off[i];
    int* e = tmp.data() + off[i + 1];
    std::sort(b, e);
    ulen[i] = (int)(std::unique(b, e) - b);
  }
  int* rowptr = (int*)std::malloc(sizeof(int) * (size_t)(n + 1));
  if (!rowptr) return SPMX_ERR_ALLOC;
  long long total = 0;
  rowptr[0] = 0;
  for (int i = 0; i < n; ++i) {
    total += ulen[i];
    if (total > 2147483647LL) { std::free(rowptr); return SPMX_ERR_INVALID_VALUE; }
    rowptr[i + 1] = (int)total;
  }
  int* col = (int*)std::malloc(sizeof(int) * (size_t)std::max<long long>(total, 1));
  if (!col) { std::free(rowptr); return SPMX_ERR_ALLOC; }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int i = 0; i < n; ++i)
    std::memcpy(col + rowptr[i], tmp.data() + off[i], sizeof(int) * (size_t)ulen[i]);
  *nnz_out = total;
  *rowptr_out = rowptr;
  *col_out = col;
  return SPMX_SUCCESS;
}

}  // namespace

extern "C" void spmx_host_free(void* p) { std::free(p); }

extern "C" int spmx_gen_rmat(int scale, int edge_factor, double a, double b, double c,
                             uint64_t seed, int* m_out, long long* nnz_out, int** rowptr,
                             int** col) {
  if (scale < 1 || scale > 30 || edge_factor < 1 || !m_out || !nnz_out || !rowptr || !col)
    return SPMX_ERR_INVALID_VALUE;
  const int n = 1 << scale;
  const long long E = (long long)edge_factor << scale;
  std::vector<int> eu((size_t)E), ev((size_t)E);
  const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < E; ++e) {
    int u = 0, v = 0;
    for (int l = 0; l < scale; ++l) {
      const double r = u01(seed, kRmat, (uint64_t)e * 64 + l);
      int bu, bv;
      if (r < a) { bu = 0; bv = 0; }
      else if (r < ab) { bu = 0; bv = 1; }
      else if (r < abc) { bu = 1; bv = 0; }
      else { bu = 1; bv = 1; }
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    eu[e] = u;
    ev[e] = v;
  }
  *m_out = n;
  return build_symmetric_csr(n, eu, ev, nnz_out, rowptr, col);
}

extern "C" int spmx_gen_zipf_rows(int m, double s, int mean, int maxlen, uint64_t seed,
                                  long long* nnz_out, int** rowptr_out, int** col_out,
                                  float** val_out) {
  if (m < 1 || mean < 0 || maxlen < 1 || maxlen > m || !nnz_out || !rowptr_out || !col_out ||
      !val_out)
    return SPMX_ERR_INVALID_VALUE;
  const long long target = (long long)mean * m;
  if (target > 2147483647LL || target > (long long)maxlen * m) return SPMX_ERR_INVALID_VALUE;
  // truncated Zipf(s) on [1, maxlen]
  std::vector<double> cdf(maxlen);
  double z = 0, ez = 0;
  for (int k = 1; k <= maxlen; ++k) { const double p = std::pow((double)k, -s); z += p; ez += k * p; cdf[k - 1] = z; }
  for (auto& v : cdf) v /= z;
  ez /= z;
  const double f = ez > 0 ? (double)mean / ez : 0.0;
  std::vector<int> len(m);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < m; ++i) {
    const double r = u01(seed, kZipfLen, i);
    const int k = (int)(std::lower_bound(cdf.begin(), cdf.end(), r) - cdf.begin()) + 1;
    const double scaled = k * f;
    int L = (int)std::floor(scaled);
    if (u01(seed, kZipfRound, i) < scaled - L) ++L;
    len[i] = std::min(std::max(L, 0), maxlen);
  }
  long long tot = 0;
  for (int i = 0; i < m; ++i) tot += len[i];
  // fix the total to exactly mean*m by +-1 on random rows
  uint64_t ctr = 0;
  while (tot != target) {
    const int i = (int)(rng(seed, kZipfFix, ctr++) % (uint64_t)m);
    if (tot < target && len[i] < maxlen) { ++len[i]; ++tot; }
    else if (tot > target && len[i] > 0) { --len[i]; --tot; }
  }
  int* rowptr = (int*)std::malloc(sizeof(int) * (size_t)(m + 1));
  int* col = (int*)std::malloc(sizeof(int) * (size_t)std::max<long long>(target, 1));
  float* val = (float*)std::malloc(sizeof(float) * (size_t)std::max<long long>(target, 1));
  if (!rowptr || !col || !val) { std::free(rowptr); std::free(col); std::free(val); return SPMX_ERR_ALLOC; }
  rowptr[0] = 0;
  for (int i = 0; i < m; ++i) rowptr[i + 1] = rowptr[i] + len[i];
  const int n = m;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < m; ++i) {
    const int L = len[i];
    int* c = col + rowptr[i];
    // distinct uniform columns: draw, sort, deduplicate, redraw the shortfall
    int have = 0;
    uint64_t t = 0;
    while (have < L) {
      for (int k = have; k < L; ++k) c[k] = (int)(rng(seed, kZipfCol, ((uint64_t)i << 24) + t++) % (uint64_t)n);
      std::sort(c, c + L);
      have = (int)(std::unique(c, c + L) - c);
    }
    float* v = val + rowptr[i];
    for (int k = 0; k < L; ++k)
      v[k] = (float)(2.0 * u01(seed, kZipfVal, (uint64_t)rowptr[i] + k) - 1.0);
  }
  *nnz_out = target;
  *rowptr_out = rowptr;
  *col_out = col;
  *val_out = val;
  return SPMX_SUCCESS;
}

extern "C" int spmx_gen_chung_lu(int n, double gamma, double avg, uint64_t seed,
                                 long long* nnz_out, int** rowptr, int** col, float** val) {
  if (n < 2 || gamma <= 1.0 || avg <= 0 || !nnz_out || !rowptr || !col || !val)
    return SPMX_ERR_INVALID_VALUE;
  // expected degrees w_i ~ (i + i0)^(-1/(gamma-1)), scaled to mean avg, with
  // i0 chosen so that max w <= sqrt(sum w) (edge probabilities stay <= 1)
  const double ex = 1.0 / (gamma - 1.0);
  const double S = avg * n;
  const double wmax = std::sqrt(S);
  double i0 = 1.0;
  std::vector<double> w(n);
  for (int it = 0; it < 60; ++it) {
    double sum = 0;
    for (int i = 0; i < n; ++i) sum += std::pow(i + i0, -ex);
    const double scale = S / sum;
    if (scale * std::pow(i0, -ex) <= wmax) {
      for (int i = 0; i < n; ++i) w[i] = scale * std::pow(i + i0, -ex);
      break;
    }
    i0 *= 1.5;
  }
  std::vector<double> cdf(n);
  double acc = 0;
  for (int i = 0; i < n; ++i) { acc += w[i]; cdf[i] = acc; }
  for (auto& v : cdf) v /= acc;
  const long long E = (long long)(S / 2.0);
  std::vector<int> eu((size_t)E), ev((size_t)E);
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < E; ++e) {
    const double r1 = u01(seed, kClEdge, 2 * (uint64_t)e), r2 = u01(seed, kClEdge, 2 * (uint64_t)e + 1);
    eu[e] = (int)std::min<long long>(std::lower_bound(cdf.begin(), cdf.end(), r1) - cdf.begin(), n - 1);
    ev[e] = (int)std::min<long long>(std::lower_bound(cdf.begin(), cdf.end(), r2) - cdf.begin(), n - 1);
  }
  int rc = build_symmetric_csr(n, eu, ev, nnz_out, rowptr, col);
  if (rc) return rc;
  float* v = (float*)std::malloc(sizeof(float) * (size_t)std::max<long long>(*nnz_out, 1));
  if (!v) return SPMX_ERR_ALLOC;
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < *nnz_out; ++k) v[k] = (float)normal(seed, kClVal, (uint64_t)k);
  *val = v;
  return SPMX_SUCCESS;
}

extern "C" int spmx_gen_laplacian(int g, double sigma, uint64_t seed, long long* nnz_out,
                                  int** rowptr_out, int** col_out, float** val_out) {
  if (g < 1 || !nnz_out || !rowptr_out || !col_out || !val_out) return SPMX_ERR_INVALID_VALUE;
  const long long n = (long long)g * g;
  const long long nnz = 5 * n - 4LL * g;
  if (n > 2147483647LL || nnz > 2147483647LL) return SPMX_ERR_INVALID_VALUE;
  int* rowptr = (int*)std::malloc(sizeof(int) * (size_t)(n + 1));
  int* col = (int*)std::malloc(sizeof(int) * (size_t)nnz);
  float* val = (float*)std::malloc(sizeof(float) * (size_t)nnz);
  if (!rowptr || !col || !val) { std::free(rowptr); std::free(col); std::free(val); return SPMX_ERR_ALLOC; }
  rowptr[0] = 0;
  for (long long r = 0; r < n; ++r) {
    const int i = (int)(r / g), j = (int)(r % g);
    rowptr[r + 1] = rowptr[r] + 1 + (i > 0) + (i < g - 1) + (j > 0) + (j < g - 1);
  }
#pragma omp parallel for schedule(static)
  for (long long r = 0; r < n; ++r) {
    const int i = (int)(r / g), j = (int)(r % g);
    int p = rowptr[r];
    auto off = [&](long long c) {
      col[p] = (int)c;
      val[p] = (float)(-1.0 + sigma * normal(seed, kLapVal, (uint64_t)p));
      ++p;
    };
    if (i > 0) off(r - g);
    if (j > 0) off(r - 1);
    col[p] = (int)r; val[p] = 4.0f; ++p;
    if (j < g - 1) off(r + 1);
    if (i < g - 1) off(r + g);
  }
  *nnz_out = nnz;
  *rowptr_out = rowptr;
  *col_out = col;
  *val_out = val;
  return SPMX_SUCCESS;
}

extern "C" int spmx_gen_sparse_vector(int n, int k, int dist, uint64_t seed, int* key, float* val) {
  if (n < 0 || k < 0 || k > n || (k > 0 && (!key || !val))) return SPMX_ERR_INVALID_VALUE;
  if (k == 0) return SPMX_SUCCESS;
  if ((long long)k * 3 >= n) {
    // partial Fisher-Yates over [0, n)
    std::vector<int> p(n);
    for (int i = 0; i < n; ++i) p[i] = i;
    for (int i = 0; i < k; ++i) {
      const int j = i + (int)(rng(seed, kVecPos, i) % (uint64_t)(n - i));
      std::swap(p[i], p[j]);
    }
    std::memcpy(key, p.data(), sizeof(int) * (size_t)k);
  } else {
    std::unordered_set<int> seen;
    seen.reserve((size_t)k * 2);
    uint64_t t = 0;
    int have = 0;
    while (have < k) {
      const int c = (int)(rng(seed, kVecPos, t++) % (uint64_t)n);
      if (seen.insert(c).second) key[have++] = c;
    }
  }
  std::sort(key, key + k);
  for (int i = 0; i < k; ++i)
    val[i] = dist == 0 ? (float)(2.0 * u01(seed, kVecVal, i) - 1.0) : (float)normal(seed, kVecVal, i);
  return SPMX_SUCCESS;
}

extern "C" int spmx_host_csr2csc(int m, int n, const int* rowptr, const int* col,
                                 const float* val, int* colptr, int* row, float* cval) {
  if (m < 0 || n < 0 || !rowptr || !colptr) return SPMX_ERR_INVALID_VALUE;
  const int nnz = rowptr[m];
  std::fill(colptr, colptr + n + 1, 0);
  for (int k = 0; k < nnz; ++k) {
    if ((unsigned)col[k] >= (unsigned)n) return SPMX_ERR_INVALID_VALUE;
    colptr[col[k] + 1]++;
  }
  for (int c = 0; c < n; ++c) colptr[c + 1] += colptr[c];
  std::vector<int> cur(colptr, colptr + n);
  for (int r = 0; r < m; ++r)
    for (int k = rowptr[r]; k < rowptr[r + 1]; ++k) {
      const int p = cur[col[k]]++;
      row[p] = r;
      if (val && cval) cval[p] = val[k];
    }
  return SPMX_SUCCESS;
}
