// Batched SpMSpV and its adjoint (no reference counterpart: the reference
// runs one sparse vector per call).
//
// A batch is nvec sparse vectors in one concatenated list: vector v owns the
// entries [xptr[v], xptr[v+1]) of (xkey, xval), x_total entries in all; seen
// together they are a sparse n x nvec matrix X.  Forward: Y = alpha * A X,
// Y dense m x nvec, row-major (Y[i * nvec + v] = alpha * (A x_v)[i]).
// Backward, for an upstream gradient dY (m x nvec, row-major):
//   dxval[e] = alpha * sum_i A[i][xkey[e]] * dY[i][v(e)]
//              (the gradient of the stored values of x, same layout as xval)
//   dvals[k] = alpha * sum_{e : xkey[e] = col_k} xval[e] * dY[row_k][v(e)]
//              (the gradient of A's values, summed over the batch, CSR order)
//
// Design: the batch is inverted once per call (a stable radix sort of the
// entries by column gives, per column, the (vector, entry) pairs that use
// it; each pair is then stored as one 8-byte record of its vector and its x
// value for the forward, and one 16-byte record that adds its entry for the
// backward, so a row walk reads one sector per pair), then
//   forward  - one warp per row of A (CSR): lanes take the row's nonzeros,
//              look up their columns' pairs and add a[k] * x into a shared
//              row of nvec accumulators; the warp then stores the row of Y
//              once, coalesced.  No zero-fill, no global atomics.
//   dvals    - the same row walk against a shared copy of dY's row; every
//              nonzero's gradient is a sum over its column's pairs in sorted
//              order, stored once (deterministic).
//   dxval    - one warp per entry: a dot product of the entry's column of A
//              (CSC) with its vector's column of dY (deterministic).
// The forward's shared accumulators take atomic adds only when two entries of
// one vector meet in the same row.  Nothing is read back to the host, so after
// one call outside stream capture (which sizes the scratch for x_total) both
// entry points can be captured in a CUDA graph.
#include <algorithm>
#include <cstdint>
#include <string>

#include "common.cuh"
#include "engine.h"
#include "kernels.h"
#include "sort.h"

namespace spmx {

constexpr int kBatchWarps = 8;      // warps per CTA in the row kernels
constexpr int kBatchMaxVec = 1024;  // nvec limit (shared row accumulators)
// Row chunks of the row walks: a row weighs its nonzeros plus kBatchRowCost
// (the fixed cost of a row: its Y row store and its latency chain); chunk k
// holds the rows whose prefix weight rowptr[i] + kBatchRowCost * i starts in
// [k * kBatchChunk, (k + 1) * kBatchChunk).  Warps take chunks in order from
// a device counter, so the heavy rows (of a power-law matrix numbered by
// weight, the first ones) spread over the warps instead of landing one per
// warp in the first pass of a cyclic assignment.
constexpr int kBatchChunk = 2048;
constexpr int kBatchRowCost = 32;

// sort keys (column) and payloads (entry, vector) of every batch entry
__global__ void batch_keys_kernel(int n, int nvec, int total, const int* __restrict__ xptr,
                                  const int* __restrict__ xkey, unsigned* __restrict__ key,
                                  unsigned* __restrict__ ent, unsigned* __restrict__ vec, int* err) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    int lo = 0, hi = nvec;  // vector of entry e: last v with xptr[v] <= e
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(xptr + mid) <= e) lo = mid;
      else hi = mid;
    }
    const int j = __ldg(xkey + e);
    if ((unsigned)j >= (unsigned)n) flag_error(err, kDevErrOob);
    key[e] = (unsigned)j < (unsigned)n ? (unsigned)j : (unsigned)n;  // invalid keys sort last
    ent[e] = (unsigned)e;
    vec[e] = (unsigned)lo;
  }
}

// invptr[j] = first sorted position whose key is >= j, j in [0, n]: sorted
// position p (p in [0, total]) owns the columns after its predecessor's key
// up to its own key (n at p = total), so every column is written once
__global__ void batch_bounds_kernel(int total, const unsigned* __restrict__ skey, int n,
                                    int* __restrict__ invptr) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= total; p += gridDim.x * blockDim.x) {
    const int lo = p == 0 ? 0 : (int)__ldg(skey + p - 1) + 1;
    const int hi = p == total ? n : min((int)__ldg(skey + p), n);
    for (int j = lo; j <= hi; ++j) invptr[j] = p;
  }
}

// chunk_row[k] = first row i with rowptr[i] + kBatchRowCost * i >= k * kBatchChunk
// (chunk_row[nch] = m)
__global__ void batch_chunks_kernel(int m, const int* __restrict__ rowptr, int nch, int* __restrict__ chunk_row) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > nch) return;
  if (k == nch) {
    chunk_row[k] = m;
    return;
  }
  const long long target = (long long)k * kBatchChunk;
  int lo = 0, hi = m;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if ((long long)__ldg(rowptr + mid) + (long long)kBatchRowCost * mid < target) lo = mid + 1;
    else hi = mid;
  }
  chunk_row[k] = lo;
}

// A warp's rows, chunk by chunk: the next chunk is taken from the counter one
// chunk ahead (lane 0's atomic, broadcast), so its bounds are in registers by
// the time the current chunk runs out.  next() returns m once the chunks are
// exhausted.  Warp-uniform.
struct BatchRowIter {
  int r, end;  // next row of the current chunk, the chunk's end
  int n0, n1;  // the chunk taken ahead (n0 = m: none left)
  __device__ __forceinline__ void take(int* ctr, int nch, const int* __restrict__ chunk_row, int m, int lane) {
    int c = 0;
    if (lane == 0) c = atomicAdd(ctr, 1);
    c = __shfl_sync(0xffffffffu, c, 0);
    n0 = c < nch ? __ldg(chunk_row + c) : m;
    n1 = c < nch ? __ldg(chunk_row + c + 1) : m;
  }
  __device__ __forceinline__ void init(int* ctr, int nch, const int* __restrict__ chunk_row, int m, int lane) {
    r = end = 0;
    take(ctr, nch, chunk_row, m, lane);
  }
  __device__ __forceinline__ int next(int* ctr, int nch, const int* __restrict__ chunk_row, int m, int lane) {
    while (r >= end) {  // at most nch iterations: every pass takes a chunk
      if (n0 >= m) return m;
      r = n0;
      end = n1;
      take(ctr, nch, chunk_row, m, lane);
    }
    return r++;
  }
};

// rec[p] = (vector, x value bits) of sorted pair p, for the forward walk (four
// records per sector); rec4[p] = (vector, x value bits, entry, 0), for the
// backward walk, whose dxval atomic needs the entry
__global__ void batch_rec_kernel(int total, const unsigned* __restrict__ inv_ent,
                                 const unsigned* __restrict__ inv_vec, const float* __restrict__ xval,
                                 int2* __restrict__ rec, int4* __restrict__ rec4) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
    const int v = (int)__ldg(inv_vec + p), e = (int)__ldg(inv_ent + p);
    const int xb = __float_as_int(__ldg(xval + e));
    rec[p] = make_int2(v, xb);
    rec4[p] = make_int4(v, xb, e, 0);
  }
}

// Software pipeline of the row walks.  In the forward, a warp takes its rows
// from the row chunks (BatchRowIter); while it works on a row it already
// holds its next row's head (bounds, the lane's first column and value) with
// that column's pair range in flight, the head of the row after in flight
// and the bounds of the third in flight, so only the pair-record loads stay
// on the critical path of a row's first 32 nonzeros.  The dvals walk takes its
// rows from the chunks too, one row shallower (the next row's head and dY
// row, the bounds of the row after).  The dvals walk, which also holds the next row of dY in
// registers, runs one row shallower (row i + nw's head, row i + 2nw's
// bounds): the deeper form needs 64 registers there and loses more to the
// lower occupancy than it gains.
struct BatchRowHead {
  int a0, a1;  // row bounds
  int j;       // the lane's first column (a0 + lane), valid if has
  float a;     // its value (forward) or unused
  int p0, p1;  // the column's pair range, once looked up
  bool has;
};

__device__ __forceinline__ void batch_row_bounds(const int* __restrict__ rowptr, int m, long long i, int& a0,
                                                 int& a1) {
  a0 = a1 = 0;
  if (i < m) {
    a0 = __ldg(rowptr + i);
    a1 = __ldg(rowptr + i + 1);
  }
}

__device__ __forceinline__ BatchRowHead batch_row_head(const int* __restrict__ col, const float* __restrict__ val,
                                                       int a0, int a1, int lane) {
  BatchRowHead h{a0, a1, 0, 0.f, 0, 0, a0 + lane < a1};
  if (h.has) {
    h.j = __ldg(col + a0 + lane);
    if (val) h.a = __ldg(val + a0 + lane);
  }
  return h;
}

// the pair range of the head's column (empty for a lane without a nonzero or
// an out-of-range column, which is flagged)
__device__ __forceinline__ void batch_head_pairs(BatchRowHead& h, const int* __restrict__ invptr, int n, int* err) {
  h.p0 = h.p1 = 0;
  if (h.has) {
    if ((unsigned)h.j < (unsigned)n) {
      h.p0 = __ldg(invptr + h.j);
      h.p1 = __ldg(invptr + h.j + 1);
    } else {
      flag_error(err, kDevErrOob);
    }
  }
}

// acc[v] += a * x over the pairs [p0, p1), two records in flight at a time
__device__ __forceinline__ void batch_add_pairs(float* acc, const int2* __restrict__ rec, int p0, int p1, float a) {
  int p = p0;
  for (; p + 1 < p1; p += 2) {
    const int2 e = __ldg(rec + p), f = __ldg(rec + p + 1);
    atomicAdd(acc + e.x, a * __int_as_float(e.y));
    atomicAdd(acc + f.x, a * __int_as_float(f.y));
  }
  if (p < p1) {
    const int2 e = __ldg(rec + p);
    atomicAdd(acc + e.x, a * __int_as_float(e.y));
  }
}

// Y[i][:] = alpha * sum_k A[i][k] * X[col_k][:], one warp per row
__global__ void __launch_bounds__(kBatchWarps * 32)
batch_forward_kernel(int m, int n, int nvec, const int* __restrict__ rowptr, const int* __restrict__ col,
                     const float* __restrict__ val, const int* __restrict__ invptr,
                     const int2* __restrict__ rec, float alpha, float* __restrict__ Y, int vec4,
                     const int* __restrict__ chunk_row, int nch, int* ctr, int* err) {
  extern __shared__ __align__(16) float s_acc[];  // kBatchWarps rows of nvec
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* acc = s_acc + warp * nvec;
  for (int v = lane; v < nvec; v += 32) acc[v] = 0.f;
  __syncwarp();
  BatchRowIter it;
  it.init(ctr, nch, chunk_row, m, lane);
  int i = it.next(ctr, nch, chunk_row, m, lane);  // this row, then the next three of the warp
  int i1 = it.next(ctr, nch, chunk_row, m, lane);
  int i2 = it.next(ctr, nch, chunk_row, m, lane);
  int b0, b1;
  batch_row_bounds(rowptr, m, i, b0, b1);
  BatchRowHead cur = batch_row_head(col, val, b0, b1, lane);
  batch_row_bounds(rowptr, m, i1, b0, b1);
  BatchRowHead nxt = batch_row_head(col, val, b0, b1, lane);
  batch_head_pairs(cur, invptr, n, err);
  batch_row_bounds(rowptr, m, i2, b0, b1);  // row i2's bounds
  while (i < m) {
    // in flight meanwhile: row i1's pair range, row i2's head, the bounds of the row after
    batch_head_pairs(nxt, invptr, n, err);
    const BatchRowHead nn = batch_row_head(col, val, b0, b1, lane);
    const int i3 = it.next(ctr, nch, chunk_row, m, lane);
    int c0, c1;
    batch_row_bounds(rowptr, m, i3, c0, c1);
    batch_add_pairs(acc, rec, cur.p0, cur.p1, cur.a);
    // the row's nonzeros past the first 32, two per lane at a time
    for (int k = cur.a0 + 32 + lane; k < cur.a1; k += 64) {
      const bool two = k + 32 < cur.a1;
      const int j0 = __ldg(col + k), j1 = two ? __ldg(col + k + 32) : 0;
      const float v0 = __ldg(val + k), v1 = two ? __ldg(val + k + 32) : 0.f;
      const bool ok0 = (unsigned)j0 < (unsigned)n, ok1 = two && (unsigned)j1 < (unsigned)n;
      if (!ok0 || (two && !ok1)) flag_error(err, kDevErrOob);
      const int q00 = ok0 ? __ldg(invptr + j0) : 0, q01 = ok0 ? __ldg(invptr + j0 + 1) : 0;
      const int q10 = ok1 ? __ldg(invptr + j1) : 0, q11 = ok1 ? __ldg(invptr + j1 + 1) : 0;
      batch_add_pairs(acc, rec, q00, q01, v0);
      batch_add_pairs(acc, rec, q10, q11, v1);
    }
    __syncwarp();
    float* yr = Y + (size_t)i * nvec;
    if (vec4) {  // nvec % 4 == 0 and Y 16-byte aligned (checked on the host): vector stores
      float4* y4 = reinterpret_cast<float4*>(yr);
      float4* a4 = reinterpret_cast<float4*>(acc);
      for (int v = lane; v < (nvec >> 2); v += 32) {
        const float4 t = a4[v];
        y4[v] = make_float4(alpha * t.x, alpha * t.y, alpha * t.z, alpha * t.w);
        a4[v] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    } else {
      for (int v = lane; v < nvec; v += 32) {
        yr[v] = alpha * acc[v];
        acc[v] = 0.f;
      }
    }
    __syncwarp();
    cur = nxt;
    nxt = nn;
    b0 = c0;
    b1 = c1;
    i = i1;
    i1 = i2;
    i2 = i3;
  }
}

// 16-byte asynchronous copy global -> shared (L2 only), and its group waits
__device__ __forceinline__ void batch_cp16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void batch_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void batch_cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// dvals[k] = alpha * sum over column col_k's pairs of xval[e] * dY[i][v(e)],
// one warp per row with dY's row in shared memory.  With dxval (fused form,
// dxval zeroed before) every pair also adds alpha * a[k] * dY[i][v(e)] into
// dxval[e] with an atomic add.  The same pipeline as the forward; for
// nvec <= 256 with 16-byte rows (pre) each warp has two shared dY rows, and
// the next row of dY is copied into the other one (cp.async, no registers
// held) while this row is walked.
__global__ void __launch_bounds__(kBatchWarps * 32, 5)
batch_dvals_kernel(int m, int n, int nvec, const int* __restrict__ rowptr, const int* __restrict__ col,
                   const int* __restrict__ invptr, const int4* __restrict__ rec, float alpha,
                   const float* __restrict__ dY, float* __restrict__ dvals, const float* __restrict__ val,
                   float* __restrict__ dxval, int vec4, const int* __restrict__ chunk_row, int nch, int* ctr,
                   int* err) {
  extern __shared__ __align__(16) float s_dy[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool pre = vec4 && nvec <= 256;  // two shared dY rows per warp (the host sizes them)
  float* const g0 = s_dy + (size_t)warp * (pre ? 2 : 1) * nvec;
  const int n4 = nvec >> 2;
  int buf = 0;  // pre: the shared row holding this row's dY
  // pre: row r's dY (if the row has nonzeros) into shared row `into`; one
  // commit group per call, empty or not
  auto fetch = [&](int r, int a0, int a1, int into) {
    if (r < m && a0 < a1) {
      const float4* d4 = reinterpret_cast<const float4*>(dY + (size_t)r * nvec);
      float4* s4 = reinterpret_cast<float4*>(g0 + into * nvec);
      if (lane < n4) batch_cp16(s4 + lane, d4 + lane);
      if (lane + 32 < n4) batch_cp16(s4 + lane + 32, d4 + lane + 32);
    }
    batch_cp_commit();
  };
  BatchRowIter it;
  it.init(ctr, nch, chunk_row, m, lane);
  int i = it.next(ctr, nch, chunk_row, m, lane);  // this row and the warp's next
  int i1 = it.next(ctr, nch, chunk_row, m, lane);
  const float* aval = dxval ? val : nullptr;
  int b0, b1;
  batch_row_bounds(rowptr, m, i, b0, b1);
  BatchRowHead cur = batch_row_head(col, aval, b0, b1, lane);
  if (pre) fetch(i, b0, b1, 0);
  batch_row_bounds(rowptr, m, i1, b0, b1);
  while (i < m) {
    // in flight meanwhile: the next row's head and dY row, the bounds after it
    const BatchRowHead nxt = batch_row_head(col, aval, b0, b1, lane);
    if (pre) fetch(i1, b0, b1, buf ^ 1);  // the other row was last read before the previous __syncwarp
    const int i2 = it.next(ctr, nch, chunk_row, m, lane);
    int c0, c1;
    batch_row_bounds(rowptr, m, i2, c0, c1);
    if (cur.a0 < cur.a1) {  // warp-uniform
      float* const g = g0 + (pre ? buf * nvec : 0);
      if (pre) {
        batch_cp_wait<1>();  // every group but the next row's: this row's dY has landed
      } else if (vec4) {
        const float4* d4 = reinterpret_cast<const float4*>(dY + (size_t)i * nvec);
        for (int v = lane; v < n4; v += 32) reinterpret_cast<float4*>(g)[v] = __ldg(d4 + v);
      } else {
        for (int v = lane; v < nvec; v += 32) g[v] = __ldg(dY + (size_t)i * nvec + v);
      }
      __syncwarp();
      for (int k = cur.a0 + lane; k < cur.a1; k += 32) {
        const bool first = k == cur.a0 + lane;
        const int j = first ? cur.j : __ldg(col + k);
        float s = 0.f;
        if ((unsigned)j < (unsigned)n) {
          const int q1 = __ldg(invptr + j + 1);
          const float a = dxval ? alpha * (first ? cur.a : __ldg(val + k)) : 0.f;
          for (int p = __ldg(invptr + j); p < q1; ++p) {
            const int4 r = __ldg(rec + p);
            const float gv = g[r.x];
            s += __int_as_float(r.y) * gv;
            if (dxval) atomicAdd(dxval + r.z, a * gv);
          }
        } else {
          flag_error(err, kDevErrOob);
        }
        dvals[k] = alpha * s;
      }
      __syncwarp();
    }
    cur = nxt;
    buf ^= 1;
    b0 = c0;
    b1 = c1;
    i = i1;
    i1 = i2;
  }
  batch_cp_wait<0>();
}

// dxval[e] = alpha * sum_i A[i][xkey[e]] * dY[i][v(e)], one warp per entry
__global__ void __launch_bounds__(256)
batch_dxval_kernel(int m, int n, int nvec, int total, const int* __restrict__ xptr,
                   const int* __restrict__ xkey, const int* __restrict__ colptr,
                   const int* __restrict__ row, const float* __restrict__ cval, float alpha,
                   const float* __restrict__ dY, float* __restrict__ dxval, int* err) {
  const int lane = threadIdx.x & 31;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long e = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < total; e += nw) {
    int lo = 0, hi = nvec;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(xptr + mid) <= (int)e) lo = mid;
      else hi = mid;
    }
    const int v = lo;
    const int j = __ldg(xkey + e);
    float s = 0.f;
    if ((unsigned)j < (unsigned)n) {
      const int c1 = __ldg(colptr + j + 1);
      for (int q = __ldg(colptr + j) + lane; q < c1; q += 32) {
        const int i = __ldg(row + q);
        if ((unsigned)i < (unsigned)m) s += __ldg(cval + q) * __ldg(dY + (long long)i * nvec + v);
        else flag_error(err, kDevErrOob);
      }
    }
    s = warp_sum(s);
    if (lane == 0) dxval[e] = alpha * s;
  }
}

}  // namespace spmx

using namespace spmx;

// scratch for the inverted batch of x_total entries (grown, never shrunk)
static void batch_forget_inversion(spmx_handle_t h);

// the pair records: cap int2 records, then (at a 256-byte boundary) cap int4 records
static size_t batch_rec4_offset(int cap) { return (8 * (size_t)cap + 255) & ~(size_t)255; }

static int ensure_batch_scratch(spmx_handle_t h, int total) {
  if (h->batch_cap >= total && h->batch_invptr_n == h->n && h->batch_invptr) return SPMX_SUCCESS;
  batch_forget_inversion(h);
  cudaStreamSynchronize(h->stream);
  const int cap = std::max(total, 1);
  for (auto& p : h->batch_buf) {
    dfree(p);
    p = nullptr;
  }
  dfree(h->batch_hist);
  dfree(h->batch_hoff);
  dfree(h->batch_invptr);
  dfree(h->batch_rec);
  h->batch_rec = nullptr;
  h->batch_hist = h->batch_hoff = h->batch_invptr = nullptr;
  h->batch_cap = 0;
  const char* what[6] = {"batch keys", "batch keys alt", "batch entries", "batch entries alt",
                         "batch vectors", "batch vectors alt"};
  for (int b = 0; b < 6; ++b) SPMX_TRY(dalloc(&h->batch_buf[b], 4 * (size_t)cap, what[b]));
  const size_t hn = radix_hist_ints(cap);
  SPMX_TRY(dalloc((void**)&h->batch_hist, 4 * hn, "batch hist"));
  SPMX_TRY(dalloc((void**)&h->batch_hoff, 4 * hn, "batch hist off"));
  SPMX_TRY(dalloc((void**)&h->batch_invptr, 4 * ((size_t)h->n + 1), "batch inverse pointers"));
  SPMX_TRY(dalloc(&h->batch_rec, batch_rec4_offset(cap) + 16 * (size_t)cap, "batch pair records"));
  h->batch_cap = cap;
  h->batch_invptr_n = h->n;
  return SPMX_SUCCESS;
}

static void batch_forget_inversion(spmx_handle_t h) {
  h->inv_xptr = h->inv_xkey = h->inv_xval = nullptr;
  h->inv_nvec = h->inv_total = -1;
  h->inv_ent = h->inv_vec = nullptr;
}

// invert the batch: per column, the (entry, vector) pairs in entry order.
// A forward call records which batch the inversion belongs to; a backward
// call with SPMX_BATCH_REUSE_INVERSION set reuses it for the same batch.
static int batch_invert(spmx_handle_t h, int nvec, int total, const int* xptr, const int* xkey,
                        const float* xval, bool forward, const unsigned** inv_ent, const int2** rec,
                        const int4** rec4) {
  if (!forward && (h->batch_opts & SPMX_BATCH_REUSE_INVERSION) && h->inv_ent && h->inv_xptr == xptr &&
      h->inv_xkey == xkey && h->inv_xval == xval && h->inv_nvec == nvec && h->inv_total == total &&
      h->batch_invptr_n == h->n) {
    *inv_ent = h->inv_ent;
    *rec = (const int2*)h->batch_rec;
    *rec4 = (const int4*)((const char*)h->batch_rec + batch_rec4_offset(h->batch_cap));
    return SPMX_SUCCESS;
  }
  batch_forget_inversion(h);
  SPMX_TRY(ensure_batch_scratch(h, total));
  cudaStream_t st = h->stream;
  unsigned** b = reinterpret_cast<unsigned**>(h->batch_buf);
  if (total > 0) {
    note_launch();
    batch_keys_kernel<<<std::min((total + 255) / 256, h->num_sms * 8), 256, 0, st>>>(
        h->n, nvec, total, xptr, xkey, b[0], b[2], b[4], h->d_err);
  }
  RadixBuffers rb{b[0], b[1], b[2], b[3], b[4], b[5], h->batch_hist, h->batch_hoff, false};
  int bits = 1;
  while ((1LL << bits) <= (long long)h->n) ++bits;  // keys in [0, n]
  if (radix_sort_pairs(rb, total, bits, h->ls, h->d_err, st))
    return set_error(SPMX_ERR_INVALID_VALUE, "batch sort capacity");
  const unsigned* skey = rb.result_in_alt ? b[1] : b[0];
  *inv_ent = rb.result_in_alt ? b[3] : b[2];
  const unsigned* inv_vec = rb.result_in_alt ? b[5] : b[4];
  note_launch();
  batch_bounds_kernel<<<std::min((total + 1 + 255) / 256, h->num_sms * 8), 256, 0, st>>>(total, skey, h->n,
                                                                                         h->batch_invptr);
  if (total > 0) {
    note_launch();
    batch_rec_kernel<<<std::min((total + 255) / 256, h->num_sms * 8), 256, 0, st>>>(
        total, *inv_ent, inv_vec, xval, (int2*)h->batch_rec,
        (int4*)((char*)h->batch_rec + batch_rec4_offset(h->batch_cap)));
  }
  *rec = (const int2*)h->batch_rec;
  *rec4 = (const int4*)((const char*)h->batch_rec + batch_rec4_offset(h->batch_cap));
  if (forward) {
    h->inv_xptr = xptr;
    h->inv_xkey = xkey;
    h->inv_xval = xval;
    h->inv_nvec = nvec;
    h->inv_total = total;
    h->inv_ent = *inv_ent;
    h->inv_vec = inv_vec;
  }
  return SPMX_SUCCESS;
}

// the row chunks of the matrix (built once per CSR input; the counters they
// are taken from are zeroed before every launch)
static int ensure_batch_chunks(spmx_handle_t h) {
  if (h->batch_chunk_ready) return SPMX_SUCCESS;
  const long long w = (long long)h->nnz + (long long)kBatchRowCost * h->m;
  const long long nch = w / kBatchChunk + 1;
  if (nch >= INT32_MAX) return set_error(SPMX_ERR_INVALID_VALUE, "batched SpMSpV: too many row chunks");
  if (!h->batch_chunk || h->batch_nch != (int)nch) {
    dfree(h->batch_chunk);
    h->batch_chunk = nullptr;
    SPMX_TRY(dalloc((void**)&h->batch_chunk, 4 * ((size_t)nch + 1), "batch row chunks"));
  }
  if (!h->batch_ctr) SPMX_TRY(dalloc((void**)&h->batch_ctr, 2 * sizeof(int), "batch chunk counters"));
  note_launch();
  batch_chunks_kernel<<<(unsigned)((nch + 1 + 255) / 256), 256, 0, h->stream>>>(h->m, h->rowptr, (int)nch,
                                                                                h->batch_chunk);
  h->batch_nch = (int)nch;
  h->batch_chunk_ready = true;
  return launch_ok("batch row chunks");
}

static int batched_common(spmx_handle_t h, int nvec, int total, const int* xptr) {
  if (nvec < 1 || nvec > kBatchMaxVec)
    return set_error(SPMX_ERR_INVALID_VALUE, "nvec must be in [1, 1024]");
  if (total < 0) return set_error(SPMX_ERR_INVALID_VALUE, "x_total must be >= 0");
  if (!xptr) return set_error(SPMX_ERR_INVALID_VALUE, "xptr is NULL");
  if (!h->has_csr || (!h->val && h->nnz > 0))
    return set_error(SPMX_ERR_NOT_READY, "batched SpMSpV needs the CSR input with values");
  return SPMX_SUCCESS;
}

static int batch_rows_grid(spmx_handle_t h, const void* kernel, size_t smem) {
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kBatchWarps * 32, smem) != cudaSuccess ||
      per < 1) {
    cudaGetLastError();
    per = 2;
  }
  const long long want = ((long long)h->m + kBatchWarps - 1) / kBatchWarps;
  return (int)std::max(1LL, std::min<long long>(want, (long long)per * h->num_sms));
}

extern "C" int spmx_spmspv_batched(spmx_handle_t h, int nvec, int x_total, const int* d_xptr,
                                   const int* d_xkey, const float* d_xval, float alpha, float* d_Y) {
  SPMX_CHECK_HANDLE(h);
  SPMX_TRY(batched_common(h, nvec, x_total, d_xptr));
  if (!d_Y && h->m > 0) return set_error(SPMX_ERR_INVALID_VALUE, "Y is NULL");
  if (x_total > 0 && (!d_xkey || !d_xval)) return set_error(SPMX_ERR_INVALID_VALUE, "NULL batch arrays");
  const unsigned* ie = nullptr;
  const int2* rec = nullptr;
  const int4* rec4 = nullptr;
  SPMX_TRY(batch_invert(h, nvec, x_total, d_xptr, d_xkey, d_xval, true, &ie, &rec, &rec4));
  if (h->m == 0) return SPMX_SUCCESS;
  SPMX_TRY(ensure_batch_chunks(h));
  SPMX_CUDA(cudaMemsetAsync(h->batch_ctr, 0, sizeof(int), h->stream));
  const size_t smem = 4 * (size_t)kBatchWarps * nvec;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(batch_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  note_launch();
  batch_forward_kernel<<<batch_rows_grid(h, (const void*)batch_forward_kernel, smem), kBatchWarps * 32, smem,
                         h->stream>>>(h->m, h->n, nvec, h->rowptr, h->col, h->val, h->batch_invptr, rec,
                                      alpha, d_Y, (nvec % 4 == 0 && ((uintptr_t)d_Y & 15u) == 0) ? 1 : 0,
                                      h->batch_chunk, h->batch_nch, h->batch_ctr, h->d_err);
  return launch_ok("batched spmspv");
}

extern "C" int spmx_spmspv_batched_backward(spmx_handle_t h, int nvec, int x_total, const int* d_xptr,
                                            const int* d_xkey, const float* d_xval, float alpha,
                                            const float* d_dY, float* d_dxval, float* d_dvals) {
  SPMX_CHECK_HANDLE(h);
  SPMX_TRY(batched_common(h, nvec, x_total, d_xptr));
  if (!d_dY && h->m > 0) return set_error(SPMX_ERR_INVALID_VALUE, "dY is NULL");
  if (x_total > 0 && (!d_xkey || !d_xval)) return set_error(SPMX_ERR_INVALID_VALUE, "NULL batch arrays");
  cudaStream_t st = h->stream;
  // fused form: dxval accumulated by the dvals pass
  const bool fused = (h->batch_opts & SPMX_BATCH_FUSED_DXVAL) && d_dxval && d_dvals && h->nnz > 0 && x_total > 0;
  if (fused) SPMX_CUDA(cudaMemsetAsync(d_dxval, 0, 4 * (size_t)x_total, st));
  if (d_dvals && h->nnz > 0) {
    const unsigned* ie = nullptr;
    const int2* rec = nullptr;
    const int4* rec4 = nullptr;
    SPMX_TRY(batch_invert(h, nvec, x_total, d_xptr, d_xkey, d_xval, false, &ie, &rec, &rec4));
    SPMX_TRY(ensure_batch_chunks(h));
    SPMX_CUDA(cudaMemsetAsync(h->batch_ctr + 1, 0, sizeof(int), st));
    const bool vec4 = nvec % 4 == 0 && ((uintptr_t)d_dY & 15u) == 0;
    // with 16-byte rows of at most 256 entries each warp double-buffers its dY row
    const size_t smem = 4 * (size_t)kBatchWarps * nvec * (vec4 && nvec <= 256 ? 2 : 1);
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(batch_dvals_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    note_launch();
    batch_dvals_kernel<<<batch_rows_grid(h, (const void*)batch_dvals_kernel, smem), kBatchWarps * 32, smem,
                         st>>>(h->m, h->n, nvec, h->rowptr, h->col, h->batch_invptr, rec4, alpha,
                               d_dY, d_dvals, h->val, fused ? d_dxval : nullptr, vec4 ? 1 : 0, h->batch_chunk,
                               h->batch_nch, h->batch_ctr + 1, h->d_err);
  }
  if (d_dxval && x_total > 0 && !fused) {
    if (!h->has_csc || !h->csc_val)
      return set_error(SPMX_ERR_NOT_READY, "dxval needs the CSC with values (spmx_to_csc)");
    const long long warps = x_total;
    const int grid = (int)std::min<long long>((warps * 32 + 255) / 256, (long long)h->num_sms * 16);
    note_launch();
    batch_dxval_kernel<<<grid, 256, 0, st>>>(h->m, h->n, nvec, x_total, d_xptr, d_xkey, h->csc_colptr,
                                             h->csc_row, h->csc_val, alpha, d_dY, d_dxval, h->d_err);
  }
  return launch_ok("batched spmspv backward");
}

extern "C" int spmx_set_batch_options(spmx_handle_t h, int flags) {
  SPMX_CHECK_HANDLE(h);
  if (flags & ~(SPMX_BATCH_REUSE_INVERSION | SPMX_BATCH_FUSED_DXVAL))
    return set_error(SPMX_ERR_INVALID_VALUE, "unknown batch option flags");
  h->batch_opts = flags;
  return SPMX_SUCCESS;
}
