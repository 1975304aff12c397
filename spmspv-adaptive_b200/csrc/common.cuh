// Shared device helpers for the spmx kernels: warp/block scans, bounded waits,
// a decoupled look-back tile scan and the device error word.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <utility>

namespace spmx {

constexpr int kWarp = 32;

// Bits of the per-handle device error word.  Kernels never trap: they record
// the problem here, skip the offending access and return.
enum DeviceError : int {
  kDevErrTimeout = 1,  // a bounded wait (look-back, grid barrier) gave up
  kDevErrOob = 2,      // an index outside its array (bad x key, bad column)
  kDevErrCapacity = 4, // an internal capacity was exceeded
};

// Upper bound on spin iterations of any wait; with the back-off below this is
// on the order of seconds, far beyond any legitimate wait.
constexpr long long kSpinLimit = 1LL << 24;

__device__ __forceinline__ void flag_error(int* err, int code) {
  if (err) atomicOr(err, code);
}

// mbarrier and bulk-copy (cp.async.bulk) helpers for shared-memory staging
// rings.  Every wait is bounded.
constexpr long long kBarSpinLimit = 1LL << 22;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void bar_init(unsigned long long* b, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void bar_arrive(unsigned long long* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}

__device__ __forceinline__ void bar_arrive_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes)
               : "memory");
}

// waits for the phase of parity `parity` to complete; false after the limit
// or once another warp has raised the abort flag
__device__ __forceinline__ bool bar_wait(unsigned long long* b, int parity, const volatile int* abort) {
  for (long long it = 0; it < kBarSpinLimit; ++it) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(b)), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 255) == 255 && *abort) return false;
  }
  return false;
}

// one bulk copy global -> this CTA's shared memory, counted on barrier b;
// dst, src and bytes are multiples of 16
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes,
                                          unsigned long long* b) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(b))
      : "memory");
}

// hint: bring `bytes` at src into L2 ahead of a later bulk copy
__device__ __forceinline__ void l2_prefetch(const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <class T>
__device__ __forceinline__ T warp_inclusive_sum(T v) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(0xffffffffu, v, o);
    if ((int)lane_id() >= o) v += t;
  }
  return v;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <class T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T t = __shfl_xor_sync(0xffffffffu, v, o);
    v = t > v ? t : v;
  }
  return v;
}

// Block-wide exclusive sum over NT threads.  `warp_tmp` holds NT/32 entries.
// Returns the exclusive prefix of the calling thread; *total gets the block sum.
template <int NT, class T>
__device__ __forceinline__ T block_exclusive_sum(T v, T* warp_tmp, T* total) {
  constexpr int NW = NT / 32;
  const int w = threadIdx.x >> 5;
  T inc = warp_inclusive_sum(v);
  if (lane_id() == 31) warp_tmp[w] = inc;
  __syncthreads();
  if (w == 0) {
    T s = (lane_id() < (unsigned)NW) ? warp_tmp[lane_id()] : T(0);
    T si = warp_inclusive_sum(s);
    if (lane_id() < (unsigned)NW) warp_tmp[lane_id()] = si - s;
    if (lane_id() == NW - 1) warp_tmp[NW] = si;
  }
  __syncthreads();
  T ex = warp_tmp[w] + inc - v;
  *total = warp_tmp[NW];
  __syncthreads();
  return ex;
}

// Segmented scan operator on (flag, value): a set flag starts a new segment.
// combine(a, b) with a before b: (a.f | b.f, b.f ? b.v : a.v + b.v).
// Block-wide EXCLUSIVE segmented scan over NT threads; returns the value of
// the segment still open at the calling thread's start (0 for thread 0).
// `tmp_f` / `tmp_v` hold NT/32 + 1 entries.
template <int NT>
__device__ __forceinline__ double block_exclusive_segscan(bool f, double v, int* tmp_f,
                                                         double* tmp_v) {
  constexpr int NW = NT / 32;
  const int w = threadIdx.x >> 5;
  const int lane = (int)lane_id();
  // inclusive within the warp
  int fi = f;
  double vi = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int f2 = __shfl_up_sync(0xffffffffu, fi, o);
    const double v2 = __shfl_up_sync(0xffffffffu, vi, o);
    if (lane >= o) {
      vi = fi ? vi : v2 + vi;
      fi |= f2;
    }
  }
  // exclusive within the warp
  int fe = __shfl_up_sync(0xffffffffu, fi, 1);
  double ve = __shfl_up_sync(0xffffffffu, vi, 1);
  if (lane == 0) { fe = 0; ve = 0.0; }
  if (lane == 31) { tmp_f[w] = fi; tmp_v[w] = vi; }
  __syncthreads();
  if (w == 0) {
    int gf = lane < NW ? tmp_f[lane] : 0;
    double gv = lane < NW ? tmp_v[lane] : 0.0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int f2 = __shfl_up_sync(0xffffffffu, gf, o);
      const double v2 = __shfl_up_sync(0xffffffffu, gv, o);
      if (lane >= o) {
        gv = gf ? gv : v2 + gv;
        gf |= f2;
      }
    }
    // exclusive over warps
    int xf = __shfl_up_sync(0xffffffffu, gf, 1);
    double xv = __shfl_up_sync(0xffffffffu, gv, 1);
    if (lane == 0) { xf = 0; xv = 0.0; }
    if (lane < NW) { tmp_f[lane] = xf; tmp_v[lane] = xv; }
  }
  __syncthreads();
  // prefix of earlier warps, then this warp's exclusive part
  const double wv = tmp_v[w];
  const double res = fe ? ve : wv + ve;
  __syncthreads();
  return res;
}

// Block-wide inclusive max-scan of ints over NT threads.
template <int NT>
__device__ __forceinline__ int block_inclusive_max(int v, int* warp_tmp) {
  constexpr int NW = NT / 32;
  const int w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if ((int)lane_id() >= o) v = max(v, t);
  }
  if (lane_id() == 31) warp_tmp[w] = v;
  __syncthreads();
  if (w == 0) {
    int s = (lane_id() < (unsigned)NW) ? warp_tmp[lane_id()] : INT_MIN;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, s, o);
      if ((int)lane_id() >= o) s = max(s, t);
    }
    if (lane_id() < (unsigned)NW) warp_tmp[lane_id()] = s;
  }
  __syncthreads();
  int carry = (w > 0) ? warp_tmp[w - 1] : INT_MIN;
  __syncthreads();
  return max(v, carry);
}

__device__ __forceinline__ unsigned long long ld_volatile_u64(
    const unsigned long long* p) {
  return *(const volatile unsigned long long*)p;
}
__device__ __forceinline__ void st_volatile_u64(unsigned long long* p,
                                                unsigned long long v) {
  *(volatile unsigned long long*)p = v;
}

// ---------------------------------------------------------------------------
// Decoupled look-back for a single-pass tile scan of 32-bit sums.
//
// Status word (64 bit): [63:34] epoch (30 bits), [33:32] state, [31:0] value.
// state 1 = tile aggregate available, 2 = inclusive prefix available; a word
// whose epoch differs from the launch's epoch reads as "not ready", so the
// status array never needs clearing between launches.  Tiles are handed out in
// launch order through an atomic ticket, so every predecessor of a tile is
// already resident and the look-back always terminates; the wait is still
// bounded and reports kDevErrTimeout instead of hanging.
//
// The epoch lives in device memory (words[1]), not in the launch parameters:
// every tile reads it when its look-back starts, and the launch's last tile to
// publish its prefix (counted in words[2]) advances it for the next launch.
// All tiles of a launch have read the epoch before that last publish, and the
// next launch on the stream starts after this one ends, so each launch sees a
// fresh epoch even when it is a replay of a captured CUDA graph (whose launch
// parameters never change).  words[0..2] start at zero.
// ---------------------------------------------------------------------------
struct LookbackState {
  unsigned long long* status;  // one word per tile
  unsigned* words;             // [0] tile ticket, [1] epoch, [2] tiles published
};

__device__ __forceinline__ unsigned long long lb_pack(unsigned epoch,
                                                      unsigned state,
                                                      unsigned value) {
  return ((unsigned long long)(epoch & 0x3fffffffu) << 34) |
         ((unsigned long long)(state & 3u) << 32) | (unsigned long long)value;
}

// Acquire a tile id (call from all threads; uses one smem word).
__device__ __forceinline__ int lb_acquire_tile(const LookbackState& st,
                                               int ntiles, int* smem_word) {
  if (threadIdx.x == 0) {
    unsigned t = atomicAdd(st.words, 1u);
    // The last tile handed out resets the ticket for the next launch: every
    // other tile already holds its id, and the grid has exactly ntiles CTAs.
    if ((int)t == ntiles - 1) atomicExch(st.words, 0u);
    *smem_word = (int)t;
  }
  __syncthreads();
  int t = *smem_word;
  __syncthreads();
  return t;
}

// lane 0: count this tile's publish; the launch's last one advances the epoch
__device__ __forceinline__ void lb_published(const LookbackState& st, int ntiles) {
  if (atomicAdd(st.words + 2, 1u) == (unsigned)ntiles - 1u) {
    atomicExch(st.words + 2, 0u);
    atomicAdd(st.words + 1, 1u);
  }
}

// Called by warp 0 of every tile (all ntiles of them).  Publishes the tile
// aggregate, looks back over the predecessors and publishes the inclusive
// prefix.  Returns the exclusive prefix of the tile (valid in all lanes of
// warp 0).
//
// Each step reads a window of kLbWindow * 32 predecessors at once (lane l,
// slot q: tile j - 32q - l): when every tile of a launch is in flight, few of
// them have published an inclusive prefix yet, and a look-back that moved 32
// tiles per memory round trip needed up to 16 round trips at 512 tiles; with
// 256 per step it needs at most 2.  A window is accepted once every tile
// nearer than its nearest inclusive prefix has published its aggregate.
constexpr int kLbWindow = 8;
__device__ __forceinline__ unsigned lb_warp_lookback(const LookbackState& st,
                                                     int tile, int ntiles,
                                                     unsigned aggregate,
                                                     int* err) {
  constexpr unsigned FULL = 0xffffffffu;
  const unsigned lane = lane_id();
  unsigned epoch = 0;
  if (lane == 0) epoch = *reinterpret_cast<volatile unsigned*>(st.words + 1);
  epoch = __shfl_sync(FULL, epoch, 0) & 0x3fffffffu;
  if (tile == 0) {
    if (lane == 0) {
      st_volatile_u64(&st.status[0], lb_pack(epoch, 2u, aggregate));
      lb_published(st, ntiles);
    }
    return 0u;
  }
  if (lane == 0) st_volatile_u64(&st.status[tile], lb_pack(epoch, 1u, aggregate));
  unsigned exclusive = 0;
  int j = tile - 1;
  bool timed_out = false;
  while (true) {
    unsigned state[kLbWindow], value[kLbWindow];
    long long spins = 0;
    unsigned sum = 0;
    bool done = false;
    while (true) {
#pragma unroll
      for (int q = 0; q < kLbWindow; ++q) {
        const int idx = j - 32 * q - (int)lane;
        state[q] = 2u;  // before tile 0: an inclusive prefix of 0
        value[q] = 0u;
        if (idx >= 0) {
          const unsigned long long w = ld_volatile_u64(&st.status[idx]);
          state[q] = ((unsigned)(w >> 34) == epoch) ? (unsigned)((w >> 32) & 3u) : 0u;
          value[q] = (unsigned)w;
        }
      }
      // nearest inclusive prefix in the window: slot qf, lane lf
      int qf = kLbWindow, lf = 32;
#pragma unroll
      for (int q = kLbWindow - 1; q >= 0; --q) {
        const unsigned pm = __ballot_sync(FULL, state[q] == 2u);
        if (pm) { qf = q; lf = __ffs(pm) - 1; }
      }
      // every tile nearer than it (or the whole window) must have published
      bool missing = false;
      sum = 0;
#pragma unroll
      for (int q = 0; q < kLbWindow; ++q) {
        const bool in = q < qf || (q == qf && (int)lane <= lf);
        if (in) {
          missing |= state[q] == 0u;
          sum += value[q];
        }
      }
      done = qf < kLbWindow;
      if (!__any_sync(FULL, missing)) break;
      if (++spins > kSpinLimit) { timed_out = true; break; }
      __nanosleep(32);
    }
    if (__any_sync(FULL, timed_out)) {
      if (lane == 0) flag_error(err, kDevErrTimeout);
      exclusive = 0;
      break;
    }
    exclusive += warp_sum(sum);
    if (done) break;
    j -= 32 * kLbWindow;
  }
  if (lane == 0) {
    st_volatile_u64(&st.status[tile], lb_pack(epoch, 2u, exclusive + aggregate));
    lb_published(st, ntiles);
  }
  return exclusive;
}

// ---------------------------------------------------------------------------
// Grid barrier for cooperative launches (all CTAs co-resident).  Bounded: a
// CTA that waits too long records kDevErrTimeout, raises the abort word and
// returns false; callers then leave the kernel.
// ---------------------------------------------------------------------------
struct GridBarrier {
  unsigned* count;
  unsigned* generation;
  int* abort_flag;
};

__device__ __forceinline__ bool grid_sync(const GridBarrier& b, int* err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned gen = *(volatile unsigned*)b.generation;
    __threadfence();
    unsigned arrived = atomicAdd(b.count, 1u);
    if (arrived == gridDim.x - 1) {
      *(volatile unsigned*)b.count = 0u;
      __threadfence();
      atomicAdd(b.generation, 1u);
    } else {
      long long spins = 0;
      while (*(volatile unsigned*)b.generation == gen) {
        if (*(volatile int*)b.abort_flag) { ok = 0; break; }
        if (++spins > kSpinLimit) {
          flag_error(err, kDevErrTimeout);
          atomicExch(b.abort_flag, 1);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    if (*(volatile int*)b.abort_flag) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ---------------------------------------------------------------------------
// Programmatic dependent launch: the grid may start while the grid before it
// on the stream is still running, once that grid has executed
// griddepcontrol.launch_dependents (or exited).  A kernel launched this way
// executes griddepcontrol.wait in every thread before it touches memory that
// an earlier grid on the stream writes, and before it writes memory that an
// earlier grid reads; and it executes launch_dependents only after that wait,
// so that whatever it lets start finds every earlier grid complete.
// ---------------------------------------------------------------------------
template <class... KArgs, class... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// ---------------------------------------------------------------------------
// Launch with an L2 access-policy window: the window [base, base + bytes) is
// marked persisting for this launch only (no stream state changes), so a
// small gathered operand (the dense x, a frontier bitmap) stays in L2 while
// the streamed matrix passes through it.  bytes == 0 launches plainly; the
// window is off unless SPMX_L2_WINDOW is set to a non-zero value.
// ---------------------------------------------------------------------------
size_t l2_window_bytes(const void* base, size_t bytes);  // clamp; 0 = disabled

template <class... KArgs, class... Args>
cudaError_t launch_l2_window(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                             cudaStream_t st, const void* win_base, size_t win_bytes,
                             Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  const size_t wb = win_base ? l2_window_bytes(win_base, win_bytes) : 0;
  if (wb) {
    attr[0].id = cudaLaunchAttributeAccessPolicyWindow;
    attr[0].val.accessPolicyWindow.base_ptr = const_cast<void*>(win_base);
    attr[0].val.accessPolicyWindow.num_bytes = wb;
    attr[0].val.accessPolicyWindow.hitRatio = 1.0f;
    attr[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    attr[0].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace spmx
