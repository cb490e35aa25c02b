// Single-pass device-wide scan with decoupled look-back, over a length held in
// device memory.  Tiles are claimed through an atomic ticket, so a tile only
// ever waits on tiles whose blocks are already running, and every wait is
// bounded: a wait that runs out raises an error flag and the block carries on.
//
// A "Producer" supplies per-item values and consumes the exclusive prefix:
//   struct Producer {
//     using T = ...;                                    // value type with operator+
//     __device__ T value(long long i) const;            // i < n
//     __device__ void emit(long long i, const T& v, const T& excl) const;
//     __device__ void total(const T& t) const;          // called once, with the grand total
//   };
#pragma once
#include "common.cuh"

namespace exafmm_b200 {

struct ScanScratch {
  unsigned *ticket;          // tile ticket, reset by the last block out
  unsigned *done;            // blocks finished, reset by the last block out
  unsigned *flags;           // per tile: (epoch << 2) | state, state 1 = aggregate, 2 = inclusive
  void *aggregates;          // per tile T
  void *inclusive;           // per tile T
  int *error;                // device error word
  long long max_tiles;
};

// Shuffle helpers for the value types used with the scan.
__device__ __forceinline__ int shfl_up_any(int v, int o) { return __shfl_up_sync(0xffffffffu, v, o); }
__device__ __forceinline__ unsigned long long shfl_up_any(unsigned long long v, int o) {
  return __shfl_up_sync(0xffffffffu, v, o);
}
__device__ __forceinline__ int shfl_any(int v, int src) { return __shfl_sync(0xffffffffu, v, src); }
__device__ __forceinline__ unsigned long long shfl_any(unsigned long long v, int src) {
  return __shfl_sync(0xffffffffu, v, src);
}

struct Count2 {
  unsigned long long a, b;
  __host__ __device__ Count2 operator+(const Count2 &o) const { return {a + o.a, b + o.b}; }
};
__device__ __forceinline__ Count2 shfl_up_any(Count2 v, int o) {
  return {__shfl_up_sync(0xffffffffu, v.a, o), __shfl_up_sync(0xffffffffu, v.b, o)};
}
__device__ __forceinline__ Count2 shfl_any(Count2 v, int src) {
  return {__shfl_sync(0xffffffffu, v.a, src), __shfl_sync(0xffffffffu, v.b, src)};
}

template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T u = shfl_up_any(v, o);
    if (lane >= o) v = v + u;
  }
  return v;
}

template <typename T> __device__ __forceinline__ T zero_value() { return T{}; }

// A value another block published: read from L2 (ld.global.cg), never from
// a line this SM's L1 may hold from before it was written.
template <typename T>
__device__ __forceinline__ T load_cg(const T *p) {
  static_assert(sizeof(T) % 4 == 0, "whole 32-bit words");
  T v;
  unsigned *d = reinterpret_cast<unsigned *>(&v);
  const unsigned *src = reinterpret_cast<const unsigned *>(p);
#pragma unroll
  for (int i = 0; i < (int)(sizeof(T) / 4); i++) d[i] = __ldcg(src + i);
  return v;
}

// Bounded spin: about a second of polling before giving up.
constexpr unsigned kSpinLimit = 1u << 22;

template <int BLOCK, int ITEMS, typename Producer>
__global__ void __launch_bounds__(BLOCK)
scan_kernel(Producer prod, const long long *n_ptr, long long n_const, ScanScratch s, unsigned epoch) {
  using T = typename Producer::T;
  constexpr int TILE = BLOCK * ITEMS;
  constexpr int WARPS = BLOCK / 32;
  __shared__ T warp_tot[WARPS];
  __shared__ T tile_excl;
  __shared__ long long tile_id;
  const long long n = n_ptr ? *n_ptr : n_const;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T *aggs = (T *)s.aggregates;
  T *incl = (T *)s.inclusive;
  volatile unsigned *flags = s.flags;
  if (n == 0 && blockIdx.x == 0 && threadIdx.x == 0) prod.total(zero_value<T>());
  while (true) {
    if (threadIdx.x == 0) tile_id = atomicAdd(s.ticket, 1u);
    __syncthreads();
    const long long t = tile_id;
    if (t * TILE >= n) break;
    if (t >= s.max_tiles) {
      if (threadIdx.x == 0) atomicOr(s.error, 32);
      break;
    }
    // Per-thread values (blocked arrangement: thread owns ITEMS consecutive items).
    T v[ITEMS];
    T run = zero_value<T>();
    const long long base = t * TILE + (long long)threadIdx.x * ITEMS;
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
      long long i = base + k;
      v[k] = (i < n) ? prod.value(i) : zero_value<T>();
      run = run + v[k];
    }
    T winc = warp_inclusive_scan(run);
    if (lane == 31) warp_tot[warp] = winc;
    __syncthreads();
    T wexcl = zero_value<T>(), agg = zero_value<T>();
    for (int w = 0; w < WARPS; w++) {
      if (w < warp) wexcl = wexcl + warp_tot[w];
      agg = agg + warp_tot[w];
    }
    T thread_excl = wexcl + shfl_up_any(winc, 1);
    if (lane == 0) thread_excl = wexcl;
    if (warp == 0) {
      // Look-back by the whole warp: lane l reads the flag of tile p - l, so
      // 32 predecessors are examined per round trip to memory.  Once every
      // tile of the window has published something, the lanes up to the
      // nearest inclusive prefix add their values (aggregates, or that
      // inclusive prefix); with no inclusive prefix in the window, the next
      // 32 tiles follow.  The values are integer counts, so the order of the
      // additions does not matter.
      T excl = zero_value<T>();
      if (t == 0) {
        if (lane == 0) {
          incl[0] = agg;
          __threadfence();
          flags[0] = (epoch << 2) | 2u;
        }
      } else {
        if (lane == 0) {
          aggs[t] = agg;
          __threadfence();
          flags[t] = (epoch << 2) | 1u;
        }
        long long p = t - 1;
        unsigned spins = 0;
        bool failed = false;
        while (true) {
          const long long q = p - lane;
          unsigned f = 0;
          while (true) {
            f = q >= 0 ? flags[q] : 0u;
            const bool ready = q < 0 || ((f >> 2) == epoch && (f & 3u) != 0);
            if (__all_sync(0xffffffffu, ready)) break;
            if (++spins > kSpinLimit) {
              failed = true;
              break;
            }
            if (spins > 64) __nanosleep(64);  // short waits poll at full rate
          }
          if (failed) {
            if (lane == 0) atomicOr(s.error, 16);
            break;
          }
          __threadfence();
          const unsigned inc = __ballot_sync(0xffffffffu, q >= 0 && (f & 3u) == 2u);
          const int stop = inc ? __ffs((int)inc) - 1 : 31;
          T v = zero_value<T>();
          if (q >= 0 && lane <= stop) v = (f & 3u) == 2u ? load_cg(incl + q) : load_cg(aggs + q);
          v = warp_inclusive_scan(v);
          excl = excl + shfl_any(v, 31);
          if (inc || p < 32) break;  // an inclusive prefix, or tile 0 reached
          p -= 32;
        }
        if (lane == 0) {
          incl[t] = excl + agg;
          __threadfence();
          flags[t] = (epoch << 2) | 2u;
        }
      }
      if (lane == 0) {
        tile_excl = excl;
        if ((t + 1) * TILE >= n) prod.total(excl + agg);
      }
    }
    __syncthreads();
    T acc = tile_excl + thread_excl;
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
      long long i = base + k;
      if (i < n) prod.emit(i, v[k], acc);
      acc = acc + v[k];
    }
    __syncthreads();
  }
  // The last block out resets the ticket for the next launch on this scratch.
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned d = atomicAdd(s.done, 1u);
    if (d == gridDim.x - 1) {
      *s.ticket = 0;
      *s.done = 0;
      __threadfence();
    }
  }
}

}  // namespace exafmm_b200
