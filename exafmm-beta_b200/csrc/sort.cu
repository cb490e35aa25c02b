// Stable LSD radix sort (digits of 8 to 10 bits) of key/value pairs, and the scan work
// buffers.  Each pass: per-tile digit histograms, one device-wide scan of the
// digit-major count table, then a stable scatter in which every warp ranks its
// own contiguous chunk with __match_any_sync and the warps of a tile are ordered
// by a shared prefix table.
#include <algorithm>

#include "engine.h"

namespace exafmm_b200 {

ScanScratch ScanWork::prepare(cudaStream_t st, int *err, long long tiles, size_t elem) {
  if (!zeroed || ctrl.cap < 2) {
    ctrl.ensure(2);
    EXA_CUDA(cudaMemsetAsync(ctrl.p, 0, 2 * sizeof(unsigned), st));
    zeroed = true;
  }
  if ((long long)flags.cap < tiles) {
    flags.ensure(tiles);
    EXA_CUDA(cudaMemsetAsync(flags.p, 0, flags.cap * sizeof(unsigned), st));
  }
  aggs.ensure(tiles * elem);
  incl.ensure(tiles * elem);
  epoch = (epoch + 1) & 0x3fffffffu;
  if (epoch == 0) {
    EXA_CUDA(cudaMemsetAsync(flags.p, 0, flags.cap * sizeof(unsigned), st));
    epoch = 1;
  }
  ScanScratch s;
  s.ticket = ctrl.p;
  s.done = ctrl.p + 1;
  s.flags = flags.p;
  s.aggregates = aggs.p;
  s.inclusive = incl.p;
  s.error = err;
  s.max_tiles = (long long)flags.cap;
  return s;
}

namespace {

constexpr int kSortWarps = 8;
constexpr int kSortItems = 16;
constexpr int kSortThreads = kSortWarps * 32;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 items per tile

// BUCKETS = 2^BITS digit values; a pass uses the low `width` bits of
// key >> shift (width <= BITS).
template <typename K, int BITS>
__global__ void __launch_bounds__(kSortThreads)
radix_hist(const K *keys, long long n, int shift, unsigned mask, unsigned *counts, int ntiles) {
  constexpr int B = 1 << BITS;
  __shared__ unsigned h[B];
  for (int i = threadIdx.x; i < B; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * kSortTile;
  for (int k = threadIdx.x; k < kSortTile; k += blockDim.x) {
    long long i = base + k;
    if (i < n) atomicAdd(&h[(unsigned)(keys[i] >> shift) & mask], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < B; d += blockDim.x) counts[(long long)d * ntiles + blockIdx.x] = h[d];
}

// Exclusive scan of the digit-major count table, in place.
struct CountScan {
  using T = int;
  unsigned *counts;
  __device__ T value(long long i) const { return (int)counts[i]; }
  __device__ void emit(long long i, const T &, const T &excl) const { counts[i] = (unsigned)excl; }
  __device__ void total(const T &) const {}
};

template <typename K, int BITS>
__global__ void __launch_bounds__(kSortThreads)
radix_scatter(const K *keys_in, const int *vals_in, K *keys_out, int *vals_out, long long n, int shift,
              unsigned mask, const unsigned *offsets, int ntiles) {
  constexpr int B = 1 << BITS;
  __shared__ unsigned wcnt[kSortWarps][B];
  __shared__ unsigned toff[B];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kSortWarps * B; i += blockDim.x) (&wcnt[0][0])[i] = 0;
  for (int d = threadIdx.x; d < B; d += blockDim.x) toff[d] = offsets[(long long)d * ntiles + blockIdx.x];
  __syncthreads();
  const long long base = (long long)blockIdx.x * kSortTile + warp * (32 * kSortItems);
  K key[kSortItems];
  int val[kSortItems];
  unsigned rank[kSortItems];
  const unsigned lt_mask = (1u << lane) - 1u;
#pragma unroll
  for (int it = 0; it < kSortItems; it++) {
    const long long i = base + it * 32 + lane;
    const bool valid = i < n;
    key[it] = valid ? keys_in[i] : K(0);
    val[it] = valid ? vals_in[i] : 0;
    const unsigned dig = valid ? ((unsigned)(key[it] >> shift) & mask) : (unsigned)B;
    const unsigned peers = __match_any_sync(0xffffffffu, dig);
    const unsigned r = __popc(peers & lt_mask);
    unsigned b = valid ? wcnt[warp][dig] : 0u;
    __syncwarp();
    if (valid && (peers & lt_mask) == 0) wcnt[warp][dig] = b + __popc(peers);
    __syncwarp();
    rank[it] = b + r;
  }
  __syncthreads();
  // Exclusive prefix over warps, per digit.
  for (int d = threadIdx.x; d < B; d += blockDim.x) {
    unsigned run = 0;
    for (int w = 0; w < kSortWarps; w++) {
      unsigned c = wcnt[w][d];
      wcnt[w][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < kSortItems; it++) {
    const long long i = base + it * 32 + lane;
    if (i < n) {
      const unsigned dig = (unsigned)(key[it] >> shift) & mask;
      const unsigned pos = toff[dig] + wcnt[warp][dig] + rank[it];
      keys_out[pos] = key[it];
      vals_out[pos] = val[it];
    }
  }
}

template <typename K, int BITS>
void radix_pass(const K *kin, const int *vin, K *kout, int *vout, long long n, int shift, int width, int ntiles,
                SortWork &w, int *err, cudaStream_t st) {
  const unsigned mask = (1u << width) - 1u;
  radix_hist<K, BITS><<<ntiles, kSortThreads, 0, st>>>(kin, n, shift, mask, w.counts.p, ntiles);
  EXA_CHECK_LAUNCH();
  CountScan cs{w.counts.p};
  const long long cells = (long long)(1 << BITS) * ntiles;
  launch_scan<256, 8>(cs, nullptr, cells, cells, w.scan, err, st);
  radix_scatter<K, BITS><<<ntiles, kSortThreads, 0, st>>>(kin, vin, kout, vout, n, shift, mask, w.counts.p, ntiles);
  EXA_CHECK_LAUNCH();
}

// Byte passes, or passes of up to 10 bits where that saves at least a quarter
// of them (17-bit cell ids: 2 passes instead of 3); a wider pass costs more
// (a 4x larger count table to scan, more scattered writes), so 63-bit octree
// keys keep their 8 byte passes.
template <typename K>
bool radix_sort_impl(K *keys, int *vals, K *keys_alt, int *vals_alt, long long n, int begin_bit, int end_bit,
                     SortWork &w, int *err, cudaStream_t st) {
  if (n <= 1 || end_bit <= begin_bit) return false;
  const int ntiles = div_up(n, kSortTile);
  const int range = end_bit - begin_bit;
  const int p8 = (range + 7) / 8, p10 = (range + 9) / 10;
  const int passes = 4 * p10 <= 3 * p8 ? p10 : p8;
  const int bits = (range + passes - 1) / passes;
  w.counts.ensure((size_t)(bits > 8 ? 1024 : 256) * ntiles);
  K *kin = keys, *kout = keys_alt;
  int *vin = vals, *vout = vals_alt;
  bool in_alt = false;
  for (int shift = begin_bit; shift < end_bit; shift += bits) {
    const int width = std::min(bits, end_bit - shift);
    if (width > 8) radix_pass<K, 10>(kin, vin, kout, vout, n, shift, width, ntiles, w, err, st);
    else radix_pass<K, 8>(kin, vin, kout, vout, n, shift, width, ntiles, w, err, st);
    K *tk = kin; kin = kout; kout = tk;
    int *tv = vin; vin = vout; vout = tv;
    in_alt = !in_alt;
  }
  return in_alt;
}

}  // namespace

bool radix_sort_u64(uint64_t *keys, int *vals, uint64_t *keys_alt, int *vals_alt, long long n, int begin_bit,
                    int end_bit, SortWork &w, int *err, cudaStream_t st) {
  return radix_sort_impl<unsigned long long>((unsigned long long *)keys, vals, (unsigned long long *)keys_alt,
                                             vals_alt, n, begin_bit, end_bit, w, err, st);
}

bool radix_sort_u32(uint32_t *keys, int *vals, uint32_t *keys_alt, int *vals_alt, long long n, int begin_bit,
                    int end_bit, SortWork &w, int *err, cudaStream_t st) {
  return radix_sort_impl<unsigned>((unsigned *)keys, vals, (unsigned *)keys_alt, vals_alt, n, begin_bit, end_bit,
                                   w, err, st);
}

}  // namespace exafmm_b200
