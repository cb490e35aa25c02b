// Stable LSD radix sort (digits of 8 to 10 bits) of key/value pairs, and the scan work
// buffers.  Each pass: per-tile digit histograms, one device-wide scan of the
// digit-major count table, then a stable scatter in which every warp ranks its
// own contiguous chunk with __match_any_sync, the warps of a tile are ordered
// by a shared prefix table, and the tile is written out through shared memory
// in digit order (coalesced bucket runs).
#include <algorithm>
#include <atomic>

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

// Shared memory of one scatter tile: the tile's keys and values in digit
// order, per-warp digit counts, the tile's global offsets and its digit starts.
template <typename K, int BITS>
constexpr size_t scatter_smem_bytes() {
  return (size_t)kSortTile * (sizeof(K) + sizeof(int)) + (size_t)(kSortWarps + 2) * (1 << BITS) * sizeof(unsigned);
}

// Stable scatter of one tile.  Items are ranked within their warp's chunk
// (__match_any_sync) and across warps, placed in shared memory in digit order,
// then written out bucket run by bucket run, so consecutive threads store to
// consecutive addresses of a bucket instead of each lane to a different one.
template <typename K, int BITS>
__global__ void __launch_bounds__(kSortThreads)
radix_scatter(const K *keys_in, const int *vals_in, K *keys_out, int *vals_out, long long n, int shift,
              unsigned mask, const unsigned *offsets, int ntiles) {
  constexpr int B = 1 << BITS;
  constexpr int PER = (B + kSortThreads - 1) / kSortThreads;  // digits per thread in the tile scan
  extern __shared__ __align__(16) unsigned char sort_smem[];
  K *skey = reinterpret_cast<K *>(sort_smem);
  int *sval = reinterpret_cast<int *>(skey + kSortTile);
  unsigned (*wcnt)[B] = reinterpret_cast<unsigned (*)[B]>(sval + kSortTile);
  unsigned *toff = &wcnt[kSortWarps][0];  // global start of each digit's run of this tile
  unsigned *tstart = toff + B;            // start of each digit within the tile
  __shared__ unsigned wsum[kSortWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kSortWarps * B; i += blockDim.x) (&wcnt[0][0])[i] = 0;
  for (int d = threadIdx.x; d < B; d += blockDim.x) toff[d] = offsets[(long long)d * ntiles + blockIdx.x];
  __syncthreads();
  const long long tile0 = (long long)blockIdx.x * kSortTile;
  const long long base = tile0 + warp * (32 * kSortItems);
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
  // Exclusive prefix over warps, per digit; the digit's tile total goes to tstart.
  for (int d = threadIdx.x; d < B; d += blockDim.x) {
    unsigned run = 0;
    for (int w = 0; w < kSortWarps; w++) {
      unsigned c = wcnt[w][d];
      wcnt[w][d] = run;
      run += c;
    }
    tstart[d] = run;
  }
  __syncthreads();
  // Exclusive scan of the digit totals over the tile: PER consecutive digits a thread.
  {
    unsigned v[PER], sum = 0;
#pragma unroll
    for (int k = 0; k < PER; k++) {
      const int d = threadIdx.x * PER + k;
      v[k] = d < B ? tstart[d] : 0u;
      sum += v[k];
    }
    unsigned incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    unsigned before = incl - sum;
    for (int w = 0; w < warp; w++) before += wsum[w];
#pragma unroll
    for (int k = 0; k < PER; k++) {
      const int d = threadIdx.x * PER + k;
      if (d < B) tstart[d] = before;
      before += v[k];
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < kSortItems; it++) {
    const long long i = base + it * 32 + lane;
    if (i < n) {
      const unsigned dig = (unsigned)(key[it] >> shift) & mask;
      const unsigned loc = tstart[dig] + wcnt[warp][dig] + rank[it];
      skey[loc] = key[it];
      sval[loc] = val[it];
    }
  }
  __syncthreads();
  const int tile_n = (int)min((long long)kSortTile, n - tile0);
  for (int j = threadIdx.x; j < tile_n; j += blockDim.x) {
    const K k = skey[j];
    const unsigned dig = (unsigned)(k >> shift) & mask;
    const unsigned pos = toff[dig] + (unsigned)j - tstart[dig];
    keys_out[pos] = k;
    vals_out[pos] = sval[j];
  }
}

// The scatter's shared-memory opt-in, once per device and kernel: the call
// is a driver round trip that solving threads would otherwise make on every
// pass.
template <typename K, int BITS>
void scatter_smem_optin() {
  static std::atomic<unsigned long long> done{0};
  int dev = 0;
  EXA_CUDA(cudaGetDevice(&dev));
  const unsigned long long bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return;
  EXA_CUDA(cudaFuncSetAttribute(radix_scatter<K, BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)scatter_smem_bytes<K, BITS>()));
  done.fetch_or(bit, std::memory_order_release);
}

template <typename K, int BITS>
void radix_pass(const K *kin, const int *vin, K *kout, int *vout, long long n, int shift, int width, int ntiles,
                SortWork &w, int *err, cudaStream_t st) {
  const unsigned mask = (1u << width) - 1u;
  radix_hist<K, BITS><<<ntiles, kSortThreads, 0, st>>>(kin, n, shift, mask, w.counts.p, ntiles);
  EXA_CHECK_LAUNCH();
  CountScan cs{w.counts.p};
  const long long cells = (long long)(1 << BITS) * ntiles;
  launch_scan<1024, 8>(cs, nullptr, cells, cells, w.scan, err, st);
  constexpr size_t smem = scatter_smem_bytes<K, BITS>();
  scatter_smem_optin<K, BITS>();
  radix_scatter<K, BITS><<<ntiles, kSortThreads, smem, st>>>(kin, vin, kout, vout, n, shift, mask, w.counts.p,
                                                             ntiles);
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
    if (width > 9) radix_pass<K, 10>(kin, vin, kout, vout, n, shift, width, ntiles, w, err, st);
    else if (width > 8) radix_pass<K, 9>(kin, vin, kout, vout, n, shift, width, ntiles, w, err, st);
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
