// Internal host-side interfaces of the engine (not part of the C ABI).
#pragma once
#include <algorithm>
#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>

#include "common.cuh"
#include "scan.cuh"

namespace exafmm_b200 {

// Grow-only device buffer.  Contents are not preserved across growth.
// Device bytes held by the context whose entry point is running on this
// thread (null outside such a call): grow-only buffers charge it.
extern thread_local long long *g_dbuf_account;
// That context's stream: buffers are allocated and freed in its order
// (cudaMallocAsync / cudaFreeAsync), so a context that grows does not stall
// the device for the others, as cudaFree would.
extern thread_local cudaStream_t g_dbuf_stream;

template <typename T>
struct DBuf {
  T *p = nullptr;
  size_t cap = 0;
  long long *acct = nullptr;  // byte counter of the owning context, set at allocation
  cudaStream_t st = nullptr;  // stream of a stream-ordered allocation (else plain cudaMalloc)
  void ensure(size_t n) {
    if (n <= cap) return;
    release();
    size_t want = n < 16 ? 16 : n;
    st = g_dbuf_stream;
    if (st) EXA_CUDA(cudaMallocAsync((void **)&p, want * sizeof(T), st));
    else EXA_CUDA(cudaMalloc((void **)&p, want * sizeof(T)));
    cap = want;
    acct = g_dbuf_account;
    if (acct) *acct += (long long)(want * sizeof(T));
  }
  void release() {
    if (p) {
      if (st) cudaFreeAsync(p, st);
      else cudaFree(p);
      if (acct) *acct -= (long long)(cap * sizeof(T));
    }
    p = nullptr;
    cap = 0;
    acct = nullptr;
    st = nullptr;
  }
  T *get() const { return p; }
  ~DBuf() { release(); }
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
};

// Reusable state for scan_kernel launches on one stream.
struct ScanWork {
  DBuf<unsigned> ctrl;       // [0] ticket, [1] done
  DBuf<unsigned> flags;
  DBuf<unsigned char> aggs, incl;
  unsigned epoch = 0;
  bool zeroed = false;
  ScanScratch prepare(cudaStream_t st, int *err, long long tiles, size_t elem);
};

// Launch a scan over n items (n_dev may be null, then n_host is used).
// Every scan of the engine runs tiles of 1024 threads x 8 items: against 256
// x 8 (or 256 x 4) that took a 4M-body solve from 37.0 to 35.5 ms (traversal
// sweeps, tree levels, sort counts and the class-product bookkeeping), with
// the same results.
template <int BLOCK, int ITEMS, typename Producer>
void launch_scan(const Producer &prod, const long long *n_dev, long long n_host, long long max_items,
                 ScanWork &w, int *err, cudaStream_t st) {
  constexpr int TILE = BLOCK * ITEMS;
  long long tiles = (max_items + TILE - 1) / TILE + 1;
  ScanScratch s = w.prepare(st, err, tiles, sizeof(typename Producer::T));
  // as many blocks as an SM holds by threads (at most 16), so that tiles
  // waiting on their look-back overlap with others' work; but no more than
  // the most items the scan can see need (the count on the device is at most
  // max_items), so small scans do not occupy the whole GPU
  int grid = kNumSMs * std::min(16, 2048 / BLOCK);
  const long long bound = n_dev ? max_items : n_host;
  const long long need = (bound + TILE - 1) / TILE;
  if (need < grid) grid = need > 0 ? (int)need : 1;
  scan_kernel<BLOCK, ITEMS, Producer><<<grid, BLOCK, 0, st>>>(prod, n_dev, n_host, s, w.epoch);
  EXA_CHECK_LAUNCH();
}

// Stable LSD radix sort of (key, value) pairs over bits [begin_bit, end_bit).
// Returns true when the sorted data ended up in the *_alt buffers.
struct SortWork {
  DBuf<unsigned> counts;
  ScanWork scan;
};
bool radix_sort_u64(uint64_t *keys, int *vals, uint64_t *keys_alt, int *vals_alt, long long n,
                    int begin_bit, int end_bit, SortWork &w, int *err, cudaStream_t st);
bool radix_sort_u32(uint32_t *keys, int *vals, uint32_t *keys_alt, int *vals_alt, long long n,
                    int begin_bit, int end_bit, SortWork &w, int *err, cudaStream_t st);

}  // namespace exafmm_b200
