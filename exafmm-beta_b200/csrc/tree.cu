// Device octree, bit-exact with BuildTree (include/build_tree.h).
//
// The reference builds top-down: at every node it compares each body with the
// node's FP64 center and stably partitions the node's bodies by octant, with
// child centers X +- R0/2^(level+1) (build_tree.h:29-108).  Here each body
// follows its own path through that same center recurrence (identical FP64
// adds, so identical comparisons) and records one 3-bit octant digit per level
// in a 63-bit key.  A stable radix sort of the keys groups every node's bodies
// contiguously in the reference's octant order; the levels are then expanded
// breadth first by binary search on the digit of each level, and the cell
// table is laid out exactly as nodes2cells does (build_tree.h:123-165).  Inside
// a leaf the reference keeps input order (its partitions are stable), so a final
// per-leaf sort restores ascending input index there.
#include <algorithm>
#include <cstring>

#include "context.h"
#include "drift.cuh"

namespace exafmm_b200 {
namespace {

__device__ __forceinline__ unsigned long long order_enc(double d) {
  unsigned long long u = (unsigned long long)__double_as_longlong(d);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__host__ __device__ __forceinline__ double order_dec(unsigned long long u) {
  unsigned long long v = (u >> 63) ? (u ^ 0x8000000000000000ull) : ~u;
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)v);
#else
  double d;
  memcpy(&d, &v, 8);
  return d;
#endif
}

__global__ void k_bounds_init(unsigned long long *enc) {
  int t = threadIdx.x;
  if (t < 3 || (t >= 6 && t < 9)) enc[t] = ~0ull;  // running minima (exact, estimate)
  else if (t < 13) enc[t] = 0ull;                 // running maxima, max |x|
}

// BoundBox::getBounds in closed form: each body contributes g^(N-1-j)(X_j) to
// the min and the mirrored drift to the max; body 0 also carries the initial
// value, which is drifted N times.  Two passes: the unrounded estimate x_j -/+ k_j * 1e-5 is
// within k * ulp(max|x| + N * 1e-5) of the exact drifted value, so only bodies
// whose estimate lies within twice that of the extreme estimate can hold the
// exact extreme; only those evaluate the closed form.
// enc[0..5]: exact result, enc[6..11]: estimates, enc[12]: max |x| over all coordinates.
// With init6 (BoundBox::getBounds(bodies, bounds), bound_box.h:28-36) the
// running bounds start from init6 instead of the first body: every body then
// drifts n - 1 - j times and init6 itself n times.
__global__ void k_bounds_estimate(const double4 *x, long long n, unsigned long long *enc, const double *init6) {
  unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0, 0, 0}, amax = 0;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
    const double4 b = x[j];
    const double v[3] = {b.x, b.y, b.z};
    const double kc = (double)((j == 0 && !init6) ? n : n - 1 - j) * 1e-5;
    for (int d = 0; d < 3; d++) {
      const unsigned long long a = order_enc(v[d] - kc), c = order_enc(v[d] + kc);
      lo[d] = a < lo[d] ? a : lo[d];
      hi[d] = c > hi[d] ? c : hi[d];
      const unsigned long long ab = order_enc(fabs(v[d]));
      amax = ab > amax ? ab : amax;
    }
  }
  if (init6 && blockIdx.x == 0 && threadIdx.x == 0) {
    const double kc = (double)n * 1e-5;
    for (int d = 0; d < 3; d++) {
      const unsigned long long a = order_enc(init6[d] - kc), c = order_enc(init6[3 + d] + kc);
      lo[d] = a < lo[d] ? a : lo[d];
      hi[d] = c > hi[d] ? c : hi[d];
      const unsigned long long a1 = order_enc(fabs(init6[d])), a2 = order_enc(fabs(init6[3 + d]));
      amax = a1 > amax ? a1 : amax;
      amax = a2 > amax ? a2 : amax;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    for (int d = 0; d < 3; d++) {
      const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo[d], o);
      const unsigned long long c = __shfl_xor_sync(0xffffffffu, hi[d], o);
      lo[d] = a < lo[d] ? a : lo[d];
      hi[d] = c > hi[d] ? c : hi[d];
    }
    const unsigned long long m = __shfl_xor_sync(0xffffffffu, amax, o);
    amax = m > amax ? m : amax;
  }
  if ((threadIdx.x & 31) == 0) {
    for (int d = 0; d < 3; d++) {
      atomicMin(&enc[6 + d], lo[d]);
      atomicMax(&enc[9 + d], hi[d]);
    }
    atomicMax(&enc[12], amax);
  }
}

__global__ void k_bounds_exact(const double4 *x, long long n, unsigned long long *enc, const double *init6) {
  const double span = order_dec(enc[12]) + (double)n * 1e-5;
  const double B = (double)n * ldexp(1.0, ilogb(span > 1e-300 ? span : 1e-300) - 52) + 1e-300;
  double elo[3], ehi[3];
  for (int d = 0; d < 3; d++) {
    elo[d] = order_dec(enc[6 + d]) + 2.0 * B;
    ehi[d] = order_dec(enc[9 + d]) - 2.0 * B;
  }
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
    const double4 b = x[j];
    const double v[3] = {b.x, b.y, b.z};
    const long long k = (j == 0 && !init6) ? n : n - 1 - j;
    const double kc = (double)k * 1e-5;
    for (int d = 0; d < 3; d++) {
      if (v[d] - kc <= elo[d]) atomicMin(&enc[d], order_enc(drift_down(v[d], k)));
      if (v[d] + kc >= ehi[d]) atomicMax(&enc[3 + d], order_enc(drift_up(v[d], k)));
    }
  }
  if (init6 && blockIdx.x == 0 && threadIdx.x == 0) {
    const double kc = (double)n * 1e-5;
    for (int d = 0; d < 3; d++) {
      if (init6[d] - kc <= elo[d]) atomicMin(&enc[d], order_enc(drift_down(init6[d], n)));
      if (init6[3 + d] + kc >= ehi[d]) atomicMax(&enc[3 + d], order_enc(drift_up(init6[3 + d], n)));
    }
  }
}

__global__ void k_bounds_final(const unsigned long long *enc, long long n, double *bounds) {
  int t = threadIdx.x;
  if (t < 6) bounds[t] = (n > 0) ? order_dec(enc[t]) : 0.0;
}

// bounds2box (build_tree.h:168-180): center, then half-width scaled by 1.00001.
__device__ __forceinline__ double4 box_of(const double *bounds) {
  double R = 0;
  double X[3];
  for (int d = 0; d < 3; d++) X[d] = (bounds[3 + d] + bounds[d]) / 2;
  for (int d = 0; d < 3; d++) {
    double a = X[d] - bounds[d];
    R = (R < a) ? a : R;
    double b = bounds[3 + d] - X[d];
    R = (R < b) ? b : R;
  }
  return make_double4(X[0], X[1], X[2], __dmul_rn(R, 1.00001));
}

__global__ void k_box(const double *bounds, double *box) {
  if (threadIdx.x != 0) return;
  const double4 b = box_of(bounds);
  box[0] = b.x;
  box[1] = b.y;
  box[2] = b.z;
  box[3] = b.w;
}

__device__ __forceinline__ double level_half(double R0, int level) {
  // R0 / (1 << (level + 1)): an exact power-of-two scaling, as in build_tree.h:97.
  return R0 / (double)(1 << (level + 1));
}

// One octant digit per level from the reference's center recurrence.
__device__ __forceinline__ unsigned long long octant_key(const double4 b, double cx, double cy, double cz, double R0) {
  unsigned long long key = 0;
#pragma unroll 1
  for (int l = 0; l < kMaxLevels; l++) {
    const int ox = b.x > cx, oy = b.y > cy, oz = b.z > cz;
    key = (key << 3) | (unsigned long long)(ox | (oy << 1) | (oz << 2));
    const double r = level_half(R0, l);
    cx = __dadd_rn(cx, r * (ox ? 1.0 : -1.0));
    cy = __dadd_rn(cy, r * (oy ? 1.0 : -1.0));
    cz = __dadd_rn(cz, r * (oz ? 1.0 : -1.0));
  }
  return key;
}

__global__ void k_keys(const double4 *x, long long n, const double *box, unsigned long long *keys, int *vals) {
  const double R0 = box[3];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    keys[i] = octant_key(x[i], box[0], box[1], box[2], R0);
    vals[i] = (int)i;
  }
}

// The deepest level whose nodes split, from the sorted keys alone: bodies i
// and i + ncrit lie in one node of level l exactly when their keys share the
// digits of levels 0..l-1 (and, in a forest, their system), and that node then
// holds more than ncrit bodies; so the deepest splitting level is the largest
// number of shared leading digits over i (kMaxLevels when the keys are equal).
// sys_off (a forest, else null) places each body's caller index in its system.
__device__ __forceinline__ int system_of(const long long *sys_off, int nsys, long long i) {
  int lo = 0, hi = nsys - 1;  // last s with sys_off[s] <= i
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (sys_off[mid] <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void k_split_level(const unsigned long long *keys, const int *perm, long long n, int ncrit,
                              const long long *sys_off, int nsys, int *out) {
  int best = -1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i + ncrit < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (sys_off && system_of(sys_off, nsys, perm[i]) != system_of(sys_off, nsys, perm[i + ncrit])) continue;
    const unsigned long long x = keys[i] ^ keys[i + ncrit];
    const int shared = x == 0 ? kMaxLevels : kMaxLevels - 1 - (63 - __clzll((long long)x)) / 3;
    best = max(best, shared);
  }
  for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0 && best >= 0) atomicMax(out, best);
}

__global__ void k_tree_root(long long n, long long *lvl, int *nd_begin, int *nd_count, double4 *nd_x,
                            const double *box, int *nd_cell, int *nd_pcell, int *nd_ichild) {
  if (threadIdx.x != 0) return;
  for (int l = 0; l <= kMaxLevels; l++) {
    lvl[l] = 0;
    lvl[kMaxLevels + 1 + l] = 0;
  }
  if (n > 0) {
    lvl[0] = 1;
    nd_begin[0] = 0;
    nd_count[0] = (int)n;
    nd_x[0] = make_double4(box[0], box[1], box[2], 0.0);
    nd_cell[0] = 0;
    nd_pcell[0] = 0;
    nd_ichild[0] = 1;
  }
}

__device__ __forceinline__ int digit_at(unsigned long long key, int level) {
  return (int)((key >> (3 * (kMaxLevels - 1 - level))) & 7ull);
}

// First index in [b, e) whose level digit is >= o (digits are sorted inside a node).
__device__ __forceinline__ int lower_digit(const unsigned long long *keys, int b, int e, int level, int o) {
  int lo = b, hi = e;
  while (lo < hi) {
    int mid = lo + ((hi - lo) >> 1);
    if (digit_at(keys[mid], level) < o) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

struct TreeArgs {
  const unsigned long long *keys;
  long long *lvl;
  int *nd_begin, *nd_count, *nd_nchild, *nd_childbeg, *nd_nnode, *nd_cell, *nd_pcell, *nd_ichild;
  double4 *nd_x;
  int4 *cell_b;
  int2 *cell_pl;
  double4 *cell_x;
  int *cell_node;
  const double *box;
  int *nd_sys;            // forest: node -> system (null: one system, box)
  const double4 *sys_box;  // forest: X0, R0 per system
  long long node_cap, cell_cap;
  int ncrit;
  int *err;
};

// Root half-width of the system a node belongs to.
__device__ __forceinline__ double node_R0(const TreeArgs &a, long long node) {
  return a.nd_sys ? a.sys_box[a.nd_sys[node]].w : a.box[3];
}

// Eight threads per node: thread o finds where octant o ends.
__global__ void k_expand(TreeArgs a, int level) {
  const long long cnt = a.lvl[level], start = a.lvl[kMaxLevels + 1 + level];
  const long long total = cnt * 8;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ((total + 31) / 32) * 32;
       t += (long long)gridDim.x * blockDim.x) {
    const bool live = t < total;
    const long long node = start + (live ? t / 8 : 0);
    const int o = (int)(t & 7);
    int nonempty = 0;
    int b = 0, c = 0;
    if (live) {
      b = a.nd_begin[node];
      c = a.nd_count[node];
    }
    // Keys hold digits for levels 0..kMaxLevels-1, so nodes down to that level split.
    const bool split = live && c > a.ncrit && level < kMaxLevels;
    if (live && c > a.ncrit && level == kMaxLevels && o == 0) atomicOr(a.err, kErrTreeTooDeep);
    if (split) {
      int s = lower_digit(a.keys, b, b + c, level, o);
      int e = lower_digit(a.keys, b, b + c, level, o + 1);
      nonempty = e > s;
    }
    unsigned m = __ballot_sync(0xffffffffu, nonempty);
    const int lane = threadIdx.x & 31;
    unsigned group = (m >> (lane & ~7)) & 0xffu;
    if (live && o == 0) a.nd_nchild[node] = __popc(group);
  }
}

// Exclusive scan of child counts over one level; its start is only known on the device.
struct LevelScan {
  using T = int;
  TreeArgs a;
  int level;
  const long long *startp;
  __device__ T value(long long i) const { return a.nd_nchild[*startp + i]; }
  __device__ void emit(long long i, const T &, const T &excl) const { a.nd_childbeg[*startp + i] = excl; }
  // Children beyond the node capacity are not created (k_emit skips them and
  // flags the overflow, which makes the host grow the buffers and rebuild), so
  // the next level's count is clamped to what fits: no kernel of this build
  // then touches a node slot past the capacity.
  __device__ void total(const T &t) const {
    const long long nstart = *startp + a.lvl[level];
    long long cnt = t;
    if (nstart + cnt > a.node_cap) {
      atomicOr(a.err, kErrCellOverflow);
      cnt = a.node_cap > nstart ? a.node_cap - nstart : 0;
    }
    a.lvl[level + 1] = cnt;
    a.lvl[kMaxLevels + 1 + level + 1] = nstart;
  }
};

__global__ void k_scan_prep(long long *lvl, int level, long long *n_out, long long *start_out) {
  *n_out = lvl[level];
  *start_out = lvl[kMaxLevels + 1 + level];
}

__global__ void k_emit(TreeArgs a, int level) {
  const long long cnt = a.lvl[level], start = a.lvl[kMaxLevels + 1 + level];
  const long long nstart = a.lvl[kMaxLevels + 1 + level + 1];
  const long long total = cnt * 8;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ((total + 31) / 32) * 32;
       t += (long long)gridDim.x * blockDim.x) {
    const bool live = t < total;
    const long long node = start + (live ? t / 8 : 0);
    const int o = (int)(t & 7);
    int b = 0, c = 0, s = 0, e = 0;
    if (live) {
      b = a.nd_begin[node];
      c = a.nd_count[node];
    }
    const bool split = live && c > a.ncrit && level < kMaxLevels;
    if (split) {
      s = lower_digit(a.keys, b, b + c, level, o);
      e = lower_digit(a.keys, b, b + c, level, o + 1);
    }
    const int nonempty = split && e > s;
    unsigned m = __ballot_sync(0xffffffffu, nonempty);
    const int lane = threadIdx.x & 31;
    unsigned group = (m >> (lane & ~7)) & 0xffu;
    if (nonempty) {
      const int rank = __popc(group & ((1u << o) - 1u));
      const long long child = nstart + a.nd_childbeg[node] + rank;
      if (child >= a.node_cap) {
        atomicOr(a.err, kErrCellOverflow);
      } else {
        const double4 X = a.nd_x[node];
        const double r = level_half(node_R0(a, node), level);
        if (a.nd_sys) a.nd_sys[child] = a.nd_sys[node];
        a.nd_begin[child] = s;
        a.nd_count[child] = e - s;
        a.nd_x[child] = make_double4(__dadd_rn(X.x, r * ((o & 1) ? 1.0 : -1.0)),
                                     __dadd_rn(X.y, r * ((o & 2) ? 1.0 : -1.0)),
                                     __dadd_rn(X.z, r * ((o & 4) ? 1.0 : -1.0)), 0.0);
        a.nd_nchild[child] = 0;
      }
    }
  }
}

// Subtree sizes, deepest level first.
__global__ void k_nnode(TreeArgs a, int level) {
  const long long cnt = a.lvl[level], start = a.lvl[kMaxLevels + 1 + level];
  const long long nstart = (level < kMaxLevels) ? a.lvl[kMaxLevels + 1 + level + 1] : 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cnt; i += (long long)gridDim.x * blockDim.x) {
    const long long node = start + i;
    if (node >= a.node_cap) continue;
    int nn = 1;
    const int nc = a.nd_nchild[node];
    const long long cb = nstart + a.nd_childbeg[node];
    for (int k = 0; k < nc; k++)
      if (cb + k < a.node_cap) nn += a.nd_nnode[cb + k];
    a.nd_nnode[node] = nn;
  }
}

// Reference cell layout, root first.
__global__ void k_cells(TreeArgs a, int level) {
  const long long cnt = a.lvl[level], start = a.lvl[kMaxLevels + 1 + level];
  const long long nstart = (level < kMaxLevels) ? a.lvl[kMaxLevels + 1 + level + 1] : 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cnt; i += (long long)gridDim.x * blockDim.x) {
    const long long node = start + i;
    if (node >= a.node_cap) continue;
    const double R0 = node_R0(a, node);
    const int c = a.nd_cell[node];
    if (c < 0 || c >= a.cell_cap) {
      atomicOr(a.err, kErrCellOverflow);
      continue;
    }
    const int nc = a.nd_nchild[node];
    const int ichild = a.nd_ichild[node];
    a.cell_b[c] = make_int4(a.nd_begin[node], a.nd_count[node], nc > 0 ? ichild : 0, nc);
    a.cell_pl[c] = make_int2(a.nd_pcell[node], level);
    const double4 X = a.nd_x[node];
    a.cell_x[c] = make_double4(X.x, X.y, X.z, R0 / (double)(1 << level));
    a.cell_node[c] = (int)node;
    const long long cb = nstart + a.nd_childbeg[node];
    int next = ichild + nc;
    for (int k = 0; k < nc; k++) {
      const long long ch = cb + k;
      if (ch >= a.node_cap) break;
      a.nd_cell[ch] = ichild + k;
      a.nd_pcell[ch] = c;
      a.nd_ichild[ch] = next;
      next += a.nd_nnode[ch] - 1;
    }
  }
}

// Restore input order inside each leaf: rank each body by its caller index.
__global__ void k_leaf_order(const int *nd_count, const int *nd_begin, const int *nd_nchild, const long long *lvl,
                             int *perm, int ncrit, long long node_cap) {
  extern __shared__ int sh[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int *buf = sh + warp * ncrit;
  long long total = 0;  // every node of every level (the level counts are clamped to the capacity)
  for (int l = 0; l <= kMaxLevels; l++) total += lvl[l];
  total = total < node_cap ? total : node_cap;
  const int wpb = blockDim.x >> 5;
  for (long long node = (long long)blockIdx.x * wpb + warp; node < total; node += (long long)gridDim.x * wpb) {
    if (nd_nchild[node] != 0) continue;
    const int b = nd_begin[node], c = nd_count[node];
    if (c > ncrit) continue;  // only a too-deep tree leaves such a node, already flagged
    for (int k = lane; k < c; k += 32) buf[k] = perm[b + k];
    __syncwarp();
    for (int k = lane; k < c; k += 32) {
      const int v = buf[k];
      int r = 0;
      for (int q = 0; q < c; q++) r += buf[q] < v;
      perm[b + r] = v;
    }
    __syncwarp();
  }
}

__global__ void k_gather(const double4 *x, const int *perm, long long n, double4 *out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = x[perm[i]];
}

// ---------------------------------------------------------------- forest of systems
// Independent systems side by side: every kernel below takes one tile of at
// most kForestTile bodies of one system (tile_sys, tile_beg) or one system, and
// reproduces per system exactly what the one-system kernels above compute.

__global__ void k_fb_init(unsigned long long *enc, long long words) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < words; i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i & 15);
    enc[i] = (t < 3 || (t >= 6 && t < 9)) ? ~0ull : 0ull;
  }
}

// k_bounds_estimate per system (body j of a system of n drifts n - 1 - j
// times, its first body n times).
__global__ void k_fb_estimate(const double4 *x, const int *tile_sys, const long long *tile_beg,
                              const long long *sys_off, unsigned long long *enc) {
  const int s = tile_sys[blockIdx.x];
  const long long s0 = sys_off[s], n = sys_off[s + 1] - s0, b = tile_beg[blockIdx.x];
  const long long e = min(b + (long long)kForestTile, s0 + n);
  unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0, 0, 0}, amax = 0;
  for (long long g = b + threadIdx.x; g < e; g += blockDim.x) {
    const double4 q = x[g];
    const double v[3] = {q.x, q.y, q.z};
    const long long j = g - s0;
    const double kc = (double)(j == 0 ? n : n - 1 - j) * 1e-5;
    for (int d = 0; d < 3; d++) {
      const unsigned long long a = order_enc(v[d] - kc), c = order_enc(v[d] + kc);
      lo[d] = a < lo[d] ? a : lo[d];
      hi[d] = c > hi[d] ? c : hi[d];
      const unsigned long long ab = order_enc(fabs(v[d]));
      amax = ab > amax ? ab : amax;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    for (int d = 0; d < 3; d++) {
      const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo[d], o);
      const unsigned long long c = __shfl_xor_sync(0xffffffffu, hi[d], o);
      lo[d] = a < lo[d] ? a : lo[d];
      hi[d] = c > hi[d] ? c : hi[d];
    }
    const unsigned long long m = __shfl_xor_sync(0xffffffffu, amax, o);
    amax = m > amax ? m : amax;
  }
  if ((threadIdx.x & 31) == 0) {
    unsigned long long *es = enc + 16 * (long long)s;
    for (int d = 0; d < 3; d++) {
      atomicMin(&es[6 + d], lo[d]);
      atomicMax(&es[9 + d], hi[d]);
    }
    atomicMax(&es[12], amax);
  }
}

// k_bounds_exact per system.
__global__ void k_fb_exact(const double4 *x, const int *tile_sys, const long long *tile_beg,
                           const long long *sys_off, unsigned long long *enc) {
  const int s = tile_sys[blockIdx.x];
  const long long s0 = sys_off[s], n = sys_off[s + 1] - s0, b = tile_beg[blockIdx.x];
  const long long e = min(b + (long long)kForestTile, s0 + n);
  unsigned long long *es = enc + 16 * (long long)s;
  const double span = order_dec(es[12]) + (double)n * 1e-5;
  const double B = (double)n * ldexp(1.0, ilogb(span > 1e-300 ? span : 1e-300) - 52) + 1e-300;
  double elo[3], ehi[3];
  for (int d = 0; d < 3; d++) {
    elo[d] = order_dec(es[6 + d]) + 2.0 * B;
    ehi[d] = order_dec(es[9 + d]) - 2.0 * B;
  }
  for (long long g = b + threadIdx.x; g < e; g += blockDim.x) {
    const double4 q = x[g];
    const double v[3] = {q.x, q.y, q.z};
    const long long j = g - s0;
    const long long k = (j == 0) ? n : n - 1 - j;
    const double kc = (double)k * 1e-5;
    for (int d = 0; d < 3; d++) {
      if (v[d] - kc <= elo[d]) atomicMin(&es[d], order_enc(drift_down(v[d], k)));
      if (v[d] + kc >= ehi[d]) atomicMax(&es[3 + d], order_enc(drift_up(v[d], k)));
    }
  }
}

// Bounds (k_bounds_final) and root box (bounds2box) of every system.
__global__ void k_fb_final(const unsigned long long *enc, const long long *sys_off, int nsys, double *bounds,
                           double4 *sys_box) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsys; s += gridDim.x * blockDim.x) {
    const long long n = sys_off[s + 1] - sys_off[s];
    double b[6];
    for (int t = 0; t < 6; t++) {
      b[t] = (n > 0) ? order_dec(enc[16 * (long long)s + t]) : 0.0;
      bounds[6 * (long long)s + t] = b[t];
    }
    sys_box[s] = box_of(b);
  }
}

__global__ void k_fkeys(const double4 *x, const int *tile_sys, const long long *tile_beg, const long long *sys_off,
                        const double4 *sys_box, unsigned long long *keys, int *vals) {
  const int s = tile_sys[blockIdx.x];
  const long long b = tile_beg[blockIdx.x], e = min(b + (long long)kForestTile, sys_off[s + 1]);
  const double4 box = sys_box[s];
  for (long long g = b + threadIdx.x; g < e; g += blockDim.x) {
    keys[g] = octant_key(x[g], box.x, box.y, box.z, box.w);
    vals[g] = (int)g;
  }
}

// System of each key-sorted body (bodies of system s are [sys_off[s], sys_off[s+1]) in caller order).
__global__ void k_fsys(const int *perm, long long n, const long long *sys_off, int nsys, unsigned *skey, int *idx) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long c = perm[i];
    int lo = 0, hi = nsys - 1;  // last s with sys_off[s] <= c
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (sys_off[mid] <= c) lo = mid;
      else hi = mid - 1;
    }
    skey[i] = (unsigned)lo;
    idx[i] = (int)i;
  }
}

__global__ void k_fgather(const unsigned long long *keys_in, const int *perm_in, const int *idx, long long n,
                          unsigned long long *keys_out, int *perm_out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int j = idx[i];
    keys_out[i] = keys_in[j];
    perm_out[i] = perm_in[j];
  }
}

// One root node per non-empty system, in system order, at level 0.
__global__ void k_froot(int nroots, const int *root_sys, const long long *sys_off, const double4 *sys_box,
                        long long *lvl, int *nd_begin, int *nd_count, double4 *nd_x, int *nd_sys) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int l = 0; l <= kMaxLevels; l++) {
      lvl[l] = 0;
      lvl[kMaxLevels + 1 + l] = 0;
    }
    lvl[0] = nroots;
  }
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nroots; k += gridDim.x * blockDim.x) {
    const int s = root_sys[k];
    const double4 X = sys_box[s];
    nd_begin[k] = (int)sys_off[s];
    nd_count[k] = (int)(sys_off[s + 1] - sys_off[s]);
    nd_x[k] = make_double4(X.x, X.y, X.z, 0.0);
    nd_sys[k] = s;
  }
}

// First cell of every system's tree: an exclusive scan of the root subtree
// sizes in system order (one block).  A root cell is its own parent, as cell 0
// is in the reference's layout, and its children start right after it.
__global__ void __launch_bounds__(1024) k_froot_cells(int nsys, const int *sys_root, const int *nd_nnode,
                                                      int *nd_cell, int *nd_pcell, int *nd_ichild, int *sys_cell,
                                                      long long cell_cap, int *err) {
  __shared__ long long part[1024];
  const int t = threadIdx.x, per = (nsys + 1023) / 1024;
  const int b = t * per, e = min(nsys, b + per);
  long long sum = 0;
  for (int s = b; s < e; s++) sum += sys_root[s] >= 0 ? nd_nnode[sys_root[s]] : 0;
  part[t] = sum;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const long long v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  long long base = part[t] - sum;
  for (int s = b; s < e; s++) {
    sys_cell[s] = (int)base;
    const int k = sys_root[s];
    if (k >= 0) {
      nd_cell[k] = (int)base;
      nd_pcell[k] = (int)base;
      nd_ichild[k] = (int)base + 1;
      base += nd_nnode[k];
    }
  }
  if (t == 1023) {
    sys_cell[nsys] = (int)part[1023];
    if (part[1023] > cell_cap) atomicOr(err, kErrCellOverflow);
  }
}

int grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > kNumSMs * 16) g = kNumSMs * 16;
  return (int)g;
}

}  // namespace

// Per-system bounds and root boxes of a forest (BoundBox::getBounds and
// bounds2box of every system on its own).
static void forest_bounds(Context &C) {
  TreeBufs &T = C.tree;
  cudaStream_t st = C.stream;
  const long long words = 16LL * T.nsys;
  T.sys_enc.ensure(words);
  T.sys_bounds.ensure(6LL * T.nsys);
  T.sys_box.ensure(T.nsys);
  k_fb_init<<<grid_for(words, 256), 256, 0, st>>>(T.sys_enc.p, words);
  EXA_CHECK_LAUNCH();
  if (T.ntiles > 0) {
    k_fb_estimate<<<(unsigned)T.ntiles, 256, 0, st>>>(T.xyzq.p, T.tile_sys.p, T.tile_beg.p, T.sys_off.p, T.sys_enc.p);
    EXA_CHECK_LAUNCH();
    k_fb_exact<<<(unsigned)T.ntiles, 256, 0, st>>>(T.xyzq.p, T.tile_sys.p, T.tile_beg.p, T.sys_off.p, T.sys_enc.p);
    EXA_CHECK_LAUNCH();
  }
  k_fb_final<<<grid_for(T.nsys, 128), 128, 0, st>>>(T.sys_enc.p, T.sys_off.p, T.nsys, T.sys_bounds.p, T.sys_box.p);
  EXA_CHECK_LAUNCH();
}

void compute_bounds(Context &C) {
  TreeBufs &T = C.tree;
  if (T.nsys) {
    forest_bounds(C);
    return;
  }
  T.bounds.ensure(6);
  T.bounds_enc.ensure(16);
  k_bounds_init<<<1, 32, 0, C.stream>>>(T.bounds_enc.p);
  EXA_CHECK_LAUNCH();
  if (T.n > 0) {
    k_bounds_estimate<<<grid_for(T.n, 256), 256, 0, C.stream>>>(T.xyzq.p, T.n, T.bounds_enc.p, nullptr);
    EXA_CHECK_LAUNCH();
    k_bounds_exact<<<grid_for(T.n, 256), 256, 0, C.stream>>>(T.xyzq.p, T.n, T.bounds_enc.p, nullptr);
    EXA_CHECK_LAUNCH();
  }
  k_bounds_final<<<1, 32, 0, C.stream>>>(T.bounds_enc.p, T.n, T.bounds.p);
  EXA_CHECK_LAUNCH();
}

void extend_bounds(Context &C, const double4 *x, long long n) {
  TreeBufs &T = C.tree;
  if (n <= 0) return;  // no bodies: the bounds stay as they are
  T.bounds_enc.ensure(16);
  k_bounds_init<<<1, 32, 0, C.stream>>>(T.bounds_enc.p);
  EXA_CHECK_LAUNCH();
  k_bounds_estimate<<<grid_for(n, 256), 256, 0, C.stream>>>(x, n, T.bounds_enc.p, T.bounds.p);
  EXA_CHECK_LAUNCH();
  k_bounds_exact<<<grid_for(n, 256), 256, 0, C.stream>>>(x, n, T.bounds_enc.p, T.bounds.p);
  EXA_CHECK_LAUNCH();
  k_bounds_final<<<1, 32, 0, C.stream>>>(T.bounds_enc.p, n, T.bounds.p);
  EXA_CHECK_LAUNCH();
}

void set_bounds(Context &C, const double *b6) {
  C.tree.bounds.ensure(6);
  EXA_CUDA(cudaMemcpyAsync(C.tree.bounds.p, b6, 6 * sizeof(double), cudaMemcpyHostToDevice, C.stream));
}

static void ensure_nodes(TreeBufs &T, long long cap) {
  T.node_cap = cap;
  T.nd_begin.ensure(cap);
  T.nd_count.ensure(cap);
  T.nd_nchild.ensure(cap);
  T.nd_childbeg.ensure(cap);
  T.nd_nnode.ensure(cap);
  T.nd_cell.ensure(cap);
  T.nd_pcell.ensure(cap);
  T.nd_ichild.ensure(cap);
  T.nd_x.ensure(cap);
  T.cell_cap = cap;
  T.cell_b.ensure(cap);
  T.cell_pl.ensure(cap);
  T.cell_x.ensure(cap);
  T.cell_node.ensure(cap);
}

void build_tree(Context &C) {
  TreeBufs &T = C.tree;
  const long long n = T.n;
  const int ncrit = C.prm.ncrit;
  const bool forest = T.nsys > 0;
  cudaStream_t st = C.stream;
  T.box.ensure(4);
  T.lvl.ensure(2 * (kMaxLevels + 1) + 4);
  // Node capacity for this system (a reused context may receive a larger one);
  // deeper trees than this estimate overflow, are flagged and rebuilt larger.
  const long long est = 1024 + 8 * 4 * (n / (ncrit + 1) + 1) + 8LL * T.nroots;
  if (est > T.node_cap) ensure_nodes(T, est);
  T.keys.ensure(n);
  T.keys_alt.ensure(n);
  T.perm.ensure(n);
  T.perm_alt.ensure(n);
  T.xyzq_tree.ensure(n);
  if (forest) {
    T.nd_sys.ensure(T.node_cap);
    T.sys_cell.ensure(T.nsys + 1);
  } else {
    k_box<<<1, 32, 0, st>>>(T.bounds.p, T.box.p);
    EXA_CHECK_LAUNCH();
  }
  if (n > 0 && !forest) {
    k_keys<<<grid_for(n, 256), 256, 0, st>>>(T.xyzq.p, n, T.box.p, T.keys.p, T.perm.p);
    EXA_CHECK_LAUNCH();
    bool alt = radix_sort_u64((uint64_t *)T.keys.p, T.perm.p, (uint64_t *)T.keys_alt.p, T.perm_alt.p, n, 0,
                              3 * kMaxLevels, C.sort, C.err.p, st);
    if (alt) {
      std::swap(T.keys.p, T.keys_alt.p);
      std::swap(T.perm.p, T.perm_alt.p);
    }
  } else if (n > 0) {
    // keys of every body in its own system's box, sorted; then a stable pass
    // on the system makes the order (system, key), each system's bodies in
    // exactly the order its solo tree gives them
    k_fkeys<<<(unsigned)T.ntiles, 256, 0, st>>>(T.xyzq.p, T.tile_sys.p, T.tile_beg.p, T.sys_off.p, T.sys_box.p,
                                                T.keys.p, T.perm.p);
    EXA_CHECK_LAUNCH();
    bool alt = radix_sort_u64((uint64_t *)T.keys.p, T.perm.p, (uint64_t *)T.keys_alt.p, T.perm_alt.p, n, 0,
                              3 * kMaxLevels, C.sort, C.err.p, st);
    if (alt) {
      std::swap(T.keys.p, T.keys_alt.p);
      std::swap(T.perm.p, T.perm_alt.p);
    }
    if (T.nsys > 1) {
      T.fs_key.ensure(n);
      T.fs_key_alt.ensure(n);
      T.fs_idx.ensure(n);
      T.fs_idx_alt.ensure(n);
      k_fsys<<<grid_for(n, 256), 256, 0, st>>>(T.perm.p, n, T.sys_off.p, T.nsys, T.fs_key.p, T.fs_idx.p);
      EXA_CHECK_LAUNCH();
      int bits = 0;
      while ((1LL << bits) <= (long long)(T.nsys - 1)) bits++;
      const bool alt2 = radix_sort_u32(T.fs_key.p, T.fs_idx.p, T.fs_key_alt.p, T.fs_idx_alt.p, n, 0, bits, C.sort,
                                       C.err.p, st);
      k_fgather<<<grid_for(n, 256), 256, 0, st>>>(T.keys.p, T.perm.p, alt2 ? T.fs_idx_alt.p : T.fs_idx.p, n,
                                                  T.keys_alt.p, T.perm_alt.p);
      EXA_CHECK_LAUNCH();
      std::swap(T.keys.p, T.keys_alt.p);
      std::swap(T.perm.p, T.perm_alt.p);
    }
  }
  TreeArgs a;
  a.keys = T.keys.p;
  a.lvl = T.lvl.p;
  a.nd_begin = T.nd_begin.p;
  a.nd_count = T.nd_count.p;
  a.nd_nchild = T.nd_nchild.p;
  a.nd_childbeg = T.nd_childbeg.p;
  a.nd_nnode = T.nd_nnode.p;
  a.nd_cell = T.nd_cell.p;
  a.nd_pcell = T.nd_pcell.p;
  a.nd_ichild = T.nd_ichild.p;
  a.nd_x = T.nd_x.p;
  a.cell_b = T.cell_b.p;
  a.cell_pl = T.cell_pl.p;
  a.cell_x = T.cell_x.p;
  a.cell_node = T.cell_node.p;
  a.box = T.box.p;
  a.nd_sys = forest ? T.nd_sys.p : nullptr;
  a.sys_box = forest ? T.sys_box.p : nullptr;
  a.node_cap = T.node_cap;
  a.cell_cap = T.cell_cap;
  a.ncrit = ncrit;
  a.err = C.err.p;
  if (forest) {
    k_froot<<<grid_for(T.nroots, 128), 128, 0, st>>>(T.nroots, T.root_sys.p, T.sys_off.p, T.sys_box.p, T.lvl.p,
                                                     T.nd_begin.p, T.nd_count.p, T.nd_x.p, T.nd_sys.p);
  } else {
    k_tree_root<<<1, 32, 0, st>>>(n, T.lvl.p, T.nd_begin.p, T.nd_count.p, T.nd_x.p, T.box.p, T.nd_cell.p,
                                  T.nd_pcell.p, T.nd_ichild.p);
  }
  EXA_CHECK_LAUNCH();
  // The level kernels run down to one level below the deepest splitting one
  // (its nodes are leaves), so a shallow tree costs a few launches per
  // level, not kMaxLevels of them; the deepest splitting level is read back
  // from the sorted keys first (one small transfer).
  int last = 0;
  if (n > ncrit) {
    T.split_level.ensure(1);
    EXA_CUDA(cudaMemsetAsync(T.split_level.p, 0xff, sizeof(int), st));
    k_split_level<<<grid_for(n, 256), 256, 0, st>>>(T.keys.p, T.perm.p, n, ncrit, forest ? T.sys_off.p : nullptr,
                                                   T.nsys, T.split_level.p);
    EXA_CHECK_LAUNCH();
    int *deepest_h = reinterpret_cast<int *>(C.pin + kPinScratch);
    EXA_CUDA(cudaMemcpyAsync(deepest_h, T.split_level.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    EXA_CUDA(cudaStreamSynchronize(st));
    const int deepest = *deepest_h;
    last = std::min(deepest + 1, kMaxLevels);
  }
  // per-level kernels: eight threads per node at most node_cap nodes
  const int node_grid = (int)std::max<long long>(1, std::min<long long>(kNumSMs * 4, (8 * T.node_cap + 255) / 256));
  long long *lvl_n = T.lvl.p + 2 * (kMaxLevels + 1);
  long long *lvl_s = lvl_n + 1;
  for (int l = 0; l <= last; l++) {
    k_expand<<<node_grid, 256, 0, st>>>(a, l);
    EXA_CHECK_LAUNCH();
    if (l == kMaxLevels) break;  // deepest level: only the too-deep check runs
    k_scan_prep<<<1, 1, 0, st>>>(T.lvl.p, l, lvl_n, lvl_s);
    EXA_CHECK_LAUNCH();
    LevelScan ls{a, l, lvl_s};
    launch_scan<1024, 8>(ls, lvl_n, 0, T.node_cap, C.scan, C.err.p, st);
    k_emit<<<node_grid, 256, 0, st>>>(a, l);
    EXA_CHECK_LAUNCH();
  }
  if (C.ev_link) EXA_CUDA(cudaEventRecord(C.ev_link, st));  // BuildTree: growTree done, linkTree next
  for (int l = last; l >= 0; l--) {
    k_nnode<<<node_grid, 256, 0, st>>>(a, l);
    EXA_CHECK_LAUNCH();
  }
  if (forest) {
    k_froot_cells<<<1, 1024, 0, st>>>(T.nsys, T.sys_root.p, T.nd_nnode.p, T.nd_cell.p, T.nd_pcell.p, T.nd_ichild.p,
                                      T.sys_cell.p, T.cell_cap, C.err.p);
    EXA_CHECK_LAUNCH();
  }
  for (int l = 0; l <= last; l++) {
    k_cells<<<node_grid, 256, 0, st>>>(a, l);
    EXA_CHECK_LAUNCH();
  }
  if (n > 0) {
    const int wpb = 4;
    k_leaf_order<<<kNumSMs * 8, 32 * wpb, wpb * ncrit * sizeof(int), st>>>(T.nd_count.p, T.nd_begin.p,
                                                                           T.nd_nchild.p, T.lvl.p, T.perm.p,
                                                                           ncrit, T.node_cap);
    EXA_CHECK_LAUNCH();
    k_gather<<<grid_for(n, 256), 256, 0, st>>>(T.xyzq.p, T.perm.p, n, T.xyzq_tree.p);
    EXA_CHECK_LAUNCH();
  }
}

void sync_tree(Context &C) {
  TreeBufs &T = C.tree;
  // staging in the context's pinned block: level counts, then the cell count
  // (or a forest's per-system cell offsets, when they fit)
  static_assert(kPinScratch + sizeof(T.lvl_host) + sizeof(int) <= 1024, "pinned staging layout");
  long long *lvl_h = reinterpret_cast<long long *>(C.pin + kPinScratch);
  int *nn_h = reinterpret_cast<int *>(C.pin + 1024);
  const bool sys_pinned = (size_t)(T.nsys + 1) * sizeof(int) <= kPinBytes - 1024;
  EXA_CUDA(cudaMemcpyAsync(lvl_h, T.lvl.p, sizeof(T.lvl_host), cudaMemcpyDeviceToHost, C.stream));
  if (T.nsys) {
    T.sys_cell_host.assign(T.nsys + 1, 0);
    EXA_CUDA(cudaMemcpyAsync(sys_pinned ? (void *)nn_h : (void *)T.sys_cell_host.data(), T.sys_cell.p,
                             (T.nsys + 1) * sizeof(int), cudaMemcpyDeviceToHost, C.stream));
  } else if (T.n > 0) {
    EXA_CUDA(cudaMemcpyAsync(nn_h, T.nd_nnode.p, sizeof(int), cudaMemcpyDeviceToHost, C.stream));
  }
  EXA_CUDA(cudaMemcpyAsync(C.err_host, C.err.p, sizeof(int), cudaMemcpyDeviceToHost, C.stream));
  EXA_CUDA(cudaStreamSynchronize(C.stream));
  std::memcpy(T.lvl_host, lvl_h, sizeof(T.lvl_host));
  int nn = 0;
  if (T.nsys) {
    if (sys_pinned) std::memcpy(T.sys_cell_host.data(), nn_h, (T.nsys + 1) * sizeof(int));
    nn = T.sys_cell_host[T.nsys];
  } else if (T.n > 0) {
    nn = *nn_h;
  }
  T.ncells = (T.n > 0) ? nn : 0;
  T.depth = 0;
  for (int l = 0; l <= kMaxLevels; l++)
    if (T.lvl_host[l] > 0) T.depth = l;
}

}  // namespace exafmm_b200
