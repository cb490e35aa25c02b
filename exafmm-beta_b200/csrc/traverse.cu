// Dual tree traversal on the device (include/traversal.h:90-230, 326-352).
//
// The reference recurses over cell pairs; every pair either passes the MAC
// (M2L), is a leaf-leaf pair (P2P, or M2L when the source holds no bodies), or
// is split by splitCell's rule: split Ci when Cj is a leaf, Cj when Ci is a
// leaf, both (full child cross product, as TraverseRange visits it) when
// NBODY_i + NBODY_j >= nspawn or Ci == Cj, otherwise the larger radius (Ci on
// ties).  The set of pairs this visits does not depend on recursion order, so
// here it is walked breadth first: each sweep is one single-pass scan over the
// current pair queue that decides every pair, prefix-sums what it emits and
// writes children, M2L and P2P pairs at their scanned offsets -- deterministic
// output, no atomics.  The lists are then grouped by target cell with a stable
// radix sort, which keeps traversal order among a target's sources.
#include <algorithm>

#include "fmm.h"

namespace exafmm_b200 {
namespace {

constexpr int kMaxSweeps = 2 * (kMaxLevels + 1) + 2;
constexpr int kImgShift = 26;
constexpr int kCellMask = (1 << kImgShift) - 1;

struct PairCtx {
  const int4 *cell_b;      // target cells
  const double4 *cell_x;
  const int4 *cell_bj;     // source cells (the same table unless sources have their own tree)
  const double4 *cell_xj;
  int same;                // one tree: Ci == Cj is possible (splitCell splits both then)
  double theta;
  int nspawn;
  double cycle;
};

enum Mode : int { kM2L = 0, kP2P = 1, kSplitI = 2, kSplitJ = 3, kSplitBoth = 4 };

__device__ __forceinline__ int decide(const PairCtx &c, int2 pr, int4 &bi, int4 &bj) {
  const int ci = pr.x, cj = pr.y & kCellMask, img = pr.y >> kImgShift;
  const double4 Xi = c.cell_x[ci], Xj = c.cell_xj[cj];
  bi = c.cell_b[ci];
  bj = c.cell_bj[cj];
  const double sx = (double)(img / 9 - 1) * c.cycle;
  const double sy = (double)((img / 3) % 3 - 1) * c.cycle;
  const double sz = (double)(img % 3 - 1) * c.cycle;
  const double dx = __dsub_rn(__dsub_rn(Xi.x, Xj.x), sx);
  const double dy = __dsub_rn(__dsub_rn(Xi.y, Xj.y), sy);
  const double dz = __dsub_rn(__dsub_rn(Xi.z, Xj.z), sz);
  const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  const double rt2 = __dmul_rn(__dmul_rn(r2, c.theta), c.theta);
  const double rr = __dadd_rn(Xi.w, Xj.w);
  if (rt2 > __dmul_rn(__dmul_rn(rr, rr), 1 - 1e-3)) return kM2L;
  if (bi.w == 0 && bj.w == 0) return bj.y == 0 ? kM2L : kP2P;
  if (bj.w == 0) return kSplitI;
  if (bi.w == 0) return kSplitJ;
  if (bi.y + bj.y >= c.nspawn || (c.same && ci == cj)) return kSplitBoth;
  return (Xi.w >= Xj.w) ? kSplitI : kSplitJ;
}

struct PairScan {
  using T = Count2;  // a: child pairs; b: (m2l << 32) | p2p
  PairCtx c;
  const int2 *qin;
  int2 *qout, *m2l, *p2p;
  long long *cnt;
  int sweep;
  long long q_cap, m2l_cap, p2p_cap;
  int *err;
  // After an overflow the queue holds slots that were never written: every
  // later sweep of this attempt does nothing, and the host reruns it larger.
  __device__ bool stopped() const { return (*(volatile int *)err & (kErrQueueOverflow | kErrListOverflow)) != 0; }
  __device__ T value(long long i) const {
    if (i >= q_cap || stopped()) return T{0, 0};
    int4 bi, bj;
    const int mode = decide(c, qin[i], bi, bj);
    T v{0, 0};
    if (mode == kM2L) v.b = 1ull << 32;
    else if (mode == kP2P) v.b = 1ull;
    else if (mode == kSplitI) v.a = bi.w;
    else if (mode == kSplitJ) v.a = bj.w;
    else v.a = (unsigned long long)bi.w * bj.w;
    return v;
  }
  __device__ void emit(long long i, const T &v, const T &excl) const {
    if (i >= q_cap || stopped()) return;
    const int2 pr = qin[i];
    // value() decided this pair: M2L and P2P show in v.b; a split needs the
    // child ranges again and, in the last rule of decide(), the radii
    int4 bi = make_int4(0, 0, 0, 0), bj = make_int4(0, 0, 0, 0);
    int mode;
    if (v.b >> 32) {
      mode = kM2L;
    } else if (v.b) {
      mode = kP2P;
    } else {
      const int ci = pr.x, cj = pr.y & kCellMask;
      bi = c.cell_b[ci];
      bj = c.cell_bj[cj];
      if (bj.w == 0) mode = kSplitI;
      else if (bi.w == 0) mode = kSplitJ;
      else if (bi.y + bj.y >= c.nspawn || (c.same && ci == cj)) mode = kSplitBoth;
      else mode = (c.cell_x[ci].w >= c.cell_xj[cj].w) ? kSplitI : kSplitJ;
    }
    const int img = pr.y & ~kCellMask;
    if (mode == kM2L) {
      const long long at = cnt[3 * sweep + 1] + (long long)(excl.b >> 32);
      if (at < m2l_cap) m2l[at] = pr;
      else atomicOr(err, kErrListOverflow);
    } else if (mode == kP2P) {
      const long long at = cnt[3 * sweep + 2] + (long long)(excl.b & 0xffffffffull);
      if (at < p2p_cap) p2p[at] = pr;
      else atomicOr(err, kErrListOverflow);
    } else {
      const long long at = (long long)excl.a;
      const int cj = pr.y & kCellMask;
      int na = 1, nb = 1, a0 = pr.x, b0 = cj;
      if (mode == kSplitI || mode == kSplitBoth) { na = bi.w; a0 = bi.z; }
      if (mode == kSplitJ || mode == kSplitBoth) { nb = bj.w; b0 = bj.z; }
      if (at + (long long)na * nb > q_cap) {
        atomicOr(err, kErrQueueOverflow);
        return;
      }
      for (int a = 0; a < na; a++)
        for (int b = 0; b < nb; b++) qout[at + a * nb + b] = make_int2(a0 + a, (b0 + b) | img);
    }
  }
  __device__ void total(const T &t) const {
    cnt[3 * (sweep + 1)] = (long long)t.a;
    cnt[3 * (sweep + 1) + 1] = cnt[3 * sweep + 1] + (long long)(t.b >> 32);
    cnt[3 * (sweep + 1) + 2] = cnt[3 * sweep + 2] + (long long)(t.b & 0xffffffffull);
  }
};

__global__ void k_trav_init(int2 *q, long long *cnt, int images, long long ncells) {
  if (threadIdx.x != 0) return;
  for (int s = 0; s < 3 * (kMaxSweeps + 1); s++) cnt[s] = 0;
  if (ncells == 0) return;
  if (images == 0) {
    q[0] = make_int2(0, 13 << kImgShift);  // image 13 = no shift
    cnt[0] = 1;
  } else {
    for (int k = 0; k < 27; k++) q[k] = make_int2(0, k << kImgShift);
    cnt[0] = 27;
  }
}

// A forest starts from every system's root pair (Traversal::traverse of each
// system, free space); pairs never cross systems from there.
__global__ void k_trav_init_forest(int2 *q, long long *cnt, const int *nd_cell, int nroots) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int s = 0; s < 3 * (kMaxSweeps + 1); s++) cnt[s] = 0;
    cnt[0] = nroots;
  }
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nroots; k += gridDim.x * blockDim.x) {
    const int c = nd_cell[k];  // root node k's cell
    q[k] = make_int2(c, c | (13 << kImgShift));
  }
}

__global__ void k_split_pairs(const int2 *pairs, long long n, unsigned *key, int *val) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int2 p = pairs[i];
    key[i] = (unsigned)p.x;
    val[i] = p.y;
  }
}

__global__ void k_csr(const unsigned *key, long long n, long long ncells, int *off) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c <= ncells; c += (long long)gridDim.x * blockDim.x) {
    long long lo = 0, hi = n;
    while (lo < hi) {
      long long mid = (lo + hi) >> 1;
      if ((long long)key[mid] < c) lo = mid + 1;
      else hi = mid;
    }
    off[c] = (int)lo;
  }
}

int bits_for(long long v) {
  int b = 0;
  while ((1LL << b) <= v) b++;
  return b;
}

void group_by_target(Context &C, const int2 *pairs, long long n, long long ncells, ListBufs &lb, DBuf<int> &off,
                     DBuf<int> &src) {
  cudaStream_t st = C.stream;
  off.ensure(ncells + 1);
  src.ensure(n > 0 ? n : 1);
  lb.key.ensure(n);
  lb.key_alt.ensure(n);
  lb.val.ensure(n);
  lb.val_alt.ensure(n);
  if (n > 0) {
    k_split_pairs<<<kNumSMs * 8, 256, 0, st>>>(pairs, n, lb.key.p, lb.val.p);
    EXA_CHECK_LAUNCH();
    const int bits = bits_for(ncells);  // target cell ids
    bool alt = radix_sort_u32(lb.key.p, lb.val.p, lb.key_alt.p, lb.val_alt.p, n, 0, bits, C.sort, C.err.p, st);
    unsigned *k = alt ? lb.key_alt.p : lb.key.p;
    int *v = alt ? lb.val_alt.p : lb.val.p;
    EXA_CUDA(cudaMemcpyAsync(src.p, v, n * sizeof(int), cudaMemcpyDeviceToDevice, st));
    k_csr<<<kNumSMs * 2, 256, 0, st>>>(k, n, ncells, off.p);
    EXA_CHECK_LAUNCH();
  } else {
    EXA_CUDA(cudaMemsetAsync(off.p, 0, (ncells + 1) * sizeof(int), st));
  }
}

}  // namespace

bool traverse(Context &C, ListBufs &lb, const TreeBufs *sources) {
  const long long ncells = C.tree.ncells;
  const TreeBufs &S = sources ? *sources : C.tree;
  cudaStream_t st = C.stream;
  // capacities for this tree (a reused context may hold a larger one now)
  lb.m2l_cap = std::max(lb.m2l_cap, 256 * ncells + 1024);
  lb.p2p_cap = std::max(lb.p2p_cap, 64 * ncells + 1024);
  lb.q_cap = std::max(lb.q_cap, lb.m2l_cap + lb.p2p_cap);
  lb.q0.ensure(lb.q_cap);
  lb.q1.ensure(lb.q_cap);
  lb.m2l.ensure(lb.m2l_cap);
  lb.p2p.ensure(lb.p2p_cap);
  lb.cnt.ensure(3 * (kMaxSweeps + 1));
  if (C.tree.nsys) {
    if (sources || C.prm.images) throw_msg("a forest of systems is solved in free space with sources == targets");
    lb.q_cap = std::max<long long>(lb.q_cap, C.tree.nroots);
    lb.q0.ensure(lb.q_cap);
    lb.q1.ensure(lb.q_cap);
    k_trav_init_forest<<<std::max(1, std::min(kNumSMs, div_up(C.tree.nroots, 128))), 128, 0, st>>>(
        lb.q0.p, lb.cnt.p, C.tree.nd_cell.p, C.tree.nroots);
  } else {
    k_trav_init<<<1, 32, 0, st>>>(lb.q0.p, lb.cnt.p, C.prm.images, std::min<long long>(ncells, S.ncells));
  }
  EXA_CHECK_LAUNCH();
  PairScan ps;
  ps.c.cell_b = C.tree.cell_b.p;
  ps.c.cell_x = C.tree.cell_x.p;
  ps.c.cell_bj = S.cell_b.p;
  ps.c.cell_xj = S.cell_x.p;
  ps.c.same = sources == nullptr;
  ps.c.theta = C.prm.theta;
  ps.c.nspawn = C.prm.nspawn;
  ps.c.cycle = C.prm.cycle;
  ps.m2l = lb.m2l.p;
  ps.p2p = lb.p2p.p;
  ps.cnt = lb.cnt.p;
  ps.q_cap = lb.q_cap;
  ps.m2l_cap = lb.m2l_cap;
  ps.p2p_cap = lb.p2p_cap;
  ps.err = C.err.p;
  // Every split takes one side of a pair a level deeper and leaf pairs are
  // decided where they are met, so trees of depths di and dj need at most
  // di + dj + 1 sweeps; two more are launched, and the queue after the last
  // must be empty.
  const int nsw = std::min(kMaxSweeps, (C.tree.depth + 1) + (S.depth + 1) + 2);
  for (int s = 0; s < nsw; s++) {
    ps.sweep = s;
    ps.qin = (s & 1) ? lb.q1.p : lb.q0.p;
    ps.qout = (s & 1) ? lb.q0.p : lb.q1.p;
    // 8192-pair tiles (64 registers, one block per SM): lists 5.2 -> 4.1 ms
    // on a 4M-body solve against 2048-pair tiles of 256 threads
    launch_scan<1024, 8>(ps, lb.cnt.p + 3 * s, 0, lb.q_cap, C.scan, C.err.p, st);
  }
  static_assert(kPinScratch + 3 * (kMaxSweeps + 1) * sizeof(long long) <= kPinBytes, "pinned staging layout");
  const long long *cnt = reinterpret_cast<const long long *>(C.pin + kPinScratch);
  EXA_CUDA(cudaMemcpyAsync(C.pin + kPinScratch, lb.cnt.p, 3 * (nsw + 1) * sizeof(long long), cudaMemcpyDeviceToHost,
                           st));
  EXA_CUDA(cudaMemcpyAsync(C.err_host, C.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  EXA_CUDA(cudaStreamSynchronize(st));
  long long qmax = 0;
  lb.sweeps = 0;
  for (int s = 0; s <= nsw; s++) {
    qmax = cnt[3 * s] > qmax ? cnt[3 * s] : qmax;
    if (cnt[3 * s] > 0) lb.sweeps = s + 1;
  }
  lb.n_m2l = cnt[3 * nsw + 1];
  lb.n_p2p = cnt[3 * nsw + 2];
  const int e = *C.err_host;
  if (e & (kErrQueueOverflow | kErrListOverflow)) {
    lb.q_cap = (qmax > lb.q_cap ? qmax : 2 * lb.q_cap) * 5 / 4 + 1024;
    lb.m2l_cap = lb.n_m2l * 5 / 4 + 1024 > lb.m2l_cap ? lb.n_m2l * 5 / 4 + 1024 : 2 * lb.m2l_cap;
    lb.p2p_cap = lb.n_p2p * 5 / 4 + 1024 > lb.p2p_cap ? lb.n_p2p * 5 / 4 + 1024 : 2 * lb.p2p_cap;
    EXA_CUDA(cudaMemsetAsync(C.err.p, 0, sizeof(int), st));
    return false;
  }
  if (lb.sweeps > nsw) throw_msg("traversal did not terminate within the sweep limit");
  group_by_target(C, lb.m2l.p, lb.n_m2l, ncells, lb, lb.m2l_off, lb.m2l_src);
  group_by_target(C, lb.p2p.p, lb.n_p2p, ncells, lb, lb.p2p_off, lb.p2p_src);
  return true;
}

}  // namespace exafmm_b200
