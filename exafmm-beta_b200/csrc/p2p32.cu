// Mixed-precision P2P (kernels/laplace.h:150-235) in FP32.
//
// Coordinates.  Every body is stored once per solve as a two-float pair
// (hi + lo, about 48 significant bits) relative to the root cell's center.
// The separation of a pair is (t_hi - s_hi) + (t_lo - s_lo): for close bodies
// the hi difference is exact, so close pairs keep their relative accuracy,
// and the rest of the interaction (r^2, rsqrt, the sums) is plain FP32.
// A periodic image shift is added to the source's two-float pair when it is
// staged (TwoSum of the hi parts, the rounding error carried into lo).
//
// Work mapping.  One warp evaluates one target leaf at a time.  The leaf's
// source bodies (the bodies of every leaf in its P2P list, one after another)
// form a stream that the warp stages into shared memory in chunks.  The 32
// lanes are split into G = 32 / S groups of S lanes; each lane holds two
// targets, so a group covers 2S targets, and the G groups take interleaved
// pairs of the chunk's sources.  S is chosen from the leaf's size so that
// small leaves still fill the warp (<= 8 bodies: 8 groups of 4 lanes; <= 16:
// 4 x 8; <= 32: 2 x 16; larger: 1 x 32, in passes of 64 targets).  Two
// consecutive sources go through one packed f32x2 operation, so the
// arithmetic of two interactions is one instruction stream.
//
// Accumulation.  Each lane sums a chunk (at most 32 sources per group) in
// FP32 and then adds that partial into Kahan-compensated running sums
// (include/kahan.h:34-48 semantics), so the error does not grow with the
// number of chunks; the groups' sums are combined in FP64 and added to the
// FP64 outputs.
//
// r = 0.  A pair at zero distance contributes nothing, as in the reference
// (kernels/laplace.h:171: invR2 = 0 when R2 = 0).  The test is applied to
// every pair: it runs on the integer/select pipe, beside the FP32 pipe that
// bounds this kernel.  The rsqrt flushes subnormal inputs, so a pair closer
// than about 1e-19 (an r^2 below the FP32 normal range) also contributes
// nothing; such inputs need the FP64 plain method.
#include <algorithm>
#include <stdexcept>

#include "fmm.h"

namespace exafmm_b200 {
namespace {

constexpr int kMaxGroups = 8;                 // groups of 4 lanes
constexpr int kStagePairs = 16 * kMaxGroups;  // chunk = 32 * G sources = 16 * G pairs
constexpr unsigned kFull = 0xffffffffu;

typedef unsigned long long f2p;  // two floats in one 64-bit register

__device__ __forceinline__ f2p pk2(float a, float b) {
  f2p r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float2 unpk2(f2p v) {
  float a, b;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
  return make_float2(a, b);
}
__device__ __forceinline__ f2p add2(f2p a, f2p b) {
  f2p d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2p sub2(f2p a, f2p b) {
  f2p d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2p mul2(f2p a, f2p b) {
  f2p d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2p fma2(f2p a, f2p b, f2p c) {
  f2p d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Compensated running sum: c holds the rounding error of the last addition,
// so the sum is s - c.
struct Kahan {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

// One warp's chunk of staged sources, as pairs of consecutive sources:
//   A = (hx0, hx1, hy0, hy1), B = (hz0, hz1, q0, q1),
//   C = (lx0, lx1, ly0, ly1), D = (lz0, lz1, -, -)
// Four arrays rather than one array of 64-byte records, so that the G groups,
// which read G consecutive pairs at once, hit distinct banks.
struct Stage {
  float4 A[kStagePairs], B[kStagePairs], C[kStagePairs], D[kStagePairs];
};

// x32[2i] = (hi of x - X_root, q), x32[2i+1] = (lo parts, 0), bodies in tree order.
__global__ void k_abs32(const double4 *xt, long long n, const double4 *cell_x, float4 *x32) {
  const double4 X0 = cell_x[0];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double4 b = xt[i];
    const double dx = b.x - X0.x, dy = b.y - X0.y, dz = b.z - X0.z;
    const float hx = (float)dx, hy = (float)dy, hz = (float)dz;
    x32[2 * i] = make_float4(hx, hy, hz, (float)b.w);
    x32[2 * i + 1] = make_float4((float)(dx - (double)hx), (float)(dy - (double)hy), (float)(dz - (double)hz), 0.f);
  }
}

// The same in a forest: each body relative to its own system's root center
// (the center of its root cell, so each system's values equal its solo solve's).
__global__ void k_abs32_forest(const double4 *xt, long long n, const long long *sys_off, int nsys,
                               const double4 *sys_box, float4 *x32) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nsys - 1;  // last s with sys_off[s] <= i
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (sys_off[mid] <= i) lo = mid;
      else hi = mid - 1;
    }
    const double4 X0 = sys_box[lo];
    const double4 b = xt[i];
    const double dx = b.x - X0.x, dy = b.y - X0.y, dz = b.z - X0.z;
    const float hx = (float)dx, hy = (float)dy, hz = (float)dz;
    x32[2 * i] = make_float4(hx, hy, hz, (float)b.w);
    x32[2 * i + 1] = make_float4((float)(dx - (double)hx), (float)(dy - (double)hy), (float)(dz - (double)hz), 0.f);
  }
}

// (hi, lo) += s, with s split into two floats and the hi sum made exact by TwoSum.
__device__ __forceinline__ void add_shift(float &hi, float &lo, double s) {
  const float sh = (float)s, sl = (float)(s - (double)sh);
  const float t = hi + sh;
  const float bb = t - hi;
  const float err = (hi - (t - bb)) + (sh - bb);
  hi = t;
  lo = (lo + err) + sl;
}

template <bool PERIODIC>
__device__ __forceinline__ void stage_body(Stage &sm, int k, const float4 *x32, long long body, int img, double cycle) {
  float4 h = x32[2 * body], l = x32[2 * body + 1];
  if (PERIODIC && img != 13) {
    add_shift(h.x, l.x, (double)(img / 9 - 1) * cycle);
    add_shift(h.y, l.y, (double)((img / 3) % 3 - 1) * cycle);
    add_shift(h.z, l.z, (double)(img % 3 - 1) * cycle);
  }
  const int p = k >> 1, o = k & 1;
  float *A = reinterpret_cast<float *>(&sm.A[p]);
  float *B = reinterpret_cast<float *>(&sm.B[p]);
  float *C = reinterpret_cast<float *>(&sm.C[p]);
  float *D = reinterpret_cast<float *>(&sm.D[p]);
  A[o] = h.x;
  A[2 + o] = h.y;
  B[o] = h.z;
  B[2 + o] = h.w;
  C[o] = l.x;
  C[2 + o] = l.y;
  D[o] = l.z;
}

// Padding source: far away with zero charge, so it adds exactly zero.
__device__ __forceinline__ void stage_dummy(Stage &sm, int k) {
  const int p = k >> 1, o = k & 1;
  float *A = reinterpret_cast<float *>(&sm.A[p]);
  float *B = reinterpret_cast<float *>(&sm.B[p]);
  float *C = reinterpret_cast<float *>(&sm.C[p]);
  float *D = reinterpret_cast<float *>(&sm.D[p]);
  A[o] = 1e18f;
  A[2 + o] = 1e18f;
  B[o] = 1e18f;
  B[2 + o] = 0.f;
  C[o] = 0.f;
  C[2 + o] = 0.f;
  D[o] = 0.f;
}

// Targets of one lane (TPL of them): t[u] = packed (hx, hy, hz, lx, ly, lz), each value in both halves.
template <int TPL>
struct Targets {
  f2p t[TPL][6];
};

template <int TPL>
struct Sums {
  Kahan k[TPL][4];  // potential, gradient x, y, z
};

// One pair step: two staged sources (pair p) against the lane's targets.
template <int TPL>
__device__ __forceinline__ void pair_step(const Stage &sm, int p, const Targets<TPL> &T, f2p (&pp)[TPL],
                                          f2p (&px)[TPL], f2p (&py)[TPL], f2p (&pz)[TPL]) {
  const float4 A = sm.A[p], B = sm.B[p], C = sm.C[p], D = sm.D[p];
  const f2p shx = pk2(A.x, A.y), shy = pk2(A.z, A.w), shz = pk2(B.x, B.y), w = pk2(B.z, B.w);
  const f2p slx = pk2(C.x, C.y), sly = pk2(C.z, C.w), slz = pk2(D.x, D.y);
#pragma unroll
  for (int u = 0; u < TPL; u++) {
    const f2p dx = add2(sub2(T.t[u][0], shx), sub2(T.t[u][3], slx));
    const f2p dy = add2(sub2(T.t[u][1], shy), sub2(T.t[u][4], sly));
    const f2p dz = add2(sub2(T.t[u][2], shz), sub2(T.t[u][5], slz));
    const f2p r2 = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
    const float2 rr = unpk2(r2);
    const float i0 = rr.x >= 1.17549435e-38f ? rsqrt_ftz(rr.x) : 0.f;
    const float i1 = rr.y >= 1.17549435e-38f ? rsqrt_ftz(rr.y) : 0.f;
    const f2p inv = pk2(i0, i1);
    const f2p qr = mul2(w, inv);
    const f2p qr3 = mul2(mul2(qr, inv), inv);
    pp[u] = add2(pp[u], qr);
    px[u] = fma2(dx, qr3, px[u]);
    py[u] = fma2(dy, qr3, py[u]);
    pz[u] = fma2(dz, qr3, pz[u]);
  }
}

// Streams the bodies of the P2P list entries [qb, qe) through the warp and
// accumulates their action on the lane's targets into `acc`.
template <int S, int TPL, bool PERIODIC>
__device__ __forceinline__ void p2p_stream(Stage &sm, const int *src, const int4 *cell_b, const float4 *x32,
                                           double cycle, int qb, int qe, const Targets<TPL> &T, Sums<TPL> &acc) {
  constexpr int G = 32 / S, CH = 32 * G;
  const int lane = threadIdx.x & 31, g = lane / S;
  int q = qb, o = 0, qw = qb - 64;
  int w_start = 0, w_size = 0, w_img = 13;
  for (;;) {
    // ---- fill one chunk (warp-uniform walk over the segments) ----
    int filled = 0;
    while (filled < CH && q < qe) {
      if (q - qw >= 32) {  // next window of 32 segment descriptors, one per lane
        qw = q;
        const int qq = qw + lane;
        w_start = 0;
        w_size = 0;
        w_img = 13;
        if (qq < qe) {
          const int packed = src[qq];
          const int4 cb = cell_b[packed & 0x3ffffff];
          w_start = cb.x;
          w_size = cb.y;
          w_img = packed >> 26;
        }
      }
      const int l = q - qw;
      const int start = __shfl_sync(kFull, w_start, l);
      const int size = __shfl_sync(kFull, w_size, l);
      const int img = PERIODIC ? __shfl_sync(kFull, w_img, l) : 13;
      const int m = min(CH - filled, size - o);
      for (int k = lane; k < m; k += 32) stage_body<PERIODIC>(sm, filled + k, x32, (long long)start + o + k, img, cycle);
      filled += m;
      o += m;
      if (o == size) {
        q++;
        o = 0;
      }
    }
    if (filled == 0) break;
    const int steps = (filled + 2 * G - 1) / (2 * G);  // pair steps per group
    const int padded = 2 * G * (steps + (steps & 1));   // even step count for the unrolled loop
    for (int k = filled + lane; k < padded; k += 32) stage_dummy(sm, k);
    __syncwarp();

    // ---- evaluate: group g takes pairs g, g + G, g + 2G, ... ----
    f2p pp[TPL], px[TPL], py[TPL], pz[TPL];
#pragma unroll
    for (int u = 0; u < TPL; u++) pp[u] = px[u] = py[u] = pz[u] = 0ull;
    for (int s = 0; s < steps; s += 2) {
      pair_step(sm, g + G * s, T, pp, px, py, pz);
      pair_step(sm, g + G * (s + 1), T, pp, px, py, pz);
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < TPL; u++) {
      const float2 a = unpk2(pp[u]), bx = unpk2(px[u]), by = unpk2(py[u]), bz = unpk2(pz[u]);
      acc.k[u][0].add(a.x + a.y);
      acc.k[u][1].add(bx.x + bx.y);
      acc.k[u][2].add(by.x + by.y);
      acc.k[u][3].add(bz.x + bz.y);
    }
  }
}

// One pass over the leaf's source stream for its targets [tb, tb + S * TPL).
template <int S, int TPL, bool PERIODIC>
__device__ __forceinline__ void p2p_pass(Stage &sm, int4 cb, int tb, int b, int e, const int *src,
                                         const int4 *cell_bj, const float4 *x32, const float4 *x32j, double4 *trg,
                                         double cycle) {
  const int lane = threadIdx.x & 31, g = lane / S, j = lane % S;
  {
    Targets<TPL> T;
#pragma unroll
    for (int u = 0; u < TPL; u++) {
      const int i = tb + j + S * u;
      float4 h = make_float4(0.f, 0.f, 0.f, 0.f), l = h;
      if (i < cb.y) {
        h = x32[2 * ((long long)cb.x + i)];
        l = x32[2 * ((long long)cb.x + i) + 1];
      }
      T.t[u][0] = pk2(h.x, h.x);
      T.t[u][1] = pk2(h.y, h.y);
      T.t[u][2] = pk2(h.z, h.z);
      T.t[u][3] = pk2(l.x, l.x);
      T.t[u][4] = pk2(l.y, l.y);
      T.t[u][5] = pk2(l.z, l.z);
    }
    Sums<TPL> acc;
    p2p_stream<S, TPL, PERIODIC>(sm, src, cell_bj, x32j, cycle, b, e, T, acc);
    // combine the groups (lanes j, j + S, j + 2S, ... hold the same targets) in FP64
#pragma unroll
    for (int u = 0; u < TPL; u++) {
      double v[4];
#pragma unroll
      for (int k = 0; k < 4; k++) v[k] = (double)acc.k[u][k].s - (double)acc.k[u][k].c;
#pragma unroll
      for (int off = S; off < 32; off <<= 1)
#pragma unroll
        for (int k = 0; k < 4; k++) v[k] += __shfl_xor_sync(kFull, v[k], off);
      const int i = tb + j + S * u;
      if (g == 0 && i < cb.y) {
        double4 r = trg[cb.x + i];
        r.x += v[0];
        r.y -= v[1];
        r.z -= v[2];
        r.w -= v[3];
        trg[cb.x + i] = r;
      }
    }
  }
}

// Target slots of a leaf: passes of S lanes x TPL targets per lane, each pass
// taking the narrowest group that holds the targets still left (S = 32 while
// more than 16 TPL remain).  A 70-body leaf at two per lane: 64 + 8 slots in
// two passes, rather than 96 at three per lane or 128 in two full passes.
// Every pass streams the leaf's sources again, which costs about as much as
// a few more target slots, so a leaf takes three targets per lane when that
// costs fewer slots plus passes.  The two kinds run as separate kernels, so
// the three-target code's registers do not lower the occupancy of the
// two-target one.
__host__ __device__ __forceinline__ int pass_lanes(int left, int tpl) {
  return left <= 4 * tpl ? 4 : left <= 8 * tpl ? 8 : left <= 16 * tpl ? 16 : 32;
}
constexpr int kPassCharge = 4;  // target slots one more stream of the sources costs
__host__ __device__ __forceinline__ int pass_cost(int n, int tpl) {
  int cost = 0;
  for (int tb = 0; tb < n;) {
    const int w = pass_lanes(n - tb, tpl) * tpl;
    cost += w + kPassCharge;
    tb += w;
  }
  return cost;
}
__device__ __forceinline__ bool three_per_lane(int n) { return pass_cost(n, 3) < pass_cost(n, 2); }

// Work order: each cell's kind (0: a leaf of two targets per lane, 1: three,
// 2: no P2P list; tpl 2 or 3 gives every leaf that kind, tpl 0 chooses by the
// leaf's size) above its cost (its bodies times the bodies of its list,
// capped), reversed so that an ascending sort puts the costliest leaf of
// each kind first.  count[kind] receives the cells of each kind.
constexpr int kCostBits = 22;
constexpr unsigned kCostMax = (1u << kCostBits) - 1;

__global__ void k_p2p_keys(const int *off, const int *src, long long ncells, const int4 *cell_b,
                           const int4 *cell_bj, int tpl, unsigned *key, int *val, int *count) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncells;
       c += (long long)gridDim.x * blockDim.x) {
    const int b = off[c], e = off[c + 1];
    unsigned kind = 2, cost = 0;
    if (b < e) {
      const int nb = cell_b[c].y;
      unsigned long long s = 0;
      for (int q = b; q < e; q++) s += (unsigned)cell_bj[src[q] & 0x3ffffff].y;
      kind = (tpl == 0 ? three_per_lane(nb) : tpl == 3) ? 1u : 0u;
      cost = (unsigned)min((unsigned long long)kCostMax, s * (unsigned long long)nb);
    }
    key[c] = (kind << kCostBits) | (kCostMax - cost);
    val[c] = (int)c;
    atomicAdd(&count[kind], 1);
  }
}

// Persistent one-warp blocks, as many as fit on the GPU; each takes the next
// target leaf of its kind from a counter, in the work order above (longest
// first), until none is left, so leaves of very different cost balance out
// and the warps finish together.  A leaf's result does not depend on when or
// by which warp it is evaluated.
// Resident warps per SM: the register budgets (96 and 126 registers, no
// spills) at which the two kinds measured fastest on a 512-system batch at
// P = 10 (P2P 55.3 -> 54.5 ms against 16 and 12 warps; the same on one 4M
// solve).
constexpr int kWarps2 = 20, kWarps3 = 16;

template <bool PERIODIC, int TPL>
__global__ void __launch_bounds__(32, TPL == 2 ? kWarps2 : kWarps3)
k_p2p32(const int *off, const int *src, const int *order, const int *count, const int4 *cell_b,
        const int4 *cell_bj, const float4 *x32, const float4 *x32j, double4 *trg, double cycle,
        unsigned long long *next) {
  __shared__ Stage sm;
  const long long items = count[TPL == 2 ? 0 : 1];
  const int *mine = order + (TPL == 2 ? 0 : count[0]);
  for (;;) {
    unsigned long long k = 0;
    if (threadIdx.x == 0) k = atomicAdd(next, 1ull);
    k = __shfl_sync(kFull, k, 0);
    if ((long long)k >= items) return;
    const int c = mine[k];
    const int b = off[c], e = off[c + 1];
    const int4 cb = cell_b[c];
    for (int tb = 0; tb < cb.y;) {
      const int left = cb.y - tb;
      if (left <= 4 * TPL) {
        p2p_pass<4, TPL, PERIODIC>(sm, cb, tb, b, e, src, cell_bj, x32, x32j, trg, cycle);
        tb += 4 * TPL;
      } else if (left <= 8 * TPL) {
        p2p_pass<8, TPL, PERIODIC>(sm, cb, tb, b, e, src, cell_bj, x32, x32j, trg, cycle);
        tb += 8 * TPL;
      } else if (left <= 16 * TPL) {
        p2p_pass<16, TPL, PERIODIC>(sm, cb, tb, b, e, src, cell_bj, x32, x32j, trg, cycle);
        tb += 16 * TPL;
      } else {
        p2p_pass<32, TPL, PERIODIC>(sm, cb, tb, b, e, src, cell_bj, x32, x32j, trg, cycle);
        tb += 32 * TPL;
      }
      __syncwarp();  // the stage buffer is free before the next pass's first fill
    }
  }
}

}  // namespace

void rel_bodies32(const FmmArgs &a, float4 *x32) { rel_bodies32(a, a.xt, a.n, x32); }

void rel_bodies32(const FmmArgs &a, const double4 *xt, long long n, float4 *x32) {
  if (n <= 0) return;
  long long g = (n + 255) / 256;
  if (g > kNumSMs * 16) g = kNumSMs * 16;
  if (a.nsys) k_abs32_forest<<<(int)g, 256, 0, a.stream>>>(xt, n, a.sys_off, a.nsys, a.sys_box, x32);
  else k_abs32<<<(int)g, 256, 0, a.stream>>>(xt, n, a.cell_x, x32);
  EXA_CHECK_LAUNCH();
}

void p2p_mixed(Context &C, const FmmArgs &a, const float4 *x32, bool periodic, P2PWork &w, const float4 *x32j) {
  const int4 *cell_bj = a.src_cell_b ? a.src_cell_b : a.cell_b;
  if (!x32j) x32j = x32;
  const long long nc = a.ncells;
  if (nc <= 0) return;
  cudaStream_t st = a.stream;
  w.next.ensure(2);
  w.count.ensure(3);
  w.key.ensure(nc);
  w.key_alt.ensure(nc);
  w.order.ensure(nc);
  w.order_alt.ensure(nc);
  EXA_CUDA(cudaMemsetAsync(w.next.p, 0, 2 * sizeof(unsigned long long), st));
  EXA_CUDA(cudaMemsetAsync(w.count.p, 0, 3 * sizeof(int), st));
  const int kg = (int)std::max<long long>(1, std::min<long long>((long long)kNumSMs * 8, (nc + 255) / 256));
  k_p2p_keys<<<kg, 256, 0, st>>>(a.p2p_off, a.p2p_src, nc, a.cell_b, cell_bj, C.prm.p2p_tpl, w.key.p, w.order.p,
                                 w.count.p);
  EXA_CHECK_LAUNCH();
  const bool alt = radix_sort_u32(w.key.p, w.order.p, w.key_alt.p, w.order_alt.p, nc, 0, kCostBits + 2, C.sort,
                                  C.err.p, st);
  const int *order = alt ? w.order_alt.p : w.order.p;
  const unsigned g2 = (unsigned)std::min<long long>(nc, (long long)kNumSMs * kWarps2);
  const unsigned g3 = (unsigned)std::min<long long>(nc, (long long)kNumSMs * kWarps3);
  if (!w.side) {
    int dev = 0;
    EXA_CUDA(cudaGetDevice(&dev));
    EXA_CUDA(cudaStreamCreateWithFlags(&w.side, cudaStreamNonBlocking));
    EXA_CUDA(cudaEventCreateWithFlags(&w.fork, cudaEventDisableTiming));
    EXA_CUDA(cudaEventCreateWithFlags(&w.join, cudaEventDisableTiming));
  }
  // the two kinds write disjoint target leaves; the side stream starts after
  // the work order is sorted and the solve's stream waits for it at the end
  EXA_CUDA(cudaEventRecord(w.fork, st));
  EXA_CUDA(cudaStreamWaitEvent(w.side, w.fork, 0));
  if (periodic) {
    k_p2p32<true, 2><<<g2, 32, 0, st>>>(a.p2p_off, a.p2p_src, order, w.count.p, a.cell_b, cell_bj, x32, x32j,
                                        a.trg64, a.cycle, w.next.p);
    EXA_CHECK_LAUNCH();
    k_p2p32<true, 3><<<g3, 32, 0, w.side>>>(a.p2p_off, a.p2p_src, order, w.count.p, a.cell_b, cell_bj, x32, x32j,
                                            a.trg64, a.cycle, w.next.p + 1);
  } else {
    k_p2p32<false, 2><<<g2, 32, 0, st>>>(a.p2p_off, a.p2p_src, order, w.count.p, a.cell_b, cell_bj, x32, x32j,
                                         a.trg64, a.cycle, w.next.p);
    EXA_CHECK_LAUNCH();
    k_p2p32<false, 3><<<g3, 32, 0, w.side>>>(a.p2p_off, a.p2p_src, order, w.count.p, a.cell_b, cell_bj, x32, x32j,
                                             a.trg64, a.cycle, w.next.p + 1);
  }
  EXA_CHECK_LAUNCH();
  EXA_CUDA(cudaEventRecord(w.join, w.side));
  EXA_CUDA(cudaStreamWaitEvent(st, w.join, 0));
}

}  // namespace exafmm_b200
