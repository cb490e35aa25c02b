// Register-resident M2L for a fixed expansion order P (kernels/laplace.h:292-322).
//
//   L_j^k = (-1)^j A_j^k R_t^{-(j+1)} sum_{n,m} s(k,m) M''_n^m S'_{j+n}^{m-k}(d / R_t)
//   M''_n^m = A_n^m M_n^m R_t^{-n},   S'_p^q = Y2_p^q / A_p^q,
//   s = +1 (m < 0), (-1)^m (0 <= m <= k), (-1)^k (m > k)
// which is the reference's Cnm contraction with every factor moved to one side.
//
// One warp serves one target cell; each lane takes whole source cells of the
// target's list.  For one (target, source) pair a lane holds the source's
// scaled multipole M'' and the target's partial local expansion in registers
// and generates the singular harmonics S' column by column (fixed order q,
// degree p rising) with the three-term recurrence, using each value at once
// for every (j, k, n, m) it feeds -- no shared-memory traffic in the inner
// product.
//
// The straight-line code is generated from a constexpr list of operations
// (diagonal step, recurrence step, complex multiply-add), expanded by an
// index_sequence fold, so every register index is a compile-time constant and
// nothing depends on the compiler's unrolling heuristics.  To bound register
// use, a pair's work can be split over warps by output degree j in [J0, J1)
// and source degree n in [N0, N1).
#pragma once
#include <utility>

#include "common.cuh"

namespace exafmm_b200 {

template <typename T> struct Cx { T x, y; };

// Recurrence tables (a, b, diagonal factor, 1/A) in constant memory.
template <typename T> struct RecTab {
  T ra[(2 * kMaxP) * (2 * kMaxP + 1) / 2];
  T rb[(2 * kMaxP) * (2 * kMaxP + 1) / 2];
  T rd[2 * kMaxP + 1];
  T ainv[(2 * kMaxP) * (2 * kMaxP + 1) / 2];
};

constexpr int ctri(int n) { return n * (n + 1) / 2; }
constexpr int cabs(int v) { return v < 0 ? -v : v; }
constexpr int cmax(int a, int b) { return a > b ? a : b; }
constexpr int cmin(int a, int b) { return a < b ? a : b; }

// One generated operation.
//   kind 0: diagonal step to column c            (a = c)
//   kind 1: recurrence step to degree p, column c (a = p, b = c)
//   kind 2: acc[a] += sg * M[b]^(mconj) * S^(sconj)
struct M2LOp {
  int kind, a, b, c;
  int mconj, sconj, neg;
};

template <int P, int J0, int J1, int N0, int N1>
struct M2LProgram {
  static constexpr int PMAX = (J1 - 1) + (N1 - 1);

  template <typename Emit>
  static constexpr int walk(Emit emit) {
    int count = 0;
    for (int c = 0; c <= PMAX; c++) {
      emit(count++, M2LOp{0, c, 0, 0, 0, 0, 0});
      for (int p = c; p <= PMAX; p++) {
        emit(count++, M2LOp{1, p, c, 0, 0, 0, 0});
        for (int sgn = 1; sgn >= -1; sgn -= 2) {
          if (sgn < 0 && c == 0) continue;
          const int q = sgn * c;
          for (int j = cmax(J0, p - (N1 - 1)); j <= cmin(J1 - 1, p - N0); j++) {
            const int n = p - j;
            for (int k = cmax(0, -n - q); k <= cmin(j, n - q); k++) {
              const int m = q + k;
              const int neg = (m < 0) ? 0 : ((m <= k) ? (m & 1) : (k & 1));
              emit(count++, M2LOp{2, ctri(j) - ctri(J0) + k, ctri(n) - ctri(N0) + cabs(m), 0, m < 0 ? 1 : 0,
                                  sgn < 0 ? 1 : 0, neg});
            }
          }
        }
      }
    }
    return count;
  }

  struct Counter {
    constexpr void operator()(int, M2LOp) const {}
  };
  static constexpr int size = walk(Counter{});

  struct Table {
    M2LOp ops[size];
  };
  struct Filler {
    Table *t;
    constexpr void operator()(int i, M2LOp o) const { t->ops[i] = o; }
  };
  static constexpr Table make() {
    Table t{};
    walk(Filler{&t});
    return t;
  }
  static constexpr Table table = make();
};

template <typename T>
__host__ __device__ __forceinline__ T inv_sqrt(T v) {
#ifdef __CUDA_ARCH__
  return rsqrt(v);
#else
  return T(1) / sqrt(v);
#endif
}

template <typename T>
struct M2LState {
  T x, y, z, inv_r2;
  Cx<T> diag, prev, cur, sp;
};

template <typename T, typename Prog, int I, int NM, int NA>
__host__ __device__ __forceinline__ void m2l_step(const RecTab<T> &tab, const Cx<T> (&Mv)[NM], Cx<T> (&acc)[NA],
                                         M2LState<T> &s) {
  constexpr M2LOp op = Prog::table.ops[I];
  if constexpr (op.kind == 0) {
    // A warp barrier per column keeps the scheduler from running the whole
    // recurrence ahead of its uses (which would hold every S' value live).
#ifdef __CUDA_ARCH__
    __syncwarp();
#endif
    if constexpr (op.a > 0) {
      const T f = -tab.rd[op.a] * s.inv_r2;
      const Cx<T> d0 = s.diag;
      s.diag.x = f * (d0.x * s.x - d0.y * s.y);
      s.diag.y = f * (d0.x * s.y + d0.y * s.x);
    }
  } else if constexpr (op.kind == 1) {
    if constexpr (op.a == op.b) {
      s.prev = Cx<T>{T(0), T(0)};
      s.cur = s.diag;
    } else {
      const T a = tab.ra[ctri(op.a - 1) + op.b] * s.inv_r2;
      const T b = tab.rb[ctri(op.a - 1) + op.b] * s.inv_r2;
      Cx<T> nxt;
      nxt.x = a * s.z * s.cur.x - b * s.prev.x;
      nxt.y = a * s.z * s.cur.y - b * s.prev.y;
      s.prev = s.cur;
      s.cur = nxt;
    }
    const T sc = tab.ainv[ctri(op.a) + op.b];
    s.sp.x = s.cur.x * sc;
    s.sp.y = s.cur.y * sc;
  } else {
    // acc += (+/-) M^(conj) * S^(conj), signs folded into the FMAs
    const T mx = Mv[op.b].x, my = op.mconj ? -Mv[op.b].y : Mv[op.b].y;
    const T sx = s.sp.x, sy = op.sconj ? -s.sp.y : s.sp.y;
    Cx<T> &a = acc[op.a];
    if constexpr (op.neg) {
      a.x = fma(-mx, sx, a.x);
      a.x = fma(my, sy, a.x);
      a.y = fma(-mx, sy, a.y);
      a.y = fma(-my, sx, a.y);
    } else {
      a.x = fma(mx, sx, a.x);
      a.x = fma(-my, sy, a.x);
      a.y = fma(mx, sy, a.y);
      a.y = fma(my, sx, a.y);
    }
  }
}

template <typename T, typename Prog, int NM, int NA, size_t... I>
__host__ __device__ __forceinline__ void m2l_run(const RecTab<T> &tab, const Cx<T> (&Mv)[NM], Cx<T> (&acc)[NA],
                                        M2LState<T> &s, std::index_sequence<I...>) {
  (m2l_step<T, Prog, (int)I, NM, NA>(tab, Mv, acc, s), ...);
}

// ---- FP32 on the device: packed f32x2 arithmetic (sm_100) ----
// A complex multiply-add acc += M * S is two packed FMAs on (re, im) pairs:
//   acc += (mx, mx) * (sx, sy) + (my, my) * (-sy, sx)
// with the operand signs of the conjugated / negated variants folded into the
// packed S operands, which are formed once per S' value and reused by every
// multiply-add that needs them.
typedef unsigned long long f2p;

__device__ __forceinline__ f2p pk2(float a, float b) {
  f2p r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void ffma2(f2p &acc, f2p a, f2p b) {
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(a), "l"(b));
}
__device__ __forceinline__ float2 unpk2(f2p v) {
  float a, b;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
  return make_float2(a, b);
}

struct M2LStateF2 {
  float x, y, z, inv_r2;
  Cx<float> diag, prev, cur, sp;
  // packed S' operand variants: v1[conj][neg], v2[conj][flip]
  f2p v1[2][2], v2[2][2];
};

template <typename Prog, int I, int NM, int NA>
__device__ __forceinline__ void m2l_step_f2(const RecTab<float> &tab, const f2p (&Mxx)[NM], const f2p (&Myy)[NM],
                                            f2p (&acc)[NA], M2LStateF2 &s) {
  constexpr M2LOp op = Prog::table.ops[I];
  if constexpr (op.kind == 0) {
    __syncwarp();
    if constexpr (op.a > 0) {
      const float f = -tab.rd[op.a] * s.inv_r2;
      const Cx<float> d0 = s.diag;
      s.diag.x = f * (d0.x * s.x - d0.y * s.y);
      s.diag.y = f * (d0.x * s.y + d0.y * s.x);
    }
  } else if constexpr (op.kind == 1) {
    if constexpr (op.a == op.b) {
      s.prev = Cx<float>{0.f, 0.f};
      s.cur = s.diag;
    } else {
      const float a = tab.ra[ctri(op.a - 1) + op.b] * s.inv_r2;
      const float b = tab.rb[ctri(op.a - 1) + op.b] * s.inv_r2;
      Cx<float> nxt;
      nxt.x = a * s.z * s.cur.x - b * s.prev.x;
      nxt.y = a * s.z * s.cur.y - b * s.prev.y;
      s.prev = s.cur;
      s.cur = nxt;
    }
    const float sc = tab.ainv[ctri(op.a) + op.b];
    const float sx = s.cur.x * sc, sy = s.cur.y * sc;
    // S = (sx, sy); conj S = (sx, -sy).  v1 = +-S^c, v2 = +-(-Im S^c, Re S^c).
    s.v1[0][0] = pk2(sx, sy);
    s.v1[0][1] = pk2(-sx, -sy);
    s.v1[1][0] = pk2(sx, -sy);
    s.v1[1][1] = pk2(-sx, sy);
    s.v2[0][0] = pk2(-sy, sx);
    s.v2[0][1] = pk2(sy, -sx);
    s.v2[1][0] = pk2(sy, sx);
    s.v2[1][1] = pk2(-sy, -sx);
  } else {
    // term = sgn * (mx + i my') * S^c, my' = -my when mconj
    //      = mx * (sgn S^c) + my * (sgn * (mconj ? -1 : 1) * (-Im S^c, Re S^c))
    constexpr int flip = op.neg ^ op.mconj;
    ffma2(acc[op.a], Mxx[op.b], s.v1[op.sconj][op.neg]);
    ffma2(acc[op.a], Myy[op.b], s.v2[op.sconj][flip]);
  }
}

template <typename Prog, int NM, int NA, size_t... I>
__device__ __forceinline__ void m2l_run_f2(const RecTab<float> &tab, const f2p (&Mxx)[NM], const f2p (&Myy)[NM],
                                           f2p (&acc)[NA], M2LStateF2 &s, std::index_sequence<I...>) {
  (m2l_step_f2<Prog, (int)I, NM, NA>(tab, Mxx, Myy, acc, s), ...);
}

// FP32 pair on the device with packed arithmetic; acc holds (re, im) pairs.
template <int P, int J0, int J1, int N0, int N1>
__device__ __forceinline__ void m2l_pair_f32x2(const RecTab<float> &tab, const f2p (&Mxx)[ctri(N1) - ctri(N0)],
                                               const f2p (&Myy)[ctri(N1) - ctri(N0)],
                                               f2p (&acc)[ctri(J1) - ctri(J0)], float x, float y, float z) {
  using Prog = M2LProgram<P, J0, J1, N0, N1>;
  M2LStateF2 s;
  s.x = x;
  s.y = y;
  s.z = z;
  const float r2 = x * x + y * y + z * z;
  s.inv_r2 = 1.f / r2;
  s.diag = Cx<float>{rsqrtf(r2), 0.f};
  s.prev = s.cur = s.sp = Cx<float>{0.f, 0.f};
  m2l_run_f2<Prog>(tab, Mxx, Myy, acc, s, std::make_index_sequence<Prog::size>{});
}

// Accumulate one pair: outputs j in [J0, J1), source degrees n in [N0, N1).
// Mv holds M''_n^m (m >= 0) for n in [N0, N1) at index ctri(n) - ctri(N0) + m;
// acc holds outputs (j, k) at ctri(j) - ctri(J0) + k; (x, y, z) = d / R_t.
template <typename T, int P, int J0, int J1, int N0, int N1>
__host__ __device__ __forceinline__ void m2l_pair_unrolled(const RecTab<T> &tab, const Cx<T> (&Mv)[ctri(N1) - ctri(N0)],
                                                  Cx<T> (&acc)[ctri(J1) - ctri(J0)], T x, T y, T z) {
  using Prog = M2LProgram<P, J0, J1, N0, N1>;
  M2LState<T> s;
  s.x = x;
  s.y = y;
  s.z = z;
  const T r2 = x * x + y * y + z * z;
  s.inv_r2 = T(1) / r2;
  s.diag = Cx<T>{inv_sqrt(r2), T(0)};
  s.prev = s.cur = s.sp = Cx<T>{T(0), T(0)};
  m2l_run<T, Prog>(tab, Mv, acc, s, std::make_index_sequence<Prog::size>{});
}

}  // namespace exafmm_b200
