// Spherical-harmonic expansion math of kernels/laplace.h, in a trig-free
// Cartesian form.
//
// The reference evaluates, for a vector d with spherical angles (alpha, beta),
//   regular   Y_n^m  = rho^n      P_n^m(cos alpha) pref_n^m e^{i m beta}   (evalMultipole, laplace.h:48-80)
//   singular  Y2_n^m = rho^{-n-1} P_n^m(cos alpha) pref_n^m e^{i m beta}   (evalLocal,     laplace.h:83-113)
// with pref_n^m = sqrt((n-|m|)!/(n+|m|)!) and the Condon-Shortley phase in P.
// Both are computed here straight from (x, y, z) with the normalized three-term
// recurrences (no acos/atan2/exp):
//   Y_m^m     = Y_{m-1}^{m-1} * (-(x + i y)) * sqrt((2m-1)/(2m))
//   Y_{n+1}^m = a_n^m z Y_n^m - b_n^m rho^2 Y_{n-1}^m
//   a_n^m = (2n+1)/sqrt((n+1)^2-m^2),  b_n^m = sqrt((n^2-m^2)/((n+1)^2-m^2))
// and for the singular family the same recurrence divided by rho^2 with
// Y2_0^0 = 1/rho.  Expansions are stored for m >= 0 at index n(n+1)/2+m;
// negative orders are conjugates.
#pragma once
#include "common.cuh"

namespace exafmm_b200 {

// Device-side tables for one expansion order P (all FP64, n < 2P).
struct TransOp {
  double w;
  int a;  // source coefficient index | conj << 16
  int b;  // harmonic index | conj << 16
};

struct DevTables {
  int P;
  int nterm;            // P(P+1)/2
  const double *anm;    // A_n^m = (-1)^n / sqrt((n-m)!(n+m)!), index n*(n+1)/2+|m|
  const double *ainv;   // 1 / A_n^m
  const double *ra;     // a_n^m, index n*(n+1)/2+m
  const double *rb;     // b_n^m
  const double *rd;     // sqrt((2m-1)/(2m)), rd[0] = 1
  // Translation terms of M2M and L2L (laplace.h:254-290, 324-357) per output
  // coefficient o = tri(j) + k: terms [m2m_start[o], m2m_start[o + 1]) of
  // m2m_ops, each acc += src[a] * (Y[b] * w) with src or Y conjugated where
  // the flag in bit 16 of a or b is set; the sign and phase of the term are in w.
  const TransOp *m2m_ops;
  const int *m2m_start;
  const TransOp *l2l_ops;
  const int *l2l_start;
  // The output coefficients each lane of a warp sums in k_m2m: lane l takes
  // entries [l * MAXO, l * MAXO + MAXO) (-1: none), MAXO = ceil(NT / 32),
  // assigned longest first to the least loaded lane so that the lanes' term
  // counts are about equal (the warp waits for its busiest).
  const short *m2m_lane;
  // Work split of k_l2l over the 32 lanes of a warp.  Each output
  // coefficient's terms are cut into pieces of about the lanes' average share
  // (piece q: int4 (o, first term, end term, 0), pieces of one output
  // consecutive, [piece_start[o], piece_start[o + 1])); lane l sums the pieces
  // slot[l * slots + u] (-1: none), assigned longest first to the least
  // loaded lane, and an output is the sum of its pieces in order.  L2L needs
  // it: its (0, 0) coefficient sums every term.
  const int4 *l2l_piece;
  const int *l2l_piece_start;
  const short *l2l_slot;
  int l2l_slots, l2l_pieces;
  // L2P factors per (n, m), index tri(n) + m, n + 1 < P (laplace.h:359-388 as
  // restated in k_l2p): w_m sqrt((n+1)^2 - m^2), sqrt((n+m+2)(n+m+1)/2), and
  // -sqrt((n+1)n/2) (m = 1) or -sqrt((n+2-m)(n+1-m)/2) (m >= 2).
  const double *l2p_gz;
  const double *l2p_s1;
  const double *l2p_s2;
};

// Host construction (tables.cu).
struct HostTables;
const DevTables &device_tables(int P);

// Column m of the regular family for n = m .. nmax-1, written to Y[tri(n)+m].
// conj_phase selects e^{-i m beta} (P2M, M2M) instead of e^{+i m beta}.
__device__ __forceinline__ void regular_column(const DevTables &t, int m, int nmax, double x, double y, double z,
                                               bool conj_phase, double2 *Y) {
  const double r2 = x * x + y * y + z * z;
  const double yy = conj_phase ? -y : y;
  double2 w = make_double2(1.0, 0.0);
  for (int k = 1; k <= m; k++) {
    const double f = -t.rd[k];
    w = make_double2(f * (w.x * x - w.y * yy), f * (w.x * yy + w.y * x));
  }
  if (m >= nmax) return;
  Y[tri(m) + m] = w;
  double2 prev = make_double2(0.0, 0.0), cur = w;
  for (int n = m; n + 1 < nmax; n++) {
    const double a = t.ra[tri(n) + m], b = t.rb[tri(n) + m];
    double2 nxt = make_double2(a * z * cur.x - b * r2 * prev.x, a * z * cur.y - b * r2 * prev.y);
    Y[tri(n + 1) + m] = nxt;
    prev = cur;
    cur = nxt;
  }
}

// Column m of the singular family for n = m .. nmax-1, each scaled by scale[tri(n)+m]
// when scale is non-null.
__device__ __forceinline__ void singular_column(const DevTables &t, int m, int nmax, double x, double y, double z,
                                                const double *scale, double2 *Y) {
  const double r2 = x * x + y * y + z * z;
  const double inv_r2 = 1.0 / r2;
  double2 w = make_double2(rsqrt(r2), 0.0);
  for (int k = 1; k <= m; k++) {
    const double f = -t.rd[k] * inv_r2;
    w = make_double2(f * (w.x * x - w.y * y), f * (w.x * y + w.y * x));
  }
  if (m >= nmax) return;
  double s = scale ? scale[tri(m) + m] : 1.0;
  Y[tri(m) + m] = make_double2(w.x * s, w.y * s);
  double2 prev = make_double2(0.0, 0.0), cur = w;
  for (int n = m; n + 1 < nmax; n++) {
    const double a = t.ra[tri(n) + m] * inv_r2, b = t.rb[tri(n) + m] * inv_r2;
    double2 nxt = make_double2(a * z * cur.x - b * prev.x, a * z * cur.y - b * prev.y);
    s = scale ? scale[tri(n + 1) + m] : 1.0;
    Y[tri(n + 1) + m] = make_double2(nxt.x * s, nxt.y * s);
    prev = cur;
    cur = nxt;
  }
}

// Coefficient (n, m) for either sign of m from m >= 0 storage.
__device__ __forceinline__ double2 coef_any(const double2 *E, int n, int m) {
  return m >= 0 ? E[tri(n) + m] : cconj(E[tri(n) - m]);
}

__device__ __forceinline__ int sgn_pow(int e) { return (e & 1) ? -1 : 1; }

// (n, m) of a storage index o = n(n+1)/2 + m.
__device__ __forceinline__ void tri_decode(int o, int &n, int &m) {
  n = (int)((sqrt(8.0 * o + 1.0) - 1.0) * 0.5);
  while (tri(n + 1) <= o) n++;
  while (tri(n) > o) n--;
  m = o - tri(n);
}

}  // namespace exafmm_b200
