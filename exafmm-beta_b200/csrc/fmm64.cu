// FP64 expansion operators: P2M, M2M, M2L, L2L, L2P, P2P (kernels/laplace.h:150-388),
// one warp per cell, in the conventions of harmonics.cuh.
#include <algorithm>

#include "fmm.h"
#include "harmonics.cuh"

namespace exafmm_b200 {
namespace {

constexpr int kWarpsPerBlock = 4;

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 acc) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
  return acc;
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void image_shift(int img, double cycle, double &sx, double &sy, double &sz) {
  sx = (double)(img / 9 - 1) * cycle;
  sy = (double)((img / 3) % 3 - 1) * cycle;
  sz = (double)(img % 3 - 1) * cycle;
}

// ---------------------------------------------------------------- P2M
// M_n^m = sum_b q_b conj(Y_n^m(x_b - X_c)) (laplace.h:237-252); lanes take
// bodies.  The terms come out of the recurrence in (m, n) order; each lane
// stages its body's terms for a window of 16 of them in shared memory, then
// lane l adds component l / 16 of window term l % 16 over the bodies (four
// running sums over the bodies mod 4, added pairwise): one load and one add a
// body and double, where a shuffle tree costs five of each.  The cell's sums
// are kept in that (m, n) order and written out at tri(n) + m.
constexpr int kP2mWin = 16;
constexpr int kP2mRow = kP2mWin + 1;  // odd stride in double2: lane rows hit distinct banks

__device__ __forceinline__ void p2m_flush(const double2 *stage, double *acc, int lane, int cols, int rows) {
  __syncwarp();
  const int j = lane & (kP2mWin - 1);
  if (j < cols) {
    const double *col = reinterpret_cast<const double *>(stage) + 2 * j + (lane >> 4);
    constexpr int RS = 2 * kP2mRow;
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    int r = 0;
    for (; r + 4 <= rows; r += 4) {
      a0 += col[r * RS];
      a1 += col[(r + 1) * RS];
      a2 += col[(r + 2) * RS];
      a3 += col[(r + 3) * RS];
    }
    for (; r < rows; r++) a0 += col[r * RS];
    acc[2 * j + (lane >> 4)] += (a0 + a1) + (a2 + a3);
  }
  __syncwarp();
}

__global__ void k_p2m(DevTables t, const int4 *cell_b, const double4 *cell_x, const double4 *xt, double2 *M,
                      long long ncells) {
  extern __shared__ double2 sh[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int P = t.P, NT = t.nterm;
  double *ra = reinterpret_cast<double *>(sh);  // block: the recurrence's a_n^m, b_n^m and rd
  double *rb = ra + NT;
  double *rd = rb + NT;
  for (int o = threadIdx.x; o < NT; o += blockDim.x) {
    ra[o] = t.ra[o];
    rb[o] = t.rb[o];
  }
  for (int m = threadIdx.x; m < P; m += blockDim.x) rd[m] = t.rd[m];
  __syncthreads();
  double2 *acc = sh + NT + (P + 1) / 2 + warp * (NT + 32 * kP2mRow);  // (m, n) order
  double2 *stage = acc + NT;
  double2 *mine = stage + lane * kP2mRow;
  double *accd = reinterpret_cast<double *>(acc);
  for (long long c = (long long)blockIdx.x * kWarpsPerBlock + warp; c < ncells;
       c += (long long)gridDim.x * kWarpsPerBlock) {
    const int4 cb = cell_b[c];
    if (cb.w != 0) continue;
    const double4 X = cell_x[c];
    for (int s = lane; s < NT; s += 32) acc[s] = make_double2(0.0, 0.0);
    for (int base = 0; base < cb.y; base += 32) {
      const int i = base + lane, rows = min(32, cb.y - base);
      double x = 0, y = 0, z = 0, q = 0;
      if (i < cb.y) {
        const double4 b = xt[cb.x + i];
        x = b.x - X.x;
        y = b.y - X.y;
        z = b.z - X.z;
        q = b.w;
      }
      const double r2 = x * x + y * y + z * z;
      double2 w = make_double2(q, 0.0);  // q * diagonal, with e^{-i m beta}
      int k = 0, win = 0;
      for (int m = 0; m < P; m++) {
        if (m > 0) {
          const double f = -rd[m];
          w = make_double2(f * (w.x * x + w.y * y), f * (w.y * x - w.x * y));
        }
        double2 prev = make_double2(0.0, 0.0), cur = w;
        for (int n = m; n < P; n++) {
          mine[k] = cur;
          if (++k == kP2mWin) {
            p2m_flush(stage, accd + 2 * win, lane, kP2mWin, rows);
            win += kP2mWin;
            k = 0;
          }
          if (n + 1 < P) {
            const double a = ra[tri(n) + m], b = rb[tri(n) + m];
            double2 nxt = make_double2(a * z * cur.x - b * r2 * prev.x, a * z * cur.y - b * r2 * prev.y);
            prev = cur;
            cur = nxt;
          }
        }
      }
      if (k) p2m_flush(stage, accd + 2 * win, lane, k, rows);
    }
    __syncwarp();
    for (int s = lane; s < NT; s += 32) {
      int m = 0, r = s;
      while (r >= P - m) {
        r -= P - m;
        m++;
      }
      M[c * NT + tri(m + r) + m] = acc[s];
    }
    __syncwarp();
  }
}

// acc + sum over terms [b, e) of src[a] * (Y[b] * w), conjugations per flag (DevTables::m2m_ops).
__device__ __forceinline__ double2 trans_sum(const TransOp *ops, int b, int e, const double2 *src, const double2 *Y,
                                             double2 a) {
  for (int i = b; i < e; i++) {
    const TransOp op = ops[i];
    double2 s = src[op.a & 0xffff];
    if (op.a >> 16) s.y = -s.y;
    double2 z = Y[op.b & 0xffff];
    if (op.b >> 16) z.y = -z.y;
    a = cfma(s, cscale(z, op.w), a);
  }
  return a;
}

// ---------------------------------------------------------------- M2M
// One child's contribution to the lane's parent coefficients (laplace.h:254-290):
// Y = regular harmonics of X_parent - X_child, Mc = the child's multipole.
template <int MAXO>
__device__ __forceinline__ void m2m_accumulate(const DevTables &t, const int (&oj)[MAXO], const int (&ok)[MAXO],
                                               const double2 *Y, const double2 *Mc, double2 (&acc)[MAXO]) {
#pragma unroll
  for (int u = 0; u < MAXO; u++) {
    const int j = oj[u], k = ok[u];
    if (j < 0) continue;
    acc[u] = trans_sum(t.m2m_ops, t.m2m_start[tri(j) + k], t.m2m_start[tri(j) + k + 1], Mc, Y, acc[u]);
  }
}

// Parent M from each child in child order (laplace.h:254-290), d = X_parent - X_child.
template <int MAXO>
__global__ void k_m2m(DevTables t, const long long *lvl, int level, const int *nd_cell, const int4 *cell_b,
                      const double4 *cell_x, double2 *M) {
  extern __shared__ double2 sh[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int P = t.P, NT = t.nterm;
  double2 *Y = sh + warp * 2 * NT;
  double2 *Mc = Y + NT;
  const long long cnt = lvl[level], start = lvl[kMaxLevels + 1 + level];
  int oj[MAXO], ok[MAXO];
#pragma unroll
  for (int u = 0; u < MAXO; u++) {
    const int o = t.m2m_lane[lane * MAXO + u];
    if (o >= 0) tri_decode(o, oj[u], ok[u]);
    else oj[u] = ok[u] = -1;
  }
  for (long long i = (long long)blockIdx.x * kWarpsPerBlock + warp; i < cnt; i += (long long)gridDim.x * kWarpsPerBlock) {
    const int c = nd_cell[start + i];
    const int4 cb = cell_b[c];
    if (cb.w == 0) continue;
    const double4 Xp = cell_x[c];
    double2 acc[MAXO];
#pragma unroll
    for (int u = 0; u < MAXO; u++) acc[u] = make_double2(0.0, 0.0);
    for (int ch = cb.z; ch < cb.z + cb.w; ch++) {
      const double4 Xc = cell_x[ch];
      const double dx = Xp.x - Xc.x, dy = Xp.y - Xc.y, dz = Xp.z - Xc.z;
      if (lane < P) regular_column(t, lane, P, dx, dy, dz, true, Y);
      for (int o = lane; o < NT; o += 32) Mc[o] = M[(long long)ch * NT + o];
      __syncwarp();
      m2m_accumulate<MAXO>(t, oj, ok, Y, Mc, acc);
      __syncwarp();
    }
#pragma unroll
    for (int u = 0; u < MAXO; u++)
      if (oj[u] >= 0) M[(long long)c * NT + tri(oj[u]) + ok[u]] = acc[u];
  }
}

// ---------------------------------------------------------------- M2L
// One source's contribution to the lane's target coefficients: Mp = A M of the
// source, S = singular harmonics of d over A (singular_column with t.ainv).
template <int MAXO>
__device__ __forceinline__ void m2l_accumulate(const DevTables &t, const int (&oj)[MAXO], const int (&ok)[MAXO],
                                               const double2 *Mp, const double2 *S, double2 (&acc)[MAXO]) {
  const int P = t.P;
#pragma unroll
  for (int u = 0; u < MAXO; u++) {
    const int j = oj[u], k = ok[u];
    if (j < 0) continue;
    double2 a = acc[u];
    for (int n = 0; n < P; n++) {
      const int p = j + n;
      for (int m = -n; m <= n; m++) {
        const double2 Mv = m >= 0 ? Mp[tri(n) + m] : cconj(Mp[tri(n) - m]);
        const int qq = m - k;
        const double2 Sv = qq >= 0 ? S[tri(p) + qq] : cconj(S[tri(p) - qq]);
        const double s = (m < 0) ? 1.0 : (m <= k ? (double)sgn_pow(m) : (double)sgn_pow(k));
        a = cfma(cscale(Mv, s), Sv, a);
      }
    }
    acc[u] = a;
  }
}

// L_j^k += (-1)^j A_j^k sum_{n,m} s(k,m) (A_n^m M_n^m) (Y2_{j+n}^{m-k} / A_{j+n}^{m-k})
// which is the reference's Cnm product (laplace.h:137-147, 292-322) with the
// sign s = +1 (m < 0), (-1)^m (0 <= m <= k), (-1)^k (m > k).
template <int MAXO>
__global__ void k_m2l(DevTables t, const int *off, const int *src, long long ncells, const double4 *cell_x,
                      const double4 *cell_xj, const double2 *M, double2 *L, double cycle, const int2 *cell_pl,
                      const int2 *cell_plj, int skip_min_level, int skip_max_dl) {
  extern __shared__ double2 sh[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int P = t.P, NT = t.nterm, NS = tri(2 * P - 1);
  double2 *Mp = sh + warp * (NT + NS);
  double2 *S = Mp + NT;
  int oj[MAXO], ok[MAXO];
#pragma unroll
  for (int u = 0; u < MAXO; u++) {
    const int o = lane + 32 * u;
    if (o < NT) tri_decode(o, oj[u], ok[u]);
    else oj[u] = ok[u] = -1;
  }
  for (long long c = (long long)blockIdx.x * kWarpsPerBlock + warp; c < ncells; c += (long long)gridDim.x * kWarpsPerBlock) {
    const int b = off[c], e = off[c + 1];
    if (b == e) continue;
    const double4 Xi = cell_x[c];
    double2 acc[MAXO];
#pragma unroll
    for (int u = 0; u < MAXO; u++) acc[u] = make_double2(0.0, 0.0);
    const int lt = cell_pl ? cell_pl[c].y : 0;
    for (int q = b; q < e; q++) {
      const int packed = src[q];
      const int cj = packed & 0x3ffffff, img = packed >> 26;
      if (cell_pl) {
        // pairs the mixed-precision kernel takes are skipped here
        const int dl = lt - cell_plj[cj].y;
        if (lt >= skip_min_level && dl <= skip_max_dl && dl >= -skip_max_dl) continue;
      }
      double sx, sy, sz;
      image_shift(img, cycle, sx, sy, sz);
      const double4 Xj = cell_xj[cj];
      const double dx = Xi.x - Xj.x - sx, dy = Xi.y - Xj.y - sy, dz = Xi.z - Xj.z - sz;
      for (int o = lane; o < NT; o += 32) Mp[o] = cscale(M[(long long)cj * NT + o], t.anm[o]);
      for (int m = lane; m < 2 * P - 1; m += 32) singular_column(t, m, 2 * P - 1, dx, dy, dz, t.ainv, S);
      __syncwarp();
      m2l_accumulate<MAXO>(t, oj, ok, Mp, S, acc);
      __syncwarp();
    }
#pragma unroll
    for (int u = 0; u < MAXO; u++) {
      const int j = oj[u], k = ok[u];
      if (j < 0) continue;
      const int o = tri(j) + k;
      const double w = sgn_pow(j) * t.anm[o];
      double2 *dst = &L[(long long)c * NT + o];
      *dst = cadd(*dst, cscale(acc[u], w));
    }
  }
}

// ---------------------------------------------------------------- L2L
// Child L from its parent (laplace.h:324-357), d = X_child - X_parent.
template <int MI>
__global__ void k_l2l(DevTables t, const long long *lvl, int level, const int *nd_cell, const int2 *cell_pl,
                      const double4 *cell_x, double2 *L) {
  extern __shared__ double2 sh[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int P = t.P, NT = t.nterm;
  double2 *Y = sh + warp * (2 * NT + 32 * MI);
  double2 *Lp = Y + NT;
  double2 *part = Lp + NT;  // the warp's piece sums
  const long long cnt = lvl[level], start = lvl[kMaxLevels + 1 + level];
  int pid[MI], pb[MI], pe[MI];
#pragma unroll
  for (int u = 0; u < MI; u++) {
    pid[u] = t.l2l_slot[lane * MI + u];
    pb[u] = pe[u] = 0;
    if (pid[u] >= 0) {
      const int4 pc = t.l2l_piece[pid[u]];
      pb[u] = pc.y;
      pe[u] = pc.z;
    }
  }
  for (long long i = (long long)blockIdx.x * kWarpsPerBlock + warp; i < cnt; i += (long long)gridDim.x * kWarpsPerBlock) {
    const int c = nd_cell[start + i];
    const int p = cell_pl[c].x;
    const double4 Xc = cell_x[c], Xp = cell_x[p];
    const double dx = Xc.x - Xp.x, dy = Xc.y - Xp.y, dz = Xc.z - Xp.z;
    if (lane < P) regular_column(t, lane, P, dx, dy, dz, false, Y);
    for (int o = lane; o < NT; o += 32) Lp[o] = L[(long long)p * NT + o];
    __syncwarp();
#pragma unroll
    for (int u = 0; u < MI; u++)
      if (pid[u] >= 0) part[pid[u]] = trans_sum(t.l2l_ops, pb[u], pe[u], Lp, Y, make_double2(0.0, 0.0));
    __syncwarp();
    for (int o = lane; o < NT; o += 32) {
      const int q0 = t.l2l_piece_start[o], q1 = t.l2l_piece_start[o + 1];
      double2 v = part[q0];
      for (int q = q0 + 1; q < q1; q++) v = cadd(v, part[q]);
      double2 *dst = &L[(long long)c * NT + o];
      *dst = cadd(*dst, v);
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------- L2P
// Potential and gradient of the local expansion at each body (laplace.h:359-388),
// evaluated as the j <= 1 terms of the expansion re-centered on the body:
//   pot = sum w_m Re(L_n^m Y_n^m),  w_0 = 1, w_m = 2
//   dz  = sum_{m<n} w_m sqrt(n^2-m^2) Re(L_n^m Y_{n-1}^m)
//   L11 = sum_n [ sum_{m=1..n} L_n^m Y_{n-1}^{m-1} s(n,m) - L_n^0 conj(Y_{n-1}^1) s(n,0)
//               - sum_{u=1..n-2} conj(L_n^u) conj(Y_{n-1}^{u+1}) s(n,-u) ],  s(n,m) = sqrt((n+m)(n+m-1)/2)
//   dx  = -sqrt(2) Re L11,  dy = sqrt(2) Im L11
// This has no 1/sin(theta) factor, so no offset of the body from the cell center is needed.
// Per leaf, the products of its local expansion that do not depend on the
// body are formed once in shared memory (per term o = (n, m)):
//   W = w_m L_n^m,  G = gz_o L_{n+1}^m,  A = s1_o L_{n+1}^{m+1},
//   B = s2_o L_{n+1}^0 (m = 1) or s2_o conj(L_{n+1}^{m-1}) (m >= 2),
// so a body's pass over the terms is four complex products with its regular
// harmonic and the recurrence, from shared memory only (the recurrence
// coefficients are staged once per block).
__global__ void k_l2p(DevTables t, const int4 *cell_b, const double4 *cell_x, const double4 *xt, const double2 *L,
                      double4 *trg, long long ncells) {
  extern __shared__ double2 sh[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int P = t.P, NT = t.nterm;
  double *ra = reinterpret_cast<double *>(sh);  // block: a_n^m, b_n^m, then rd
  double *rb = ra + NT;
  double *rd = rb + NT;
  double2 *Wc = sh + NT + (P + 1) / 2 + warp * 4 * NT;
  double2 *Gc = Wc + NT, *Ac = Gc + NT, *Bc = Ac + NT;
  for (int o = threadIdx.x; o < NT; o += blockDim.x) {
    ra[o] = t.ra[o];
    rb[o] = t.rb[o];
  }
  for (int m = threadIdx.x; m < P; m += blockDim.x) rd[m] = t.rd[m];
  __syncthreads();
  for (long long c = (long long)blockIdx.x * kWarpsPerBlock + warp; c < ncells; c += (long long)gridDim.x * kWarpsPerBlock) {
    const int4 cb = cell_b[c];
    if (cb.w != 0) continue;
    const double4 X = cell_x[c];
    const double2 *Lg = L + c * NT;
    for (int o = lane; o < NT; o += 32) {
      int n, m;
      tri_decode(o, n, m);
      const double2 Lnm = Lg[o];
      Wc[o] = m == 0 ? Lnm : cscale(Lnm, 2.0);
      double2 g = make_double2(0.0, 0.0), a = g, b = g;
      if (n + 1 < P) {
        g = cscale(Lg[tri(n + 1) + m], t.l2p_gz[o]);
        a = cscale(Lg[tri(n + 1) + m + 1], t.l2p_s1[o]);
        if (m == 1) b = cscale(Lg[tri(n + 1)], t.l2p_s2[o]);
        else if (m >= 2) b = cscale(cconj(Lg[tri(n + 1) + m - 1]), t.l2p_s2[o]);
      }
      Gc[o] = g;
      Ac[o] = a;
      Bc[o] = b;
    }
    __syncwarp();
    for (int i = lane; i < cb.y; i += 32) {
      const double4 bd = xt[cb.x + i];
      const double x = bd.x - X.x, y = bd.y - X.y, z = bd.z - X.z;
      const double r2 = x * x + y * y + z * z;
      double pot = 0, gz = 0;
      double2 l11 = make_double2(0.0, 0.0);
      double2 diag = make_double2(1.0, 0.0);
      for (int m = 0; m < P; m++) {
        if (m > 0) {
          const double f = -rd[m];
          diag = make_double2(f * (diag.x * x - diag.y * y), f * (diag.x * y + diag.y * x));
        }
        double2 prev = make_double2(0.0, 0.0), cur = diag;
        for (int n = m; n < P; n++) {
          // cur = Y_n^m
          const int o = tri(n) + m;
          const double2 w = Wc[o];
          pot += w.x * cur.x - w.y * cur.y;
          if (n + 1 < P) {
            const double2 g = Gc[o];
            gz += g.x * cur.x - g.y * cur.y;
            l11 = cfma(Ac[o], cur, l11);
            if (m >= 1) l11 = cfma(Bc[o], cconj(cur), l11);
            const double az = ra[o] * z, br = rb[o] * r2;
            double2 nxt = make_double2(az * cur.x - br * prev.x, az * cur.y - br * prev.y);
            prev = cur;
            cur = nxt;
          }
        }
      }
      double4 r = trg[cb.x + i];
      r.x += pot;
      r.y += -1.4142135623730951 * l11.x;
      r.z += 1.4142135623730951 * l11.y;
      r.w += gz;
      trg[cb.x + i] = r;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------- P2P
// pot += q/r, grad += q (x_j - x_i)/r^3 with r = 0 pairs skipped (laplace.h:150-235).
template <int TPL>
__global__ void k_p2p(const int *off, const int *src, long long ncells, const int4 *cell_b, const double4 *xt,
                      const int4 *cell_bj, const double4 *xtj, double4 *trg, double cycle) {
  __shared__ double4 sbuf[kWarpsPerBlock][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (long long c = (long long)blockIdx.x * kWarpsPerBlock + warp; c < ncells; c += (long long)gridDim.x * kWarpsPerBlock) {
    const int b = off[c], e = off[c + 1];
    if (b == e) continue;
    const int4 ci = cell_b[c];
    for (int tb = 0; tb < ci.y; tb += 32 * TPL) {
      double xi[TPL], yi[TPL], zi[TPL], pot[TPL], ax[TPL], ay[TPL], az[TPL];
#pragma unroll
      for (int u = 0; u < TPL; u++) {
        const int i = tb + lane + 32 * u;
        double4 v = make_double4(0, 0, 0, 0);
        if (i < ci.y) v = xt[ci.x + i];
        xi[u] = v.x;
        yi[u] = v.y;
        zi[u] = v.z;
        pot[u] = ax[u] = ay[u] = az[u] = 0.0;
      }
      for (int q = b; q < e; q++) {
        const int packed = src[q];
        const int cj = packed & 0x3ffffff, img = packed >> 26;
        double sx, sy, sz;
        image_shift(img, cycle, sx, sy, sz);
        const int4 cjb = cell_bj[cj];
        for (int sb = 0; sb < cjb.y; sb += 32) {
          const int ns = min(32, cjb.y - sb);
          if (lane < ns) {
            double4 s = xtj[cjb.x + sb + lane];
            s.x += sx;
            s.y += sy;
            s.z += sz;
            sbuf[warp][lane] = s;
          }
          __syncwarp();
          for (int s = 0; s < ns; s++) {
            const double4 sj = sbuf[warp][s];
#pragma unroll
            for (int u = 0; u < TPL; u++) {
              const double dx = xi[u] - sj.x, dy = yi[u] - sj.y, dz = zi[u] - sj.z;
              const double r2 = dx * dx + dy * dy + dz * dz;
              if (r2 != 0.0) {
                const double inv = rsqrt(r2);
                const double qr = sj.w * inv;
                const double qr3 = qr * inv * inv;
                pot[u] += qr;
                ax[u] = fma(dx, qr3, ax[u]);
                ay[u] = fma(dy, qr3, ay[u]);
                az[u] = fma(dz, qr3, az[u]);
              }
            }
          }
          __syncwarp();
        }
      }
#pragma unroll
      for (int u = 0; u < TPL; u++) {
        const int i = tb + lane + 32 * u;
        if (i < ci.y) {
          double4 r = trg[ci.x + i];
          r.x += pot[u];
          r.y -= ax[u];
          r.z -= ay[u];
          r.w -= az[u];
          trg[ci.x + i] = r;
        }
      }
    }
  }
}

// ---------------------------------------------------------------- periodic lattice
// Traversal::traversePeriodic (traversal.h:233-287).  The root multipole is
// replicated over a supercell of nb^3 copies (nb = 2 prange + 1).  Each lattice
// level adds, into the root's local expansion, the M2L from every copy in the
// nb^3 - 1 neighboring supercells; then the supercell's multipole is formed by
// M2M of its nb^3 - 1 shifted copies onto the center, and the lattice spacing
// grows by nb.  Root-level work: FP64 in every precision mode.  The warps write
// partial sums that k_part_sum adds in a fixed order.

__device__ __forceinline__ void lattice_index(int idx, int nb, int prange, int &x, int &y, int &z) {
  x = idx / (nb * nb) - prange;
  y = (idx / nb) % nb - prange;
  z = idx % nb - prange;
}

template <int MAXO>
__global__ void k_lattice_m2l(DevTables t, const double2 *Msup, double cycle, int prange, double2 *part) {
  extern __shared__ double2 sh[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int P = t.P, NT = t.nterm, NS = tri(2 * P - 1);
  double2 *Mp = sh + warp * (NT + NS);
  double2 *S = Mp + NT;
  const int nb = 2 * prange + 1, n3 = nb * nb * nb;
  const long long nshift = (long long)(n3 - 1) * n3;
  const long long gw = (long long)blockIdx.x * kWarpsPerBlock + warp, nw = (long long)gridDim.x * kWarpsPerBlock;
  int oj[MAXO], ok[MAXO];
  double2 acc[MAXO];
#pragma unroll
  for (int u = 0; u < MAXO; u++) {
    const int o = lane + 32 * u;
    if (o < NT) tri_decode(o, oj[u], ok[u]);
    else oj[u] = ok[u] = -1;
    acc[u] = make_double2(0.0, 0.0);
  }
  for (int o = lane; o < NT; o += 32) Mp[o] = cscale(Msup[o], t.anm[o]);
  __syncwarp();
  for (long long s = gw; s < nshift; s += nw) {
    int im = (int)(s / n3);
    const int cl = (int)(s - (long long)im * n3);
    if (im >= (n3 - 1) / 2) im++;  // the central supercell is not an image
    int ix, iy, iz, cx, cy, cz;
    lattice_index(im, nb, prange, ix, iy, iz);
    lattice_index(cl, nb, prange, cx, cy, cz);
    // d = X_root - X_root - Xperiodic
    const double dx = -(double)(ix * nb + cx) * cycle, dy = -(double)(iy * nb + cy) * cycle,
                 dz = -(double)(iz * nb + cz) * cycle;
    for (int m = lane; m < 2 * P - 1; m += 32) singular_column(t, m, 2 * P - 1, dx, dy, dz, t.ainv, S);
    __syncwarp();
    m2l_accumulate<MAXO>(t, oj, ok, Mp, S, acc);
    __syncwarp();
  }
#pragma unroll
  for (int u = 0; u < MAXO; u++) {
    const int j = oj[u], k = ok[u];
    if (j < 0) continue;
    const int o = tri(j) + k;
    part[gw * NT + o] = cscale(acc[u], sgn_pow(j) * t.anm[o]);
  }
}

template <int MAXO>
__global__ void k_lattice_m2m(DevTables t, const double2 *Msup, double cycle, int prange, double2 *part) {
  extern __shared__ double2 sh[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int P = t.P, NT = t.nterm;
  double2 *Y = sh + warp * 2 * NT;
  double2 *Mc = Y + NT;
  const int nb = 2 * prange + 1, n3 = nb * nb * nb;
  const long long gw = (long long)blockIdx.x * kWarpsPerBlock + warp, nw = (long long)gridDim.x * kWarpsPerBlock;
  int oj[MAXO], ok[MAXO];
  double2 acc[MAXO];
#pragma unroll
  for (int u = 0; u < MAXO; u++) {
    const int o = lane + 32 * u;
    if (o < NT) tri_decode(o, oj[u], ok[u]);
    else oj[u] = ok[u] = -1;
    acc[u] = make_double2(0.0, 0.0);
  }
  for (int o = lane; o < NT; o += 32) Mc[o] = Msup[o];
  __syncwarp();
  for (long long s = gw; s < n3 - 1; s += nw) {
    int im = (int)s;
    if (im >= (n3 - 1) / 2) im++;
    int ix, iy, iz;
    lattice_index(im, nb, prange, ix, iy, iz);
    // d = X_parent - X_child = -(i * cycle)
    if (lane < P)
      regular_column(t, lane, P, -(double)ix * cycle, -(double)iy * cycle, -(double)iz * cycle, true, Y);
    __syncwarp();
    m2m_accumulate<MAXO>(t, oj, ok, Y, Mc, acc);
    __syncwarp();
  }
#pragma unroll
  for (int u = 0; u < MAXO; u++) {
    const int o = lane + 32 * u;
    if (o < NT) part[gw * NT + o] = acc[u];
  }
}

// out[o] = (base ? base[o] : out[o]) + sum_w part[w][o]: one block per
// coefficient o; thread i sums the parts w = i (mod kPartThreads) in order,
// then a shared-memory tree adds the threads' sums in a fixed order, so the
// result does not depend on timing.
constexpr int kPartThreads = 256;
__global__ void __launch_bounds__(kPartThreads)
k_part_sum(const double2 *part, int nparts, int NT, const double2 *base, double2 *out) {
  __shared__ double2 sh[kPartThreads];
  const int o = blockIdx.x;
  double2 v = make_double2(0.0, 0.0);
  for (int w = threadIdx.x; w < nparts; w += kPartThreads) v = cadd(v, part[(long long)w * NT + o]);
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int h = kPartThreads / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) sh[threadIdx.x] = cadd(sh[threadIdx.x], sh[threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[o] = cadd(base ? base[o] : out[o], sh[0]);
}

// ---------------------------------------------------------------- dipole
// UpDownPass::getDipole (up_down_pass.h:78-86): sum_i (x_i - X0) q_i in FP64.
constexpr int kDipoleBlocks = 256;

__global__ void k_dipole_part(const double4 *x, long long n, double X0x, double X0y, double X0z, double *part) {
  __shared__ double sh[3][256 / 32];
  double a[3] = {0.0, 0.0, 0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double4 b = x[i];
    a[0] += (b.x - X0x) * b.w;
    a[1] += (b.y - X0y) * b.w;
    a[2] += (b.z - X0z) * b.w;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = 0; d < 3; d++) {
    const double v = warp_sum(a[d]);
    if (lane == 0) sh[d][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); w++) v += sh[threadIdx.x][w];
    part[blockIdx.x * 3 + threadIdx.x] = v;
  }
}

__global__ void k_dipole_final(const double *part, int nparts, double *out) {
  if (threadIdx.x < 3) {
    double v = 0.0;
    for (int b = 0; b < nparts; b++) v += part[b * 3 + threadIdx.x];
    out[threadIdx.x] = v;
  }
}

// UpDownPass::dipoleCorrection (up_down_pass.h:89-99), on results in tree order.
__global__ void k_dipole_apply(const double4 *xt, double4 *trg, long long n, double coef, double dx, double dy,
                               double dz, double nbodies) {
  const double nd = dx * dx + dy * dy + dz * dz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double4 r = trg[i];
    r.x -= coef * nd / nbodies / xt[i].w;
    r.y -= coef * dx;
    r.z -= coef * dy;
    r.w -= coef * dz;
    trg[i] = r;
  }
}

int maxo_for(int P) { return (tri(P) + 31) / 32; }

template <template <int> class K>
struct Dispatch;

int blocks_for(long long items) {
  long long g = (items + kWarpsPerBlock - 1) / kWarpsPerBlock;
  if (g > kNumSMs * 32) g = kNumSMs * 32;
  return g < 1 ? 1 : (int)g;
}

template <typename F>
void set_smem(F f, size_t bytes) {
  if (bytes > 48 * 1024) EXA_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

}  // namespace

#define EXA_MAXO_SWITCH(MAXO, ...)                    \
  switch (MAXO) {                                      \
    case 1: { constexpr int MO = 1; __VA_ARGS__; } break;     \
    case 2: { constexpr int MO = 2; __VA_ARGS__; } break;     \
    case 3: { constexpr int MO = 3; __VA_ARGS__; } break;     \
    case 4: { constexpr int MO = 4; __VA_ARGS__; } break;     \
    case 5: { constexpr int MO = 5; __VA_ARGS__; } break;     \
    case 6: { constexpr int MO = 6; __VA_ARGS__; } break;     \
    case 7: { constexpr int MO = 7; __VA_ARGS__; } break;     \
    default: throw_msg("expansion order out of range"); \
  }

void p2m_fp64(const FmmArgs &a) {
  const DevTables &t = device_tables(a.P);
  size_t smem = (t.nterm + (a.P + 1) / 2 + kWarpsPerBlock * (t.nterm + 32 * kP2mRow)) * sizeof(double2);
  set_smem(k_p2m, smem);
  k_p2m<<<blocks_for(a.ncells), 32 * kWarpsPerBlock, smem, a.stream>>>(t, a.cell_b, a.cell_x, a.xt, a.M64, a.ncells);
  EXA_CHECK_LAUNCH();
}

void m2m_fp64(const FmmArgs &a, int level, long long nodes_at_level) {
  const DevTables &t = device_tables(a.P);
  size_t smem = kWarpsPerBlock * 2 * t.nterm * sizeof(double2);
  EXA_MAXO_SWITCH(maxo_for(a.P), {
    set_smem(k_m2m<MO>, smem);
    k_m2m<MO><<<blocks_for(nodes_at_level), 32 * kWarpsPerBlock, smem, a.stream>>>(t, a.lvl, level, a.nd_cell,
                                                                                   a.cell_b, a.cell_x, a.M64);
  });
  EXA_CHECK_LAUNCH();
}

void m2l_fp64(const FmmArgs &a, int skip_min_level, int skip_max_dl) {
  const DevTables &t = device_tables(a.P);
  size_t smem = kWarpsPerBlock * (t.nterm + tri(2 * a.P - 1)) * sizeof(double2);
  const int2 *pl = skip_min_level >= 0 ? a.cell_pl : nullptr;
  const int2 *plj = skip_min_level >= 0 ? (a.src_cell_pl ? a.src_cell_pl : a.cell_pl) : nullptr;
  EXA_MAXO_SWITCH(maxo_for(a.P), {
    set_smem(k_m2l<MO>, smem);
    k_m2l<MO><<<blocks_for(a.ncells), 32 * kWarpsPerBlock, smem, a.stream>>>(
        t, a.m2l_off, a.m2l_src, a.ncells, a.cell_x, a.src_cell_x ? a.src_cell_x : a.cell_x,
        a.src_M64 ? a.src_M64 : a.M64, a.L64, a.cycle, pl, plj, skip_min_level, skip_max_dl);
  });
  EXA_CHECK_LAUNCH();
}

void l2l_fp64(const FmmArgs &a, int level, long long nodes_at_level) {
  const DevTables &t = device_tables(a.P);
  size_t smem = kWarpsPerBlock * (2 * t.nterm + 32 * t.l2l_slots) * sizeof(double2);
  EXA_MAXO_SWITCH(t.l2l_slots, {
    set_smem(k_l2l<MO>, smem);
    k_l2l<MO><<<blocks_for(nodes_at_level), 32 * kWarpsPerBlock, smem, a.stream>>>(t, a.lvl, level, a.nd_cell,
                                                                                   a.cell_pl, a.cell_x, a.L64);
  });
  EXA_CHECK_LAUNCH();
}

void l2p_fp64(const FmmArgs &a) {
  const DevTables &t = device_tables(a.P);
  // recurrence tables (2 NT + P doubles), then W, G, A, B per warp
  size_t smem = (t.nterm + (a.P + 1) / 2 + kWarpsPerBlock * 4 * t.nterm) * sizeof(double2);
  set_smem(k_l2p, smem);
  k_l2p<<<blocks_for(a.ncells), 32 * kWarpsPerBlock, smem, a.stream>>>(t, a.cell_b, a.cell_x, a.xt, a.L64,
                                                                       a.trg64, a.ncells);
  EXA_CHECK_LAUNCH();
}

void p2p_fp64(const FmmArgs &a) {
  const int tpl = (a.ncrit + 31) / 32;
  const int4 *bj = a.src_cell_b ? a.src_cell_b : a.cell_b;
  const double4 *xj = a.src_xt ? a.src_xt : a.xt;
  if (tpl <= 1)
    k_p2p<1><<<blocks_for(a.ncells), 32 * kWarpsPerBlock, 0, a.stream>>>(a.p2p_off, a.p2p_src, a.ncells, a.cell_b,
                                                                          a.xt, bj, xj, a.trg64, a.cycle);
  else if (tpl <= 2)
    k_p2p<2><<<blocks_for(a.ncells), 32 * kWarpsPerBlock, 0, a.stream>>>(a.p2p_off, a.p2p_src, a.ncells, a.cell_b,
                                                                          a.xt, bj, xj, a.trg64, a.cycle);
  else
    k_p2p<4><<<blocks_for(a.ncells), 32 * kWarpsPerBlock, 0, a.stream>>>(a.p2p_off, a.p2p_src, a.ncells, a.cell_b,
                                                                          a.xt, bj, xj, a.trg64, a.cycle);
  EXA_CHECK_LAUNCH();
}

long long lattice_scratch_terms(int P) {
  return (long long)kNumSMs * 4 * kWarpsPerBlock * tri(P) + 2LL * tri(P);
}

void lattice_fp64(const FmmArgs &a, int images, double theta, double2 *scratch) {
  if (images <= 1 || a.ncells <= 0) return;
  const DevTables &t = device_tables(a.P);
  const int NT = t.nterm;
  const int prange = (int)(0.5 / theta + 1);
  const int nb = 2 * prange + 1;
  double2 *msup[2] = {scratch, scratch + NT};
  double2 *part = scratch + 2 * NT;
  EXA_CUDA(cudaMemcpyAsync(msup[0], a.M64, NT * sizeof(double2), cudaMemcpyDeviceToDevice, a.stream));
  const int grid_l = kNumSMs * 4;
  const int grid_m = std::min((nb * nb * nb - 1 + kWarpsPerBlock - 1) / kWarpsPerBlock, grid_l);
  double cycle = a.cycle;
  for (int level = 0; level < images - 1; level++) {
    double2 *cur = msup[level & 1], *nxt = msup[(level + 1) & 1];
    EXA_MAXO_SWITCH(maxo_for(a.P), {
      const size_t smem = kWarpsPerBlock * (NT + tri(2 * a.P - 1)) * sizeof(double2);
      set_smem(k_lattice_m2l<MO>, smem);
      k_lattice_m2l<MO><<<grid_l, 32 * kWarpsPerBlock, smem, a.stream>>>(t, cur, cycle, prange, part);
    });
    EXA_CHECK_LAUNCH();
    k_part_sum<<<NT, kPartThreads, 0, a.stream>>>(part, grid_l * kWarpsPerBlock, NT, nullptr, a.L64);
    EXA_CHECK_LAUNCH();
    EXA_MAXO_SWITCH(maxo_for(a.P), {
      const size_t smem = kWarpsPerBlock * 2 * NT * sizeof(double2);
      set_smem(k_lattice_m2m<MO>, smem);
      k_lattice_m2m<MO><<<grid_m, 32 * kWarpsPerBlock, smem, a.stream>>>(t, cur, cycle, prange, part);
    });
    EXA_CHECK_LAUNCH();
    k_part_sum<<<NT, kPartThreads, 0, a.stream>>>(part, grid_m * kWarpsPerBlock, NT, cur, nxt);
    EXA_CHECK_LAUNCH();
    cycle *= nb;
  }
}

void dipole_fp64(const double4 *x, long long n, const double X0[3], double *scratch, double *out3, cudaStream_t st) {
  k_dipole_part<<<kDipoleBlocks, 256, 0, st>>>(x, n, X0[0], X0[1], X0[2], scratch);
  EXA_CHECK_LAUNCH();
  k_dipole_final<<<1, 32, 0, st>>>(scratch, kDipoleBlocks, out3);
  EXA_CHECK_LAUNCH();
}

void dipole_correction_fp64(const double4 *xt, double4 *trg, long long n, double cycle, const double dip[3],
                            double nbodies, cudaStream_t st) {
  if (n <= 0) return;
  const double coef = 4 * M_PI / (3 * cycle * cycle * cycle);
  long long g = (n + 255) / 256;
  if (g > kNumSMs * 16) g = kNumSMs * 16;
  k_dipole_apply<<<(int)g, 256, 0, st>>>(xt, trg, n, coef, dip[0], dip[1], dip[2], nbodies);
  EXA_CHECK_LAUNCH();
}

}  // namespace exafmm_b200
