// M2L launchers: the register-resident unrolled kernel (m2l_fast.cuh) for the
// orders it is instantiated for, in FP64 (plain method) and FP32 (mixed form).
//
// Mixed form: pairs whose target sits at level >= kMixedMinLevel and whose
// level difference is at most kMixedMaxDl run in FP32 with FP64 accumulation
// of the per-lane partial expansions; the root levels and the rare pairs of
// very different sizes stay in FP64 (generic kernel in fmm64.cu).
#include <mutex>
#include <type_traits>

#include "fmm.h"
#include "harmonics.cuh"
#include "m2l_fast.cuh"

namespace exafmm_b200 {

__constant__ RecTab<float> c_tab32;
__constant__ RecTab<double> c_tab64;

namespace {

std::mutex g_tab_mutex;
bool g_tab_ready[64] = {};

void init_tables() {
  int dev = 0;
  EXA_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_tab_mutex);
  if (dev < 64 && g_tab_ready[dev]) return;
  RecTab<double> t64;
  RecTab<float> t32;
  const int Q = 2 * kMaxP;
  auto fact = [](int k) {
    double f = 1;
    for (int i = 2; i <= k; i++) f *= i;
    return f;
  };
  for (int n = 0; n < Q; n++)
    for (int m = 0; m <= n; m++) {
      const int o = n * (n + 1) / 2 + m;
      const double den = double(n + 1) * (n + 1) - double(m) * m;
      t64.ra[o] = (2.0 * n + 1.0) / sqrt(den);
      t64.rb[o] = sqrt((double(n) * n - double(m) * m) / den);
      const double a = ((n & 1) ? -1.0 : 1.0) / sqrt(fact(n - m) * fact(n + m));
      t64.ainv[o] = 1.0 / a;
      t32.ra[o] = (float)t64.ra[o];
      t32.rb[o] = (float)t64.rb[o];
      t32.ainv[o] = (float)t64.ainv[o];
    }
  t64.rd[0] = 1.0;
  t32.rd[0] = 1.0f;
  for (int m = 1; m <= Q; m++) {
    t64.rd[m] = sqrt((2.0 * m - 1.0) / (2.0 * m));
    t32.rd[m] = (float)t64.rd[m];
  }
  EXA_CUDA(cudaMemcpyToSymbol(c_tab64, &t64, sizeof(t64)));
  EXA_CUDA(cudaMemcpyToSymbol(c_tab32, &t32, sizeof(t32)));
  if (dev < 64) g_tab_ready[dev] = true;
}

template <typename T> __device__ __forceinline__ const RecTab<T> &tab();
template <> __device__ __forceinline__ const RecTab<float> &tab<float>() { return c_tab32; }
template <> __device__ __forceinline__ const RecTab<double> &tab<double>() { return c_tab64; }

// Ms[c][n(n+1)/2+m] = A_n^m M_n^m / R_c^n, in the working precision.
template <typename T>
__global__ void k_scale_M(DevTables t, const double2 *M, const double4 *cell_x, long long ncells, Cx<T> *Ms) {
  const int NT = t.nterm;
  const long long total = ncells * NT;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long c = i / NT;
    const int o = (int)(i - c * NT);
    int n, m;
    tri_decode(o, n, m);
    const double R = cell_x[c].w;
    const double s = t.anm[o] * pow(R, -(double)n);
    const double2 v = M[i];
    Ms[i] = Cx<T>{(T)(v.x * s), (T)(v.y * s)};
  }
}

template <int J0_, int J1_, int N0_, int N1_>
struct Part {
  static constexpr int J0 = J0_, J1 = J1_, N0 = N0_, N1 = N1_;
};
template <typename... Ps>
struct Parts {
  static constexpr int size = sizeof...(Ps);
};

struct M2LCtx {
  const int *off, *src;
  long long ncells;
  const double4 *cell_x;
  const int2 *cell_pl;
  const double4 *cell_xj;  // source cells: the same table, or a separate source tree's
  const int2 *cell_plj;
  const void *Ms;
  double cycle;
  int mode;  // 0: every pair; 1: mixed-regular pairs only
  int min_level, max_dl;
  const unsigned char *taken;  // pairs the tile kernel (m2l_gemm.cu) evaluates, or null
};

__device__ __forceinline__ bool mixed_regular(const M2LCtx &g, int lt, int ls) {
  const int dl = lt - ls;
  return lt >= g.min_level && dl <= g.max_dl && dl >= -g.max_dl;
}

// One (J, N) part of the contraction for every target: warp per target cell,
// lanes over its sources, per-lane partial expansions summed in FP64 and added
// to L with the output scaling (-1)^j A_j^k R_t^{-(j+1)}.  The parts of one
// order run as consecutive launches on one stream, so L is updated in a fixed
// order.
constexpr int kM2LWarps = 4;

template <typename T, int P, int J0, int J1, int N0, int N1>
__global__ void __launch_bounds__(32 * kM2LWarps)
k_m2l_part(M2LCtx g, DevTables t, double2 *L) {
  constexpr int NM = ctri(N1) - ctri(N0);
  constexpr int NA = ctri(J1) - ctri(J0);
  constexpr int NT = ctri(P);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const Cx<T> *Ms = (const Cx<T> *)g.Ms;
  for (long long c = (long long)blockIdx.x * kM2LWarps + warp; c < g.ncells; c += (long long)gridDim.x * kM2LWarps) {
    const int b = g.off[c], e = g.off[c + 1];
    if (b == e) continue;
    constexpr bool kPacked = std::is_same<T, float>::value;  // FP32 runs on packed f32x2 pairs
    using Acc = typename std::conditional<kPacked, f2p, Cx<T>>::type;
    Acc acc[NA];
#pragma unroll
    for (int i = 0; i < NA; i++) acc[i] = Acc{};
    const double4 Xt = g.cell_x[c];
    const int lt = g.cell_pl[c].y;
    const double inv_rt = 1.0 / Xt.w;
    // Warp-uniform trip count: the pair code holds warp barriers, so every lane
    // runs every iteration; a lane without a (kept) pair runs a dummy one with
    // zero multipoles at a unit offset, which adds nothing.
    for (int base = b; base < e; base += 32) {
      const int q = base + lane;
      bool live = q < e;
      int cj = 0, img = 13, ls = lt;
      if (live) {
        const int packed = g.src[q];
        cj = packed & 0x3ffffff;
        img = packed >> 26;
        ls = g.cell_plj[cj].y;
        if (g.mode == 1 && !mixed_regular(g, lt, ls)) live = false;
        if (g.taken && g.taken[q]) live = false;
      }
      if (!__any_sync(0xffffffffu, live)) continue;  // warp-uniform: a batch with nothing to add
      T x = T(1), y = T(0), z = T(0);
      if (live) {
        const double4 Xs = g.cell_xj[cj];
        const double sx = (double)(img / 9 - 1) * g.cycle, sy = (double)((img / 3) % 3 - 1) * g.cycle,
                     sz = (double)(img % 3 - 1) * g.cycle;
        x = (T)((Xt.x - Xs.x - sx) * inv_rt);
        y = (T)((Xt.y - Xs.y - sy) * inv_rt);
        z = (T)((Xt.z - Xs.z - sz) * inv_rt);
      }
      // M'' = Ms * (R_s / R_t)^n, an exact power of two: R_s / R_t = 2^(lt - ls).
      const T f1 = (T)ldexp(1.0, lt - ls);
      Cx<T> Mv[NM];
      T fn = live ? T(1) : T(0);
#pragma unroll
      for (int n = 0; n < N1; n++) {
        if (n >= N0) {
#pragma unroll
          for (int m = 0; m <= n; m++) {
            const Cx<T> v = Ms[(long long)cj * NT + ctri(n) + m];
            Mv[ctri(n) - ctri(N0) + m] = Cx<T>{v.x * fn, v.y * fn};
          }
        }
        fn *= f1;
      }
      if constexpr (kPacked) {
        f2p Mxx[NM], Myy[NM];
#pragma unroll
        for (int i = 0; i < NM; i++) {
          Mxx[i] = pk2(Mv[i].x, Mv[i].x);
          Myy[i] = pk2(Mv[i].y, Mv[i].y);
        }
        m2l_pair_f32x2<P, J0, J1, N0, N1>(tab<float>(), Mxx, Myy, acc, x, y, z);
      } else {
        m2l_pair_unrolled<T, P, J0, J1, N0, N1>(tab<T>(), Mv, acc, x, y, z);
      }
    }
    const double rt = Xt.w;
#pragma unroll
    for (int i = 0; i < NA; i++) {
      double re, im;
      if constexpr (kPacked) {
        const float2 v = unpk2(acc[i]);
        re = v.x;
        im = v.y;
      } else {
        re = (double)acc[i].x;
        im = (double)acc[i].y;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
      }
      if (lane == (i & 31)) {
        const int o = ctri(J0) + i;
        int j, k;
        tri_decode(o, j, k);
        const double w = ((j & 1) ? -1.0 : 1.0) * t.anm[o] * pow(rt, -(double)(j + 1));
        double2 v = L[c * NT + o];
        v.x += w * re;
        v.y += w * im;
        L[c * NT + o] = v;
      }
    }
  }
}

template <typename T, int P, typename Pt>
void launch_part(const M2LCtx &g, const DevTables &t, double2 *L, cudaStream_t st) {
  long long grid = (g.ncells + kM2LWarps - 1) / kM2LWarps;
  if (grid > kNumSMs * 16) grid = kNumSMs * 16;
  if (grid < 1) grid = 1;
  k_m2l_part<T, P, Pt::J0, Pt::J1, Pt::N0, Pt::N1><<<(int)grid, 32 * kM2LWarps, 0, st>>>(g, t, L);
  EXA_CHECK_LAUNCH();
}

template <typename T, int P, typename... Ps>
void launch_fast(const M2LCtx &g, const DevTables &t, double2 *L, cudaStream_t st) {
  (launch_part<T, P, Ps>(g, t, L, st), ...);
}

// Work splits keep each part's registers (its M'' slice plus its outputs) in budget.
template <typename T>
bool launch_for_P(int P, const M2LCtx &g, const DevTables &t, double2 *L, cudaStream_t st);

template <>
bool launch_for_P<float>(int P, const M2LCtx &g, const DevTables &t, double2 *L, cudaStream_t st) {
  switch (P) {
    case 4: launch_fast<float, 4, Part<0, 4, 0, 4>>(g, t, L, st); return true;
    case 6: launch_fast<float, 6, Part<0, 6, 0, 6>>(g, t, L, st); return true;
    case 8:
      launch_fast<float, 8, Part<0, 6, 0, 6>, Part<0, 6, 6, 8>, Part<6, 8, 0, 6>, Part<6, 8, 6, 8>>(g, t, L, st);
      return true;
    case 10:
      launch_fast<float, 10, Part<0, 6, 0, 5>, Part<0, 6, 5, 8>, Part<0, 6, 8, 10>, Part<6, 8, 0, 5>,
                  Part<6, 8, 5, 8>, Part<6, 8, 8, 10>, Part<8, 10, 0, 5>, Part<8, 10, 5, 8>, Part<8, 10, 8, 10>>(
          g, t, L, st);
      return true;
    default: return false;
  }
}

template <>
bool launch_for_P<double>(int P, const M2LCtx &g, const DevTables &t, double2 *L, cudaStream_t st) {
  switch (P) {
    case 4: launch_fast<double, 4, Part<0, 4, 0, 4>>(g, t, L, st); return true;
    case 6: launch_fast<double, 6, Part<0, 6, 0, 4>, Part<0, 6, 4, 6>>(g, t, L, st); return true;
    case 8:
      launch_fast<double, 8, Part<0, 6, 0, 6>, Part<0, 6, 6, 8>, Part<6, 8, 0, 6>, Part<6, 8, 6, 8>>(g, t, L, st);
      return true;
    case 10:
      launch_fast<double, 10, Part<0, 6, 0, 5>, Part<0, 6, 5, 8>, Part<0, 6, 8, 10>, Part<6, 8, 0, 5>,
                  Part<6, 8, 5, 8>, Part<6, 8, 8, 10>, Part<8, 10, 0, 5>, Part<8, 10, 5, 8>, Part<8, 10, 8, 10>>(
          g, t, L, st);
      return true;
    default: return false;
  }
}

}  // namespace

bool m2l_fast_supported(int P, bool mixed) {
  return mixed ? (P == 4 || P == 6 || P == 8 || P == 10) : (P == 4 || P == 6 || P == 8 || P == 10);
}

void scale_multipoles(const FmmArgs &a, bool mixed, void *Ms) {
  scale_multipoles(a.P, a.M64, a.cell_x, a.ncells, mixed, Ms, a.stream);
}

void scale_multipoles(int P, const double2 *M, const double4 *cell_x, long long ncells, bool mixed, void *Ms,
                      cudaStream_t st) {
  const DevTables &t = device_tables(P);
  const long long total = ncells * t.nterm;
  int grid = (int)((total + 255) / 256);
  if (grid > kNumSMs * 16) grid = kNumSMs * 16;
  if (grid < 1) grid = 1;
  if (mixed) k_scale_M<float><<<grid, 256, 0, st>>>(t, M, cell_x, ncells, (Cx<float> *)Ms);
  else k_scale_M<double><<<grid, 256, 0, st>>>(t, M, cell_x, ncells, (Cx<double> *)Ms);
  EXA_CHECK_LAUNCH();
}

bool m2l_fast(const FmmArgs &a, bool mixed, const void *Ms, int min_level, int max_dl, const unsigned char *taken) {
  if (!m2l_fast_supported(a.P, mixed)) return false;
  init_tables();
  const DevTables &t = device_tables(a.P);
  M2LCtx g;
  g.off = a.m2l_off;
  g.src = a.m2l_src;
  g.ncells = a.ncells;
  g.cell_x = a.cell_x;
  g.cell_pl = a.cell_pl;
  g.cell_xj = a.src_cell_x ? a.src_cell_x : a.cell_x;
  g.cell_plj = a.src_cell_pl ? a.src_cell_pl : a.cell_pl;
  g.Ms = Ms;
  g.cycle = a.cycle;
  g.mode = mixed ? 1 : 0;
  g.min_level = min_level;
  g.max_dl = max_dl;
  g.taken = taken;
  return mixed ? launch_for_P<float>(a.P, g, t, a.L64, a.stream) : launch_for_P<double>(a.P, g, t, a.L64, a.stream);
}

}  // namespace exafmm_b200
