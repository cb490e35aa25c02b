// M2L as dense tiles: pairs grouped by offset class, each class one real
// operator matrix (the mixed form's FP32 M2L for regular pairs).
//
// Between scaled expansions the M2L (kernels/laplace.h:292-322; the scaled form
// of m2l_fast.cuh) is a linear map that depends only on the offset of the two
// cell centers in units of the target radius and on the level difference:
//   acc_j^k = sum_{n,m} s(k,m) (R_s/R_t)^n Ms_n^m S'_{j+n}^{m-k}(d / R_t),
//   L_j^k  += (-1)^j A_j^k R_t^{-(j+1)} acc_j^k,        Ms = A_n^m M_n^m / R_s^n.
// Every center is the root center plus dyadic multiples of the radii, so
// d / min(R_s, R_t) is an integer vector: (level difference, that vector) is a
// class key.  Written over real degrees of freedom (Re of every coefficient,
// Im of those with m > 0: 2 NTERM - P of them, 64 at P = 8), a class's map is
// one ND x ND real matrix K.
//
// Targets are grouped by (level, octant within the parent) -- cells in the
// same position relative to their parents have alike interaction lists -- and
// cut into tiles of 32 in cell order.  The pairs are sorted by (tile, class):
// a run of equal keys pairs at most one source with each target of the tile,
// so a tile's local expansions accumulate, column per target, as
//   D[:, targets] += K_class x B,   B[:, t] = Ms of t's source of that class (or 0),
// over the tile's runs, with no scatter and in a fixed order.  FP32 products,
// FP32 sums over at most eight runs, flushed into FP64 accumulators.
//
// Classes used by fewer than kMinClassPairs pairs and pairs through periodic
// images stay with the pair-by-pair FP32 kernel, which then runs on a compacted
// list of just those pairs (left_off / left_src); pairs outside the mixed
// policy stay with the FP64 kernel as before.
#include <algorithm>
#include <stdexcept>

#include "fmm.h"
#include "harmonics.cuh"
#include "scan.cuh"

namespace exafmm_b200 {
namespace {

constexpr unsigned long long kEmpty = ~0ull;
constexpr int kMinClassPairs = 16;
constexpr int kTile = 32;         // targets per tile
constexpr int kClsBits = 20;      // class id field of the pair key
constexpr int kProbe = 64;        // hash probe limit (a pair that finds no slot stays per-pair)

__host__ __device__ inline int nd_of(int P) { return P * (P + 1) - P; }
__host__ __device__ inline int ndp_of(int P) { return (nd_of(P) + 15) / 16 * 16; }

__device__ __forceinline__ unsigned long long mix64(unsigned long long k) {
  // MurmurHash3's 64-bit finalizer
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}

// Real degree of freedom d -> (n, m, part): d < NT is Re of coefficient d,
// d >= NT the Im parts of the m > 0 coefficients in (n, m) order.
__device__ __forceinline__ void dof_decode(int d, int NT, int &n, int &m, int &part) {
  if (d < NT) {
    tri_decode(d, n, m);
    part = 0;
  } else {
    int e = d - NT;
    n = 1;
    while (e >= n) {
      e -= n;
      n++;
    }
    m = e + 1;
    part = 1;
  }
}

__device__ __forceinline__ unsigned long long class_key(int dl, long long dx, long long dy, long long dz) {
  return ((unsigned long long)(dl + 16) << 48) | ((unsigned long long)(dx + 32768) << 32) |
         ((unsigned long long)(dy + 32768) << 16) | (unsigned long long)(dz + 32768);
}

// 1. Per pair of the target-grouped list: its class's hash slot, or -1.
__global__ void k_pair_class(const int *off, const int *src, long long ncells, const double4 *cell_x,
                             const int2 *cell_pl, int min_level, int max_dl, unsigned long long *hk, unsigned *hc,
                             long long hmask, int *pair_slot) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long c = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < ncells; c += warps) {
    const int b = off[c], e = off[c + 1];
    if (b == e) continue;
    const double4 Xt = cell_x[c];
    const int lt = cell_pl[c].y;
    for (int q = b + lane; q < e; q += 32) {
      const int packed = src[q];
      const int cj = packed & 0x3ffffff, img = packed >> 26;
      const int ls = cell_pl[cj].y;
      const int dl = ls - lt;
      int slot = -1;
      if (img == 13 && lt >= min_level && dl <= max_dl && dl >= -max_dl) {
        const double4 Xs = cell_x[cj];
        const double rmin = fmin(Xt.w, Xs.w);
        const double fx = rint((Xt.x - Xs.x) / rmin), fy = rint((Xt.y - Xs.y) / rmin), fz = rint((Xt.z - Xs.z) / rmin);
        if (fabs(fx) < 32767 && fabs(fy) < 32767 && fabs(fz) < 32767) {
          const unsigned long long key = class_key(dl, (long long)fx, (long long)fy, (long long)fz);
          long long h = (long long)(mix64(key) & (unsigned long long)hmask);
          for (int p = 0; p < kProbe; p++) {
            const unsigned long long old = atomicCAS(&hk[h], kEmpty, key);
            if (old == kEmpty || old == key) {
              atomicAdd(&hc[h], 1u);
              slot = (int)h;
              break;
            }
            h = (h + 1) & hmask;
          }
        }
      }
      pair_slot[q] = slot;
    }
  }
}

// 2. Classes used often enough, in arbitrary order (sorted by key next).
__global__ void k_class_compact(const unsigned long long *hk, const unsigned *hc, long long hcap,
                                unsigned long long *ck, int *cs, int *ncls, int cap) {
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < hcap; h += (long long)gridDim.x * blockDim.x) {
    if (hk[h] != kEmpty && hc[h] >= (unsigned)kMinClassPairs) {
      const int i = atomicAdd(ncls, 1);
      if (i < cap) {
        ck[i] = hk[h];
        cs[i] = (int)h;
      }
    }
  }
}

__global__ void k_class_ids(const int *cs_sorted, int ncls, int *hid) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncls; i += gridDim.x * blockDim.x) hid[cs_sorted[i]] = i;
}

// 3. Operator of each class, k-major: Kt[class][input dof][output dof], FP32.
__global__ void k_build_K(DevTables t, const unsigned long long *ck, int P, float *Kt) {
  extern __shared__ double2 S[];  // S'_p^q, q >= 0, at d / R_t
  const int NT = t.nterm, ND = nd_of(P), NDP = ndp_of(P);
  const unsigned long long key = ck[blockIdx.x];
  const int dl = (int)((key >> 48) & 0xffff) - 16;
  const double ux = (double)(long long)((key >> 32) & 0xffff) - 32768.0;
  const double uy = (double)(long long)((key >> 16) & 0xffff) - 32768.0;
  const double uz = (double)(long long)(key & 0xffff) - 32768.0;
  const double to_rt = dl > 0 ? ldexp(1.0, -dl) : 1.0;  // min(R_s, R_t) / R_t
  if ((int)threadIdx.x < 2 * P - 1)
    singular_column(t, threadIdx.x, 2 * P - 1, ux * to_rt, uy * to_rt, uz * to_rt, t.ainv, S);
  __syncthreads();
  float *K = Kt + (long long)blockIdx.x * NDP * NDP;
  for (int e = threadIdx.x; e < NDP * NDP; e += blockDim.x) {
    const int c = e / NDP, r = e - c * NDP;
    double val = 0.0;
    if (r < ND && c < ND) {
      int j, k, rp, n, mp, cp;
      dof_decode(r, NT, j, k, rp);
      dof_decode(c, NT, n, mp, cp);
      const double fn = ldexp(1.0, -dl * n);  // (R_s / R_t)^n
      double sr = 0.0, si = 0.0;
      for (int side = 0; side < (mp > 0 ? 2 : 1); side++) {
        const int m = side == 0 ? mp : -mp;
        const int q = m - k, p = j + n;
        double2 Sv = q >= 0 ? S[tri(p) + q] : cconj(S[tri(p) - q]);
        const double s = (m < 0) ? 1.0 : (m <= k ? (double)sgn_pow(m) : (double)sgn_pow(k));
        // the input's contribution to M_n^m: Re part -> 1, Im part -> +i (m > 0) or -i (m < 0)
        double tr = s * Sv.x, ti = s * Sv.y;
        if (cp == 1) {
          const double a = tr;
          if (m > 0) {
            tr = -ti;
            ti = a;
          } else {
            tr = ti;
            ti = -a;
          }
        }
        sr += tr;
        si += ti;
      }
      val = fn * (rp == 0 ? sr : si);
    }
    K[e] = (float)val;
  }
}

// Scaled multipoles over real degrees of freedom, FP32, padded to NDP.
__global__ void k_scale_M_real(DevTables t, const double2 *M, const double4 *cell_x, long long ncells, int P,
                               float *Msr) {
  const int NT = t.nterm, ND = nd_of(P), NDP = ndp_of(P);
  const long long total = ncells * NDP;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long c = i / NDP;
    const int d = (int)(i - c * NDP);
    float v = 0.f;
    if (d < ND) {
      int n, m, part;
      dof_decode(d, NT, n, m, part);
      const int o = tri(n) + m;
      const double s = t.anm[o] * pow(cell_x[c].w, -(double)n);
      const double2 mv = M[c * NT + o];
      v = (float)((part == 0 ? mv.x : mv.y) * s);
    }
    Msr[i] = v;
  }
}

// 4. Per target: take its pairs of frequent classes; group key (level, octant) or 255.
__device__ __forceinline__ bool policy_pair(int lt, int ls, int min_level, int max_dl) {
  const int dl = lt - ls;
  return lt >= min_level && dl <= max_dl && dl >= -max_dl;
}

__global__ void k_gemm_flags(const int *off, const int *src, long long ncells, const int *pair_slot, const int *hid,
                             const double4 *cell_x, const int2 *cell_pl, int min_level, int max_dl,
                             unsigned char *taken, unsigned *grp, int *cellidx, int *left_cnt) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long c = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < ncells; c += warps) {
    const int b = off[c], e = off[c + 1];
    const int lt = cell_pl[c].y;
    bool any = false;
    int left = 0;
    for (int q = b + lane; q < e; q += 32) {
      const int s = pair_slot[q];
      const bool tk = s >= 0 && hid[s] >= 0;
      taken[q] = tk ? 1 : 0;
      any |= tk;
      if (!tk && policy_pair(lt, cell_pl[src[q] & 0x3ffffff].y, min_level, max_dl)) left++;
    }
    any = __any_sync(0xffffffffu, any);
    for (int o = 16; o > 0; o >>= 1) left += __shfl_xor_sync(0xffffffffu, left, o);
    if (lane == 0) left_cnt[c] = left;
    if (lane == 0) {
      unsigned g = 255u;
      if (any) {
        const int2 pl = cell_pl[c];
        int oct = 0;
        if (pl.x >= 0 && pl.y > 0) {
          const double4 X = cell_x[c], Xp = cell_x[pl.x];
          oct = (X.x > Xp.x ? 1 : 0) | (X.y > Xp.y ? 2 : 0) | (X.z > Xp.z ? 4 : 0);
        }
        g = (unsigned)(pl.y * 8 + oct);
        if (g > 254u) g = 254u;  // levels beyond 31 (not reachable: depth <= 21)
      }
      grp[c] = g;
      cellidx[c] = (int)c;
    }
  }
}

// 5. Group starts in the cells sorted by group, tiles per group, tile bases.
__global__ void k_tile_bases(const unsigned *gsorted, long long ncells, int *gstart, int *tbase, int *ntiles) {
  const int g = threadIdx.x;  // 256 threads
  long long lo = 0, hi = ncells;
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (gsorted[mid] < (unsigned)g) lo = mid + 1;
    else hi = mid;
  }
  long long lo2 = lo, hi2 = ncells;
  while (lo2 < hi2) {
    const long long mid = (lo2 + hi2) >> 1;
    if (gsorted[mid] <= (unsigned)g) lo2 = mid + 1;
    else hi2 = mid;
  }
  __shared__ int cnt[256];
  gstart[g] = (int)lo;
  cnt[g] = (g == 255) ? 0 : (int)((lo2 - lo + kTile - 1) / kTile);
  __syncthreads();
  if (g == 0) {
    int acc = 0;
    for (int i = 0; i < 256; i++) {
      tbase[i] = acc;
      acc += cnt[i];
    }
    *ntiles = acc;
  }
}

__global__ void k_tile_assign(const unsigned *gsorted, const int *csorted, long long ncells, const int *gstart,
                              const int *tbase, int *tile_of, int *tile_cell) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ncells; i += (long long)gridDim.x * blockDim.x) {
    const unsigned g = gsorted[i];
    const int c = csorted[i];
    if (g == 255u) {
      tile_of[c] = -1;
      continue;
    }
    const int rank = (int)(i - gstart[g]);
    const int tile = tbase[g] + rank / kTile, slot = rank % kTile;
    tile_of[c] = tile * kTile + slot;
    tile_cell[tile * kTile + slot] = c;
  }
}

// 6. Sort keys: (tile, class) for taken pairs, all ones for the rest.
__global__ void k_pair_keys(const int *off, const int *src, long long ncells, const int *pair_slot, const int *hid,
                            const unsigned char *taken, const int *tile_of, unsigned long long *pkey, int *pval) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long c = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < ncells; c += warps) {
    const int b = off[c], e = off[c + 1];
    const int ts = tile_of[c];
    for (int q = b + lane; q < e; q += 32) {
      if (taken[q] && ts >= 0) {
        const int tile = ts / kTile, slot = ts % kTile;
        pkey[q] = ((unsigned long long)tile << kClsBits) | (unsigned long long)hid[pair_slot[q]];
        pval[q] = (slot << 26) | (src[q] & 0x3ffffff);
      } else {
        pkey[q] = kEmpty;
        pval[q] = 0;
      }
    }
  }
}

// Offsets of the leftover pairs per target (exclusive scan of the counts).
struct LeftScan {
  using T = int;
  const int *cnt;
  int *off2;
  long long n;
  __device__ T value(long long i) const { return cnt[i]; }
  __device__ void emit(long long i, const T &, const T &excl) const { off2[i] = excl; }
  __device__ void total(const T &t) const { off2[n] = t; }
};

// The leftover pairs (not taken by the tiles, inside the mixed policy) in list order.
__global__ void k_left_fill(const int *off, const int *src, long long ncells, const unsigned char *taken,
                            const int2 *cell_pl, int min_level, int max_dl, const int *off2, int *src2) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long c = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < ncells; c += warps) {
    const int b = off[c], e = off[c + 1];
    const int lt = cell_pl[c].y;
    int at = off2[c];
    for (int base = b; base < e; base += 32) {
      const int q = base + lane;
      bool keep = false;
      int v = 0;
      if (q < e) {
        v = src[q];
        keep = !taken[q] && policy_pair(lt, cell_pl[v & 0x3ffffff].y, min_level, max_dl);
      }
      const unsigned m = __ballot_sync(0xffffffffu, keep);
      if (keep) src2[at + __popc(m & ((1u << lane) - 1u))] = v;
      at += __popc(m);
    }
  }
}

__device__ __forceinline__ long long lower_bound_u64(const unsigned long long *a, long long n, unsigned long long v) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (a[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// 7. One block per tile: D (NDP x 32, FP32, 4 x 4 per thread) += K x B per run.
template <int NDP>
__global__ void __launch_bounds__(NDP / 4 * (kTile / 4))
k_m2l_gemm(const unsigned long long *pkey, const int *pval, long long npairs, const int *ntiles, const float *Kt,
           const float *Msr, const int *tile_cell, const double4 *cell_x, DevTables t, int P, double2 *L) {
  constexpr int THREADS = NDP / 4 * (kTile / 4);
  extern __shared__ float sm[];
  float *sK = sm;                  // [NDP input][NDP output]
  float *sB = sm + NDP * NDP;      // [NDP input][kTile]
  __shared__ int s_len;
  const int tile = blockIdx.x;
  if (tile >= *ntiles) return;
  const long long lo = lower_bound_u64(pkey, npairs, (unsigned long long)tile << kClsBits);
  const long long hi = lower_bound_u64(pkey, npairs, (unsigned long long)(tile + 1) << kClsBits);
  const int tx = threadIdx.x % (kTile / 4), ty = threadIdx.x / (kTile / 4);
  float acc[4][4];
  double accd[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) {
      acc[a][b] = 0.f;
      accd[a][b] = 0.0;
    }
  int nrun = 0;
  for (long long p = lo; p < hi;) {
    __syncthreads();  // the previous run's products are done with sK and sB
    if (threadIdx.x < 32) {
      const unsigned long long k0 = pkey[p];
      const long long q = p + threadIdx.x;
      const bool same = q < hi && pkey[q] == k0;
      const unsigned m = __ballot_sync(0xffffffffu, same);
      if (threadIdx.x == 0) s_len = (m == 0xffffffffu) ? 32 : __ffs(~m) - 1;
    }
    const int cls = (int)(pkey[p] & ((1ull << kClsBits) - 1));
    const float4 *Kg = (const float4 *)(Kt + (long long)cls * NDP * NDP);
    for (int i = threadIdx.x; i < NDP * NDP / 4; i += THREADS) ((float4 *)sK)[i] = Kg[i];
    for (int i = threadIdx.x; i < NDP * kTile / 4; i += THREADS) ((float4 *)sB)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    const int len = s_len;
    // gather: consecutive threads take different pairs (different columns, no bank conflicts)
    for (int i = threadIdx.x; i < len * (NDP / 4); i += THREADS) {
      const int pr = i % len, q4 = i / len;
      const int v = pval[p + pr];
      const int slot = v >> 26, srcc = v & 0x3ffffff;
      const float4 m = ((const float4 *)(Msr + (long long)srcc * NDP))[q4];
      sB[(4 * q4 + 0) * kTile + slot] = m.x;
      sB[(4 * q4 + 1) * kTile + slot] = m.y;
      sB[(4 * q4 + 2) * kTile + slot] = m.z;
      sB[(4 * q4 + 3) * kTile + slot] = m.w;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < NDP; kk++) {
      const float4 a = ((const float4 *)(sK + kk * NDP))[ty];
      const float4 b = ((const float4 *)(sB + kk * kTile))[tx];
      const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[r][c] = fmaf(av[r], bv[c], acc[r][c]);
    }
    if (++nrun == 8) {
      nrun = 0;
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
          accd[r][c] += (double)acc[r][c];
          acc[r][c] = 0.f;
        }
    }
    p += len;
  }
  const int NT = t.nterm, ND = nd_of(P);
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const int cell = tile_cell[tile * kTile + 4 * tx + c];
    if (cell < 0) continue;
    const double rt = cell_x[cell].w;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int d = 4 * ty + r;
      if (d >= ND) continue;
      int j, k, part;
      dof_decode(d, NT, j, k, part);
      const int o = tri(j) + k;
      const double w = sgn_pow(j) * t.anm[o] * pow(rt, -(double)(j + 1));
      const double v = (accd[r][c] + (double)acc[r][c]) * w;
      double2 *dst = &L[(long long)cell * NT + o];
      if (part == 0) dst->x += v;
      else dst->y += v;
    }
  }
}

int bits_for(long long v) {
  int b = 0;
  while ((1LL << b) <= v) b++;
  return b;
}

template <typename F>
void set_smem(F f, size_t bytes) {
  if (bytes > 48 * 1024) EXA_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

}  // namespace

bool m2l_gemm_supported(int P) { return P == 4 || P == 6 || P == 8 || P == 10; }

bool m2l_gemm(Context &C, const FmmArgs &a, M2LGemmBufs &g, long long n_m2l, int min_level, int max_dl) {
  const int P = a.P;
  if (!m2l_gemm_supported(P) || a.ncells <= 0 || n_m2l <= 0) return false;
  cudaStream_t st = a.stream;
  const DevTables &t = device_tables(P);
  const long long nc = a.ncells;
  const int NDP = ndp_of(P);
  // ---- classes
  long long hcap = 1 << 16;
  while (hcap < 4 * std::min<long long>(n_m2l, 1LL << 22)) hcap <<= 1;
  g.hk.ensure(hcap);
  g.hc.ensure(hcap);
  g.hid.ensure(hcap);
  g.pair_slot.ensure(n_m2l);
  g.cnt.ensure(4);
  EXA_CUDA(cudaMemsetAsync(g.hk.p, 0xff, hcap * sizeof(unsigned long long), st));
  EXA_CUDA(cudaMemsetAsync(g.hc.p, 0, hcap * sizeof(unsigned), st));
  EXA_CUDA(cudaMemsetAsync(g.hid.p, 0xff, hcap * sizeof(int), st));
  EXA_CUDA(cudaMemsetAsync(g.cnt.p, 0, 4 * sizeof(int), st));
  k_pair_class<<<kNumSMs * 8, 256, 0, st>>>(a.m2l_off, a.m2l_src, nc, a.cell_x, a.cell_pl, min_level, max_dl, g.hk.p,
                                            g.hc.p, hcap - 1, g.pair_slot.p);
  EXA_CHECK_LAUNCH();
  const int ccap = (int)std::min<long long>(hcap, (1LL << kClsBits) - 1);
  g.ck.ensure(ccap);
  g.ck_alt.ensure(ccap);
  g.cs.ensure(ccap);
  g.cs_alt.ensure(ccap);
  k_class_compact<<<kNumSMs * 4, 256, 0, st>>>(g.hk.p, g.hc.p, hcap, g.ck.p, g.cs.p, g.cnt.p, ccap);
  EXA_CHECK_LAUNCH();
  int ncls = 0;
  EXA_CUDA(cudaMemcpyAsync(&ncls, g.cnt.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  EXA_CUDA(cudaStreamSynchronize(st));
  if (ncls <= 0) return false;
  if (ncls > ccap) ncls = ccap;  // the overflow classes' pairs stay per-pair
  bool alt = radix_sort_u64((uint64_t *)g.ck.p, g.cs.p, (uint64_t *)g.ck_alt.p, g.cs_alt.p, ncls, 0, 56, C.sort,
                            C.err.p, st);
  unsigned long long *ck = alt ? g.ck_alt.p : g.ck.p;
  int *cs = alt ? g.cs_alt.p : g.cs.p;
  k_class_ids<<<(ncls + 255) / 256, 256, 0, st>>>(cs, ncls, g.hid.p);
  EXA_CHECK_LAUNCH();
  g.K.ensure((long long)ncls * NDP * NDP);
  {
    const size_t smem = tri(2 * P - 1) * sizeof(double2);
    k_build_K<<<ncls, 256, smem, st>>>(t, ck, P, g.K.p);
    EXA_CHECK_LAUNCH();
  }
  g.Msr.ensure(nc * NDP);
  k_scale_M_real<<<kNumSMs * 8, 256, 0, st>>>(t, a.M64, a.cell_x, nc, P, g.Msr.p);
  EXA_CHECK_LAUNCH();
  // ---- tiles
  g.taken.ensure(n_m2l);
  g.grp.ensure(nc);
  g.grp_alt.ensure(nc);
  g.cidx.ensure(nc);
  g.cidx_alt.ensure(nc);
  g.left_cnt.ensure(nc);
  g.left_off.ensure(nc + 1);
  g.left_src.ensure(n_m2l);
  k_gemm_flags<<<kNumSMs * 8, 256, 0, st>>>(a.m2l_off, a.m2l_src, nc, g.pair_slot.p, g.hid.p, a.cell_x, a.cell_pl,
                                            min_level, max_dl, g.taken.p, g.grp.p, g.cidx.p, g.left_cnt.p);
  EXA_CHECK_LAUNCH();
  LeftScan ls{g.left_cnt.p, g.left_off.p, nc};
  launch_scan<256, 8>(ls, nullptr, nc, nc, C.scan, C.err.p, st);
  k_left_fill<<<kNumSMs * 8, 256, 0, st>>>(a.m2l_off, a.m2l_src, nc, g.taken.p, a.cell_pl, min_level, max_dl,
                                           g.left_off.p, g.left_src.p);
  EXA_CHECK_LAUNCH();
  alt = radix_sort_u32(g.grp.p, g.cidx.p, g.grp_alt.p, g.cidx_alt.p, nc, 0, 8, C.sort, C.err.p, st);
  unsigned *gs = alt ? g.grp_alt.p : g.grp.p;
  int *csort = alt ? g.cidx_alt.p : g.cidx.p;
  g.gstart.ensure(256);
  g.tbase.ensure(256);
  k_tile_bases<<<1, 256, 0, st>>>(gs, nc, g.gstart.p, g.tbase.p, g.cnt.p + 1);
  EXA_CHECK_LAUNCH();
  const long long tiles_max = nc / kTile + 257;
  g.tile_of.ensure(nc);
  g.tile_cell.ensure(tiles_max * kTile);
  EXA_CUDA(cudaMemsetAsync(g.tile_cell.p, 0xff, tiles_max * kTile * sizeof(int), st));
  k_tile_assign<<<kNumSMs * 4, 256, 0, st>>>(gs, csort, nc, g.gstart.p, g.tbase.p, g.tile_of.p, g.tile_cell.p);
  EXA_CHECK_LAUNCH();
  // ---- pairs by (tile, class)
  g.pkey.ensure(n_m2l);
  g.pkey_alt.ensure(n_m2l);
  g.pval.ensure(n_m2l);
  g.pval_alt.ensure(n_m2l);
  k_pair_keys<<<kNumSMs * 8, 256, 0, st>>>(a.m2l_off, a.m2l_src, nc, g.pair_slot.p, g.hid.p, g.taken.p, g.tile_of.p,
                                           g.pkey.p, g.pval.p);
  EXA_CHECK_LAUNCH();
  const int end_bit = std::min(64, ((kClsBits + bits_for(tiles_max + 1)) + 7) / 8 * 8);
  alt = radix_sort_u64((uint64_t *)g.pkey.p, g.pval.p, (uint64_t *)g.pkey_alt.p, g.pval_alt.p, n_m2l, 0, end_bit,
                       C.sort, C.err.p, st);
  const unsigned long long *pk = alt ? g.pkey_alt.p : g.pkey.p;
  const int *pv = alt ? g.pval_alt.p : g.pval.p;
  // ---- tile products
  switch (NDP) {
#define EXA_GEMM_CASE(N)                                                                                        \
  case N: {                                                                                                     \
    const size_t smem = (size_t)(N * N + N * kTile) * sizeof(float);                                            \
    set_smem(k_m2l_gemm<N>, smem);                                                                              \
    k_m2l_gemm<N><<<(unsigned)tiles_max, N / 4 * (kTile / 4), smem, st>>>(pk, pv, n_m2l, g.cnt.p + 1, g.K.p,    \
                                                                         g.Msr.p, g.tile_cell.p, a.cell_x, t, P, \
                                                                         a.L64);                                 \
    break;                                                                                                      \
  }
    EXA_GEMM_CASE(16)
    EXA_GEMM_CASE(48)
    EXA_GEMM_CASE(64)
    EXA_GEMM_CASE(112)
#undef EXA_GEMM_CASE
    default: return false;
  }
  EXA_CHECK_LAUNCH();
  return true;
}

}  // namespace exafmm_b200
