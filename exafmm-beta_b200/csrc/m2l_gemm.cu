// M2L as dense products per offset class (the mixed form's FP32 M2L for regular
// pairs).
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
// one ND x ND real matrix K (built once per solve from FP64 harmonics).
//
// The pairs of each frequent class are sorted together; one block takes up to
// 128 of them and forms Y = K x [Ms of their sources] as a dense product in
// FP32 (the operator loaded once per block, 8 x 8 outputs per thread), writing
// each pair's column of Y at the pair's position in the target-grouped list.
// A second pass sums, per target, its pairs' columns in list order in FP64 and
// adds them to L: deterministic, no atomics.  The 4,096 multiply-adds per pair
// (at P = 8) replace the 9,216 of the pair-by-pair complex contraction.
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

// 4. Per target: flag the pairs of frequent classes (taken) and count the
// leftover pairs of the mixed policy (for the pair-by-pair kernel).
__device__ __forceinline__ bool policy_pair(int lt, int ls, int min_level, int max_dl) {
  const int dl = lt - ls;
  return lt >= min_level && dl <= max_dl && dl >= -max_dl;
}

__global__ void k_gemm_flags(const int *off, const int *src, long long ncells, const int *pair_slot, const int *hid,
                             const int2 *cell_pl, int min_level, int max_dl, unsigned char *taken, int *left_cnt,
                             unsigned *pkey, int *pval) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long c = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < ncells; c += warps) {
    const int b = off[c], e = off[c + 1];
    const int lt = cell_pl[c].y;
    int left = 0;
    for (int q = b + lane; q < e; q += 32) {
      const int s = pair_slot[q];
      const int cls = s >= 0 ? hid[s] : -1;
      taken[q] = cls >= 0 ? 1 : 0;
      pkey[q] = cls >= 0 ? (unsigned)cls : 0xffffffffu;  // sort key: class, the rest last
      pval[q] = q;
      if (cls < 0 && policy_pair(lt, cell_pl[src[q] & 0x3ffffff].y, min_level, max_dl)) left++;
    }
    for (int o = 16; o > 0; o >>= 1) left += __shfl_xor_sync(0xffffffffu, left, o);
    if (lane == 0) left_cnt[c] = left;
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

// The leftover pairs (not taken, inside the mixed policy) in list order.
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

// 5. Class ranges in the class-sorted pairs, and chunks of kChunk pairs.
constexpr int kChunk = 128;

__global__ void k_class_ranges(const unsigned *skey, long long n, int ncls, int *cstart) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= ncls; c += gridDim.x * blockDim.x) {
    long long lo = 0, hi = n;
    while (lo < hi) {
      const long long mid = (lo + hi) >> 1;
      if (skey[mid] < (unsigned)c) lo = mid + 1;
      else hi = mid;
    }
    cstart[c] = (int)lo;
  }
}

struct ChunkScan {
  using T = int;
  const int *cstart;
  int *cbase;
  int n;
  __device__ T value(long long i) const { return (cstart[i + 1] - cstart[i] + kChunk - 1) / kChunk; }
  __device__ void emit(long long i, const T &, const T &excl) const { cbase[i] = excl; }
  __device__ void total(const T &t) const { cbase[n] = t; }
};

__device__ __forceinline__ void cp_async16(void *sdst, const void *gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// 6. One block per chunk (one class, up to kChunk pairs): Y[pair] = K_class x Ms[source].
// The operator ([input][output]) and the sources' columns ([pair][input], row
// stride BSTR) are copied into shared memory with cp.async.  Thread (tx, ty)
// holds rows 4ty..4ty+3 and H+4ty..H+4ty+3 (H = NDP / 2) of columns tx + 4j,
// j < 8: both operand reads are conflict-free (rows: consecutive threads take
// consecutive 16-byte groups; columns: the four tx read four distinct banks),
// and every 16-byte column read feeds 32 multiply-adds over four inputs.
template <int NDP>
__global__ void __launch_bounds__(128)
k_m2l_class_gemm(const unsigned *skey, const int *sval, const int *cstart, const int *cbase, int ncls,
                 const int *src, const float *Kt, const float *Msr, float *Y) {
  constexpr int H = NDP / 2;
  constexpr int RG = H / 4;                      // row groups: 8 at NDP = 64
  constexpr int CG = 128 / RG;                   // column groups: 16 at NDP = 64
  constexpr int NC = CG * 8;                     // columns per pass
  constexpr int BSTR = NDP + 4;                  // floats per staged column
  extern __shared__ float4 smem4[];
  float *sK = reinterpret_cast<float *>(smem4);  // [NDP input][NDP output]
  float *sB = sK + NDP * NDP;                    // [kChunk pair][BSTR]
  __shared__ int s_q[kChunk], s_src[kChunk];
  const int chunk = blockIdx.x;
  if (chunk >= cbase[ncls]) return;
  int lo = 0, hi = ncls;  // class of this chunk: last c with cbase[c] <= chunk
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (cbase[mid] <= chunk) lo = mid;
    else hi = mid;
  }
  const int cls = lo;
  const int p0 = cstart[cls] + (chunk - cbase[cls]) * kChunk;
  const int cnt = min(kChunk, cstart[cls + 1] - p0);
  const float *Kg = Kt + (long long)cls * NDP * NDP;
  for (int i = threadIdx.x; i < NDP * NDP / 4; i += 128) cp_async16(sK + 4 * i, Kg + 4 * i);
  if (threadIdx.x < kChunk) {
    const int q = threadIdx.x < cnt ? sval[p0 + threadIdx.x] : -1;
    s_q[threadIdx.x] = q;
    s_src[threadIdx.x] = q >= 0 ? (src[q] & 0x3ffffff) : -1;
  }
  __syncthreads();
  for (int w = threadIdx.x; w < kChunk * (NDP / 4); w += 128) {
    const int i = w / (NDP / 4), q4 = w % (NDP / 4);
    float *dst = sB + i * BSTR + 4 * q4;
    if (i < cnt) cp_async16(dst, Msr + (long long)s_src[i] * NDP + 4 * q4);
    else *reinterpret_cast<float4 *>(dst) = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  cp_async_commit();
  cp_async_wait_all();
  __syncthreads();
  const int ty = threadIdx.x % RG, tx = threadIdx.x / RG;
  if (tx >= CG) return;  // 128 threads need not split evenly (no barrier follows)
  for (int c0 = 0; c0 < cnt; c0 += NC) {
    if (c0 + tx >= cnt) continue;
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
      for (int j = 0; j < 8; j++) acc[i][j] = 0.f;
    for (int k4 = 0; k4 < NDP; k4 += 4) {
      float4 b[8];
#pragma unroll
      for (int j = 0; j < 8; j++)  // columns past the chunk (discarded below) read its last column
        b[j] = *reinterpret_cast<const float4 *>(sB + min(c0 + tx + CG * j, kChunk - 1) * BSTR + k4);
#pragma unroll
      for (int kq = 0; kq < 4; kq++) {
        const float4 a0 = *reinterpret_cast<const float4 *>(sK + (k4 + kq) * NDP + 4 * ty);
        const float4 a1 = *reinterpret_cast<const float4 *>(sK + (k4 + kq) * NDP + H + 4 * ty);
        const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const float bv = kq == 0 ? b[j].x : kq == 1 ? b[j].y : kq == 2 ? b[j].z : b[j].w;
#pragma unroll
          for (int i = 0; i < 8; i++) acc[i][j] = fmaf(av[i], bv, acc[i][j]);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int i = c0 + tx + CG * j;
      if (i < cnt) {
        float *y = Y + (long long)s_q[i] * NDP;
        *reinterpret_cast<float4 *>(y + 4 * ty) = make_float4(acc[0][j], acc[1][j], acc[2][j], acc[3][j]);
        *reinterpret_cast<float4 *>(y + H + 4 * ty) = make_float4(acc[4][j], acc[5][j], acc[6][j], acc[7][j]);
      }
    }
  }
}

// 7. Per target: its taken pairs' contributions summed in list order in FP64,
// scaled by (-1)^j A_j^k R_t^{-(j+1)}, added to L.
template <int NDP>
__global__ void k_m2l_class_reduce(const int *off, long long ncells, const unsigned char *taken, const float *Y,
                                   const double4 *cell_x, DevTables t, int P, double2 *L) {
  constexpr int PER = (NDP + 31) / 32;
  const int lane = threadIdx.x & 31;
  const int NT = t.nterm, ND = nd_of(P);
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long c = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < ncells; c += warps) {
    const int b = off[c], e = off[c + 1];
    double acc[PER];
    bool any = false;
#pragma unroll
    for (int u = 0; u < PER; u++) acc[u] = 0.0;
    for (int q = b; q < e; q++) {
      if (!taken[q]) continue;
      any = true;
      const float *y = Y + (long long)q * NDP;
#pragma unroll
      for (int u = 0; u < PER; u++)
        if (lane + 32 * u < NDP) acc[u] += (double)y[lane + 32 * u];
    }
    if (!any) continue;
    const double rt = cell_x[c].w;
#pragma unroll
    for (int u = 0; u < PER; u++) {
      const int d = lane + 32 * u;
      if (d >= ND) continue;
      int j, k, part;
      dof_decode(d, NT, j, k, part);
      const int o = tri(j) + k;
      const double v = acc[u] * sgn_pow(j) * t.anm[o] * pow(rt, -(double)(j + 1));
      double2 *dst = &L[c * NT + o];
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

// Where the class products beat the pair-by-pair kernel for one solve on a
// B200: from about 1M pairs at P = 8 and 0.4M pairs at P = 10; at P <= 6 the
// pair-by-pair code is small and fast enough that they never do.
bool m2l_gemm_worthwhile(int P, long long n_m2l) {
  if (P == 8) return n_m2l >= 1000000;
  if (P == 10) return n_m2l >= 400000;
  return false;
}

bool m2l_gemm(Context &C, const FmmArgs &a, M2LGemmBufs &g, long long n_m2l, int min_level, int max_dl) {
  const int P = a.P;
  if (!m2l_gemm_supported(P) || a.ncells <= 0 || n_m2l <= 0) return false;
  if (!g.force && !m2l_gemm_worthwhile(P, n_m2l)) return false;
  cudaStream_t st = a.stream;
  const DevTables &t = device_tables(P);
  const long long nc = a.ncells;
  const int NDP = ndp_of(P);
  // ---- classes
  // classes are far fewer than pairs (thousands to ~1e5): a table of about a
  // sixteenth of the pairs, within [2^14, 2^20] slots; a pair that finds no
  // slot stays with the pair-by-pair kernel
  long long hcap = 1 << 14;
  while (hcap < n_m2l / 16 && hcap < (1LL << 20)) hcap <<= 1;
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
  // ---- pairs of frequent classes, sorted by class
  g.taken.ensure(n_m2l);
  g.left_cnt.ensure(nc);
  g.left_off.ensure(nc + 1);
  g.left_src.ensure(n_m2l);
  g.skey.ensure(n_m2l);
  g.skey_alt.ensure(n_m2l);
  g.pval.ensure(n_m2l);
  g.pval_alt.ensure(n_m2l);
  k_gemm_flags<<<kNumSMs * 8, 256, 0, st>>>(a.m2l_off, a.m2l_src, nc, g.pair_slot.p, g.hid.p, a.cell_pl, min_level,
                                            max_dl, g.taken.p, g.left_cnt.p, g.skey.p, g.pval.p);
  EXA_CHECK_LAUNCH();
  LeftScan ls{g.left_cnt.p, g.left_off.p, nc};
  launch_scan<256, 8>(ls, nullptr, nc, nc, C.scan, C.err.p, st);
  k_left_fill<<<kNumSMs * 8, 256, 0, st>>>(a.m2l_off, a.m2l_src, nc, g.taken.p, a.cell_pl, min_level, max_dl,
                                           g.left_off.p, g.left_src.p);
  EXA_CHECK_LAUNCH();
  const int end_bit = std::min(32, (bits_for(ncls + 1) + 7) / 8 * 8);
  alt = radix_sort_u32(g.skey.p, g.pval.p, g.skey_alt.p, g.pval_alt.p, n_m2l, 0, end_bit, C.sort, C.err.p, st);
  const unsigned *sk = alt ? g.skey_alt.p : g.skey.p;
  const int *sv = alt ? g.pval_alt.p : g.pval.p;
  g.cstart.ensure(ncls + 1);
  g.cbase.ensure(ncls + 1);
  k_class_ranges<<<(ncls + 256) / 256, 256, 0, st>>>(sk, n_m2l, ncls, g.cstart.p);
  EXA_CHECK_LAUNCH();
  ChunkScan cs2{g.cstart.p, g.cbase.p, ncls};
  launch_scan<256, 8>(cs2, nullptr, ncls, ncls, C.scan, C.err.p, st);
  // ---- products per class chunk, then per-target sums
  g.Y.ensure(n_m2l * NDP);
  const long long chunks_max = n_m2l / kChunk + ncls + 1;
  switch (NDP) {
#define EXA_GEMM_CASE(N)                                                                                      \
  case N: {                                                                                                   \
    const size_t smem = (size_t)(N * N + kChunk * (N + 4)) * sizeof(float);                                   \
    set_smem(k_m2l_class_gemm<N>, smem);                                                                      \
    k_m2l_class_gemm<N><<<(unsigned)chunks_max, 128, smem, st>>>(sk, sv, g.cstart.p, g.cbase.p, ncls,        \
                                                                 a.m2l_src, g.K.p, g.Msr.p, g.Y.p);           \
    EXA_CHECK_LAUNCH();                                                                                       \
    k_m2l_class_reduce<N><<<kNumSMs * 8, 256, 0, st>>>(a.m2l_off, nc, g.taken.p, g.Y.p, a.cell_x, t, P, a.L64); \
    EXA_CHECK_LAUNCH();                                                                                       \
    break;                                                                                                    \
  }
    EXA_GEMM_CASE(16)
    EXA_GEMM_CASE(48)
    EXA_GEMM_CASE(64)
    EXA_GEMM_CASE(112)
#undef EXA_GEMM_CASE
    default: return false;
  }
  return true;
}

}  // namespace exafmm_b200
