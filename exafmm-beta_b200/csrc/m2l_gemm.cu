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
// The pairs of each class are sorted together; one block takes up to
// 128 of them and forms Y = K x [Ms of their sources] as a dense product in
// FP32 (the operator loaded once per block, 8 x 8 outputs per thread), writing
// each pair's column of Y at the pair's position in the target-grouped list.
// A second pass sums, per target, its pairs' columns in list order in FP64 and
// adds them to L: deterministic, no atomics.  The 4,096 multiply-adds per pair
// (at P = 8) replace the 9,216 of the pair-by-pair complex contraction.
//
// Pairs through periodic images form classes of their own (the image and the
// target level join the key, since the shift is not a multiple of the radii).
// Every class gets its operator, even one used by a single pair: leaving the
// classes of fewer than 8, 16, 32 or 64 pairs to the pair-by-pair kernel
// measured slower on a 4M-body solve, the 512-system batch and the periodic
// water box alike (the build of one more operator costs less than a pair
// through the pair-by-pair kernel's launches).  Pairs whose class found no
// hash slot stay with the pair-by-pair FP32 kernel, which then runs on a
// compacted list of just those pairs (left_off / left_src); pairs outside the
// mixed policy stay with the FP64 kernel as before.
//
// Two engines form the products.  The tensor-core one (k_m2l_class_mma) splits
// every operand entry into three bf16 pieces, x = hi + mid + lo (24 significant
// bits, the FP32 mantissa), and accumulates the six products of pieces whose
// weights reach 2^-16 (hi.hi, hi.mid, mid.hi, hi.lo, lo.hi, mid.mid) with
// tcgen05.mma into an FP32 accumulator in tensor memory: the terms left out
// weigh about 2^-24, FP32 rounding.  The CUDA-core one (k_m2l_class_gemm) is a
// plain FP32 product.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <type_traits>
#include <stdexcept>

#include "fmm.h"
#include "harmonics.cuh"
#include "scan.cuh"

namespace exafmm_b200 {
namespace {

constexpr unsigned long long kEmpty = ~0ull;
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

// Three bf16 pieces of x (hi, mid, lo; each the rounding of what the previous
// ones leave), as raw bits.
__device__ __forceinline__ void split_bf16x3(double x, unsigned short out[3]) {
#pragma unroll
  for (int p = 0; p < 3; p++) {
    const __nv_bfloat16 h = __double2bfloat16(x);
    out[p] = __bfloat16_as_ushort(h);
    x -= (double)__bfloat162float(h);
  }
}

// Offset, in bf16 elements, of entry (row, k) of a K-major tensor-core operand
// with NDP entries per row, in the canonical layout without swizzle: core
// matrices of 8 rows x 16 bytes (8 entries) stored as 128 contiguous bytes, the
// NDP / 8 core matrices of an 8-row group side by side along k (leading byte
// offset 128), row groups NDP / 8 x 128 bytes apart (stride byte offset).
__host__ __device__ __forceinline__ int core_off(int row, int k, int NDP) {
  return ((row >> 3) * (NDP >> 3) + (k >> 3)) * 64 + (row & 7) * 8 + (k & 7);
}

__device__ __forceinline__ unsigned long long class_key(int dl, long long dx, long long dy, long long dz) {
  return ((unsigned long long)(dl + 16) << 48) | ((unsigned long long)(dx + 32768) << 32) |
         ((unsigned long long)(dy + 32768) << 16) | (unsigned long long)(dz + 32768);
}

// A pair through a periodic image: the source sits at its cell's center plus
// the image shift (a multiple of the cycle, not of the radii), so the offset
// in units of the target radius is the integer offset of the two cells minus
// shift / R_t, which depends on the target level too.  Key: bit 63 set, the
// target level at bits 58-62, dl + 16 at 53-57, the image at 48-52, then the
// cells' integer offset as in class_key (whose keys keep bit 63 clear).
__device__ __forceinline__ unsigned long long class_key_image(int lt, int dl, int img, long long dx, long long dy,
                                                              long long dz) {
  return (1ull << 63) | ((unsigned long long)lt << 58) | ((unsigned long long)(dl + 16) << 53) |
         ((unsigned long long)img << 48) | ((unsigned long long)(dx + 32768) << 32) |
         ((unsigned long long)(dy + 32768) << 16) | (unsigned long long)(dz + 32768);
}

// 1. Per pair of the target-grouped list: its class's hash slot, or -1.
__global__ void k_pair_class(const int *off, const int *src, long long ncells, const double4 *cell_x,
                             const int2 *cell_pl, int min_level, int max_dl, unsigned long long *hk,
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
      if (lt >= min_level && lt < 32 && dl <= max_dl && dl >= -max_dl) {
        const double4 Xs = cell_x[cj];
        const double rmin = fmin(Xt.w, Xs.w);
        const double fx = rint((Xt.x - Xs.x) / rmin), fy = rint((Xt.y - Xs.y) / rmin), fz = rint((Xt.z - Xs.z) / rmin);
        if (fabs(fx) < 32767 && fabs(fy) < 32767 && fabs(fz) < 32767) {
          const unsigned long long key =
              img == 13 ? class_key(dl, (long long)fx, (long long)fy, (long long)fz)
                        : class_key_image(lt, dl, img, (long long)fx, (long long)fy, (long long)fz);
          long long h = (long long)(mix64(key) & (unsigned long long)hmask);
          for (int p = 0; p < kProbe; p++) {
            // a slot's key, once set, never changes: read it at L2 and CAS only
            // while the slot is still empty
            unsigned long long old = __ldcg(&hk[h]);
            if (old == kEmpty) old = atomicCAS(&hk[h], kEmpty, key);
            if (old == kEmpty || old == key) {
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

// 2. The classes (every occupied slot), in arbitrary order (sorted by key next).
__global__ void k_class_compact(const unsigned long long *hk, long long hcap,
                                unsigned long long *ck, int *cs, int *ncls, int cap) {
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < hcap; h += (long long)gridDim.x * blockDim.x) {
    if (hk[h] != kEmpty) {
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

// 3. Operator of each class: FP32 k-major, Kt[class][input dof][output dof]
// (CUDA-core engine), or three bf16 pieces of it per class, each an operand
// image of NDP output rows x NDP inputs in the core_off layout (tensor cores).
// cell_x[0].w (the root radius) and cycle place the image shifts of
// class_key_image keys (one system, never a forest, has image pairs).
// Operand layouts of k_build_K: FP32 k-major Kt[class][input][output] (CUDA
// cores), three bf16 pieces in the core_off image, or in the 128-byte-swizzled
// image (TMA).  NDP and the layout are template parameters so that mapping an
// entry's position to its (output, input) pair is shifts and constant
// divisions, not runtime divisions (the build was bound by integer work).
enum KLayout : int { kKFp32 = 0, kKCore = 1, kKSwizzled = 2 };

template <int NDP, int LAYOUT>
__global__ void __launch_bounds__(256)
k_build_K(DevTables t, const unsigned long long *ck, int P, float *Kt, unsigned short *Kb, const double4 *cell_x,
          double cycle) {
  extern __shared__ double2 S[];  // S'_p^q, q >= 0, at d / R_t
  constexpr int KB = (NDP + 63) / 64;  // 128-byte K-blocks of the swizzled image
  constexpr int IMG = LAYOUT == kKSwizzled ? KB * NDP * 64 : NDP * NDP;
  const int NT = t.nterm, ND = nd_of(P);
  const unsigned long long key = ck[blockIdx.x];
  const bool image = (key >> 63) != 0;
  const int dl = image ? (int)((key >> 53) & 31) - 16 : (int)((key >> 48) & 0xffff) - 16;
  const double ux = (double)(long long)((key >> 32) & 0xffff) - 32768.0;
  const double uy = (double)(long long)((key >> 16) & 0xffff) - 32768.0;
  const double uz = (double)(long long)(key & 0xffff) - 32768.0;
  const double to_rt = dl > 0 ? ldexp(1.0, -dl) : 1.0;  // min(R_s, R_t) / R_t
  double sx = 0.0, sy = 0.0, sz = 0.0;                    // image shift / R_t
  if (image) {
    const int lt = (int)((key >> 58) & 31), img = (int)((key >> 48) & 31);
    const double inv_rt = 1.0 / ldexp(cell_x[0].w, -lt);
    sx = (double)(img / 9 - 1) * cycle * inv_rt;
    sy = (double)((img / 3) % 3 - 1) * cycle * inv_rt;
    sz = (double)(img % 3 - 1) * cycle * inv_rt;
  }
  if ((int)threadIdx.x < 2 * P - 1)
    singular_column(t, threadIdx.x, 2 * P - 1, ux * to_rt - sx, uy * to_rt - sy, uz * to_rt - sz, t.ainv, S);
  // (n, m, part) of every real degree of freedom, decoded once per block, and
  // (R_s / R_t)^n for every source degree n
  __shared__ int dof_nmp[128];
  __shared__ double fn_of[32];
  for (int d = threadIdx.x; d < ND && d < 128; d += blockDim.x) {
    int n, m, part;
    dof_decode(d, NT, n, m, part);
    dof_nmp[d] = n | (m << 8) | (part << 16);
  }
  if ((int)threadIdx.x < P) fn_of[threadIdx.x] = ldexp(1.0, -dl * (int)threadIdx.x);
  __syncthreads();
  for (int e = threadIdx.x; e < IMG; e += blockDim.x) {
    int c, r;  // input and output dof; with Kb, e walks the operand image so the stores are contiguous
    if constexpr (LAYOUT == kKSwizzled) {  // K-block c / 64, row r, 16-byte chunk ((c % 64) / 8) ^ (r % 8)
      const int kb = e / (NDP * 64), w = e - kb * NDP * 64;
      r = w >> 6;
      c = kb * 64 + (((((w >> 3) & 7) ^ (r & 7))) << 3) + (w & 7);
    } else if constexpr (LAYOUT == kKCore) {
      const int ci = e >> 6, w = e & 63;
      r = (ci / (NDP >> 3)) * 8 + (w >> 3);
      c = (ci % (NDP >> 3)) * 8 + (w & 7);
    } else {
      c = e / NDP;
      r = e - c * NDP;
    }
    double val = 0.0;
    if (r < ND && c < ND) {
      const int er = dof_nmp[r], ec = dof_nmp[c];
      const int j = er & 0xff, k = (er >> 8) & 0xff, rp = er >> 16;
      const int n = ec & 0xff, mp = (ec >> 8) & 0xff, cp = ec >> 16;
      const double fn = fn_of[n];  // (R_s / R_t)^n
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
    if constexpr (LAYOUT == kKFp32) {
      Kt[(long long)blockIdx.x * NDP * NDP + c * NDP + r] = (float)val;
    } else {
      unsigned short h[3];
      split_bf16x3(val, h);
      unsigned short *dst = Kb + (long long)blockIdx.x * 3 * IMG + e;  // e == the operand offset of (r, c)
#pragma unroll
      for (int p = 0; p < 3; p++) dst[p * IMG] = h[p];
    }
  }
}

// Scaled multipoles over real degrees of freedom, padded to NDP: FP32 rows
// (Msr[cell][dof]), or three bf16 pieces per cell (Msb[cell][piece][dof]).
__global__ void k_scale_M_real(DevTables t, const double2 *M, const double4 *cell_x, long long ncells, int P,
                               float *Msr, unsigned short *Msb) {
  const int NT = t.nterm, ND = nd_of(P), NDP = ndp_of(P);
  const long long total = ncells * NDP;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long c = i / NDP;
    const int d = (int)(i - c * NDP);
    double v = 0.0;
    if (d < ND) {
      int n, m, part;
      dof_decode(d, NT, n, m, part);
      const int o = tri(n) + m;
      const double s = t.anm[o] * pow(cell_x[c].w, -(double)n);
      const double2 mv = M[c * NT + o];
      v = (part == 0 ? mv.x : mv.y) * s;
    }
    if (Msr) Msr[i] = (float)v;
    if (Msb) {
      unsigned short h[3];
      split_bf16x3(v, h);
#pragma unroll
      for (int p = 0; p < 3; p++) Msb[(c * 3 + p) * NDP + d] = h[p];
    }
  }
}

// 4. Per target: flag the pairs of classes with an operator (taken) and count the
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

// The pairs outside the mixed policy (root levels, large size ratios), which
// stay FP64: counted per target, then compacted in list order.
__global__ void k_complement_count(const int *off, const int *src, long long ncells, const int2 *cell_pl,
                                   int min_level, int max_dl, int *cnt) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long c = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < ncells; c += warps) {
    const int b = off[c], e = off[c + 1];
    const int lt = cell_pl[c].y;
    int k = 0;
    if (lt < min_level) {
      k = e - b;  // every pair of a root-level target
    } else {
      for (int q = b + lane; q < e; q += 32)
        if (!policy_pair(lt, cell_pl[src[q] & 0x3ffffff].y, min_level, max_dl)) k++;
      for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
    }
    if (lane == 0) cnt[c] = k;
  }
}

__global__ void k_complement_fill(const int *off, const int *src, long long ncells, const int2 *cell_pl,
                                  int min_level, int max_dl, const int *off2, int *src2) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long c = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < ncells; c += warps) {
    const int b = off[c], e = off[c + 1];
    const int lt = cell_pl[c].y;
    int at = off2[c];
    if (off2[c + 1] == at) continue;
    for (int base = b; base < e; base += 32) {
      const int q = base + lane;
      bool keep = false;
      int v = 0;
      if (q < e) {
        v = src[q];
        keep = lt < min_level || !policy_pair(lt, cell_pl[v & 0x3ffffff].y, min_level, max_dl);
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

// Per chunk: (class, first sorted position, pairs); and per sorted position of
// a taken pair, its source cell (so a product block starts from two
// independent loads rather than a search and a chain of dependent ones).
__global__ void k_chunk_table(const int *cstart, const int *cbase, int ncls, int4 *chunks) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncls; c += gridDim.x * blockDim.x) {
    const int b = cstart[c], e = cstart[c + 1];
    for (int j = cbase[c], p = b; p < e; j++, p += kChunk) chunks[j] = make_int4(c, p, min(kChunk, e - p), 0);
  }
}

__global__ void k_sorted_sources(const int *sval, const int *src, const int *ntaken, int *ssrc) {
  const int n = *ntaken;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    ssrc[i] = src[sval[i]] & 0x3ffffff;
}

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

// ---- tensor-core engine (tcgen05, sm_100a)
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of a K-major operand without swizzle:
// start address, leading byte offset (between the two core matrices along k
// that one instruction reads) and stride byte offset (between 8-row groups),
// all in 16-byte units; descriptor version 1 at bit 46; layout 0 = no swizzle.
__device__ __forceinline__ unsigned long long umma_desc(unsigned addr, unsigned lbo, unsigned sbo) {
  return (unsigned long long)((addr >> 4) & 0x3fffu) | ((unsigned long long)((lbo >> 4) & 0x3fffu) << 16) |
         ((unsigned long long)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_bf16(unsigned tmem_d, unsigned long long da, unsigned long long db, unsigned idesc,
                                          unsigned accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Waits for phase `parity` of the mbarrier at bar for at most about 2^31 clocks
// (about a second); false if it did not complete.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity) {
  const long long t0 = clock64();
  while (true) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > (1ll << 31)) return false;
  }
}

// TMEM columns: two accumulators of NDP FP32 columns each (hi.hi, and the
// five smaller products), at column 0 and NCOLS / 2; a power of two >= 32.
__host__ __device__ constexpr int mma_cols(int NDP) {
  return 2 * NDP <= 32 ? 32 : 2 * NDP <= 64 ? 64 : 2 * NDP <= 128 ? 128 : 256;
}

// Dynamic shared memory of k_m2l_class_mma<NDP>: the three pieces of the
// gathered source tile and of the operator, raised where needed to at least
// 456 bytes per TMEM column claimed.  An SM has 233,472 bytes of shared memory
// and 512 TMEM columns, so the CTAs that fit on one SM by shared memory never
// ask for more columns than it has and tcgen05.alloc never waits.
__host__ __device__ constexpr size_t mma_smem_bytes(int NDP) {
  return (size_t)3 * (kChunk * NDP + NDP * NDP) * 2 > (size_t)mma_cols(NDP) * 456
             ? (size_t)3 * (kChunk * NDP + NDP * NDP) * 2
             : (size_t)mma_cols(NDP) * 456;
}

// CTAs of k_m2l_class_mma<NDP> that fit on one SM (by shared memory).
__host__ __device__ constexpr int mma_ctas_per_sm(int NDP) {
  return (int)(233472 / (mma_smem_bytes(NDP) + 1152 + 1024));
}

// 6'. The per-class products on the tensor cores.  Persistent: each CTA takes a
// contiguous range of chunks (one class, up to kChunk pairs each; consecutive
// chunks mostly share a class, whose operator then stays in shared memory).
// Per chunk: D[pair][output] = sum_k Ms[source][k] K[k][output] with M = 128
// pairs, N = NDP outputs, K = NDP inputs, both operands K-major bf16 in shared
// memory (core_off layout), the accumulators (128 lanes x NDP FP32 columns) in
// tensor memory.  The tensor cores' FP32 sums are not round-to-nearest, so the
// hi.hi product gets its own accumulator and the five smaller products
// (2^-8 and 2^-16 of it) another: the large one sees NDP / 16 additions, and
// the epilogue adds the two in FP32.
// Per chunk j: thread 0 issues the 6 x NDP / 16 MMAs and commits them to an
// mbarrier; every thread loads chunk j+2's indices meanwhile (those of j+1
// were loaded during chunk j-1's products); once the
// products are done, all threads start the cp.async gather of chunk j+1's
// source pieces (lane pairs fetch whole 32-byte sectors) and, while it is in
// flight, read chunk j's accumulators (warp w: TMEM lanes 32w..32w+31) and
// write each pair's column of Y with 32-byte stores.
template <int NDP>
__device__ __forceinline__ void mma_gather(unsigned short *sA, unsigned short *sB, const int *s_src, int cnt,
                                           int cls, int &cur_cls, const unsigned short *Kb,
                                           const unsigned short *Msb) {
  constexpr int NG = NDP / 8, A_ELEMS = kChunk * NDP, B_ELEMS = NDP * NDP;
  if (cls != cur_cls) {  // a new class: its operator pieces
    const unsigned short *Kg = Kb + (long long)cls * 3 * B_ELEMS;
    for (int i = threadIdx.x; i < 3 * B_ELEMS / 8; i += 128) cp_async16(sB + 8 * i, Kg + 8 * i);
    cur_cls = cls;
  }
  // unit u: bit 0 = group parity, bits 1-4 = row within 16, then (row block of
  // 16, group pair, piece): a warp fetches 16 rows x 32 bytes (16 whole
  // sectors) and writes four whole core matrices (conflict-free)
  for (int u = threadIdx.x; u < kChunk * 3 * NG; u += 128) {
    const int i = ((u >> 5) & 7) * 16 + ((u >> 1) & 15);
    const int r2 = u >> 8;  // (group pair, piece)
    const int gp = r2 % (NG / 2), p = r2 / (NG / 2);
    const int g = 2 * gp + (u & 1);
    unsigned short *dst = sA + p * A_ELEMS + core_off(i, 8 * g, NDP);
    if (i < cnt) cp_async16(dst, Msb + ((long long)s_src[i] * 3 + p) * NDP + 8 * g);
    else *reinterpret_cast<uint4 *>(dst) = make_uint4(0u, 0u, 0u, 0u);
  }
  cp_async_commit();
}

// The gathered tiles complete and visible to the tensor cores; the previous
// TMEM reads ordered before the next MMAs.
__device__ __forceinline__ void mma_tiles_ready() {
  cp_async_wait_all();
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

__device__ __forceinline__ void tmem_ld16(unsigned taddr, unsigned (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

__device__ __forceinline__ void st_global_v8(float *p, const float (&v)[8]) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(v[0]), "f"(v[1]), "f"(v[2]),
               "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
               : "memory");
}

template <int NDP>
__global__ void __launch_bounds__(128)
k_m2l_class_mma(const int4 *chunks, const int *nchunks, const int *sval, const int *ssrc,
                const unsigned short *Kb, const unsigned short *Msb, float *Y, int *err) {
  constexpr int NG = NDP / 8;                // 16-byte groups per operand row
  constexpr int A_ELEMS = kChunk * NDP;      // one piece of the source tile
  constexpr int B_ELEMS = NDP * NDP;         // one piece of the operator
  constexpr int NCOLS = mma_cols(NDP);
  constexpr unsigned D1 = NCOLS / 2;         // column of the small products' accumulator
  constexpr unsigned SBO = NG * 128;         // bytes between 8-row groups
  // kind::f16 instruction descriptor: D FP32 (bits 4-5 = 1), A and B bf16
  // (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
  constexpr unsigned IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(NDP >> 3) << 17) |
                             ((unsigned)(kChunk >> 4) << 24);
  static_assert(NDP % 16 == 0 && NDP >= 16 && NDP <= 256, "N of an M = 128 MMA: multiple of 16 in [16, 256]");
  static_assert(2 * NDP <= NCOLS, "two accumulators");
  static_assert(kChunk == 128, "one TMEM lane and one thread per pair");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned short *sA = reinterpret_cast<unsigned short *>(smem_raw);
  unsigned short *sB = sA + 3 * A_ELEMS;
  __shared__ int s_src[kChunk];
  __shared__ __align__(8) unsigned long long s_bar;
  __shared__ unsigned s_tmem;
  const int total = *nchunks;
  const int j0 = (int)((long long)total * blockIdx.x / gridDim.x);
  const int j1 = (int)((long long)total * (blockIdx.x + 1) / gridDim.x);
  if (j0 >= j1) return;
  const unsigned bar = smem_u32(&s_bar);
  if (threadIdx.x < 32) {  // warp 0 owns the accumulators' columns
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(NCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  int4 ch = chunks[j0];  // this thread's pair of the first chunk
  int q = (int)threadIdx.x < ch.z ? sval[ch.y + threadIdx.x] : -1;
  s_src[threadIdx.x] = q >= 0 ? ssrc[ch.y + threadIdx.x] : -1;
  int cur_cls = -1;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = s_tmem;
  mma_gather<NDP>(sA, sB, s_src, ch.z, ch.x, cur_cls, Kb, Msb);
  // the next chunk's descriptor, list positions and sources, loaded one chunk
  // ahead of their use
  int4 chn = ch;
  int qn = -1, scn = -1;
  if (j0 + 1 < j1) {
    chn = chunks[j0 + 1];
    qn = (int)threadIdx.x < chn.z ? sval[chn.y + threadIdx.x] : -1;
    scn = (int)threadIdx.x < chn.z ? ssrc[chn.y + threadIdx.x] : -1;
  }
  mma_tiles_ready();
  for (int j = j0; j < j1; j++) {
    const int cnt = ch.z, qc = q;
    if (threadIdx.x == 0) {
      const unsigned a0 = smem_u32(sA), b0 = smem_u32(sB);
      // pieces (of the sources, of the operator): hi.hi into D0, the rest into D1
      const int pa[6] = {0, 0, 2, 1, 0, 1}, pb[6] = {0, 2, 0, 1, 1, 0};
#pragma unroll
      for (int t = 0; t < 6; t++)
#pragma unroll
        for (int k = 0; k < NDP / 16; k++) {  // 16 inputs = two core matrices = 256 bytes per step
          const unsigned long long da = umma_desc(a0 + (unsigned)(pa[t] * A_ELEMS * 2 + k * 256), 128, SBO);
          const unsigned long long db = umma_desc(b0 + (unsigned)(pb[t] * B_ELEMS * 2 + k * 256), 128, SBO);
          umma_bf16(tmem + (t == 0 ? 0u : D1), da, db, IDESC, (t > 1 || k > 0) ? 1u : 0u);
        }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                   : "memory");
    }
    int sc = -1;
    if (j + 1 < j1) {
      ch = chn;
      q = qn;
      sc = scn;
    }
    if (j + 2 < j1) {  // the chunk after, while the products run
      chn = chunks[j + 2];
      qn = (int)threadIdx.x < chn.z ? sval[chn.y + threadIdx.x] : -1;
      scn = (int)threadIdx.x < chn.z ? ssrc[chn.y + threadIdx.x] : -1;
    }
    bool done = true;  // one poller per warp
    if ((threadIdx.x & 31) == 0) done = mbar_wait_bounded(bar, (unsigned)((j - j0) & 1));
    done = __shfl_sync(0xffffffffu, done, 0);
    tc_fence_after();
    if (!__syncthreads_and(done)) {  // products done: the tiles and s_src are free
      if (threadIdx.x == 0) atomicOr(err, kErrMmaTimeout);
      break;
    }
    if (j + 1 < j1) {
      s_src[threadIdx.x] = sc;
      __syncthreads();
      mma_gather<NDP>(sA, sB, s_src, ch.z, ch.x, cur_cls, Kb, Msb);
    }
    {  // chunk j's accumulators -> Y, while the gather is in flight
      const int warp = threadIdx.x >> 5;  // row threadIdx.x = TMEM lane threadIdx.x
      const unsigned taddr = tmem + ((unsigned)(warp * 32) << 16);
      float *y = (int)threadIdx.x < cnt ? Y + (long long)qc * NDP : nullptr;
#pragma unroll
      for (int c0 = 0; c0 < NDP; c0 += 16) {
        unsigned r[16], v[16];
        tmem_ld16(taddr + (unsigned)c0, r);
        tmem_ld16(taddr + D1 + (unsigned)c0, v);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (y) {
#pragma unroll
          for (int h = 0; h < 2; h++) {
            float o[8];
#pragma unroll
            for (int e = 0; e < 8; e++) o[e] = __uint_as_float(r[8 * h + e]) + __uint_as_float(v[8 * h + e]);
            st_global_v8(y + c0 + 8 * h, o);
          }
        }
      }
    }
    mma_tiles_ready();
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOLS) : "memory");
  }
}

// ---- the P = 8 products with the source pieces gathered by TMA
// The operands in the canonical 128-byte-swizzle K-major layout: NDP = 64
// inputs per row = 128 bytes, row r at r * 128, its 16-byte chunk c stored at
// chunk position c ^ (r % 8), 8-row atoms of 1024 bytes (1024-byte aligned).
// TMA writes the source rows in this layout itself (tensor map swizzle 128B);
// the operator image is written so by k_build_K: entry (row, k) at bf16 offset
// row * 64 + (((k / 8) ^ (row % 8)) * 8) + k % 8.

// Shared-memory matrix descriptor of a K-major, 128-byte-swizzled operand:
// start address, stride byte offset 1024 (8-row atoms), leading byte offset
// unused (1), version 1, layout SWIZZLE_128B (2 at bit 61).
__device__ __forceinline__ unsigned long long umma_desc_sw128(unsigned addr) {
  return (unsigned long long)((addr >> 4) & 0x3fffu) | (1ull << 16) | ((unsigned long long)(1024 >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Four source rows (cells y0..y3, 64 bf16 from column x) into 4 x 128 bytes at dst.
__device__ __forceinline__ void tma_gather4(unsigned dst, const CUtensorMap *map, unsigned bar, int x, int y0, int y1,
                                            int y2, int y3) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(bar), "r"(x), "r"(y0), "r"(y1), "r"(y2), "r"(y3)
      : "memory");
}

// 128-byte K-blocks per operand row, and the kernel's shared memory (A and B
// pieces in K-blocks, plus alignment slack).
__host__ __device__ constexpr int tma_kblocks(int NDP) { return (NDP + 63) / 64; }
__host__ __device__ constexpr size_t tma_smem_bytes(int NDP) {
  return (size_t)3 * tma_kblocks(NDP) * (kChunk + NDP) * 128 + 1024;
}

// As k_m2l_class_mma<NDP>, with the chunk's source pieces (3 x KB x 128 rows
// x 128 bytes, KB = 1 at P = 8, 2 at P = 10) brought in by 96 KB
// tile::gather4 loads (3 KB per lane of warp 0) completing on an mbarrier,
// instead of cp.async of all threads.  At NDP = 112 the second K-block holds
// inputs 64-127 of a row: past 112 it reads the next piece (or zeros past the
// row's end), which no MMA step reaches (the last one ends at input 112).
template <int NDP>
__global__ void __launch_bounds__(128)
k_m2l_class_mma_tma(const __grid_constant__ CUtensorMap msb_map, const int4 *chunks, const int *nchunks,
                    const int *sval, const int *ssrc, const unsigned short *Kb, float *Y, int *err) {
  constexpr int KB = tma_kblocks(NDP);
  constexpr int A_ELEMS = KB * kChunk * 64, B_ELEMS = KB * NDP * 64;  // one piece of each, in K-blocks
  constexpr int NCOLS = mma_cols(NDP);
  constexpr unsigned D1 = NCOLS / 2;
  constexpr unsigned IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(NDP >> 3) << 17) |
                             ((unsigned)(kChunk >> 4) << 24);
  constexpr unsigned A_BYTES = 3 * A_ELEMS * 2;
  static_assert(NDP % 16 == 0 && NDP <= 128, "one or two 128-byte K-blocks");
  extern __shared__ unsigned char smem_raw[];
  unsigned short *sA = reinterpret_cast<unsigned short *>(
      (reinterpret_cast<unsigned long long>(smem_raw) + 1023) & ~1023ull);
  unsigned short *sB = sA + 3 * A_ELEMS;
  __shared__ int s_src[kChunk];
  __shared__ __align__(8) unsigned long long s_bar, s_tbar;
  __shared__ unsigned s_tmem;
  const int total = *nchunks;
  const int j0 = (int)((long long)total * blockIdx.x / gridDim.x);
  const int j1 = (int)((long long)total * (blockIdx.x + 1) / gridDim.x);
  if (j0 >= j1) return;
  const unsigned bar = smem_u32(&s_bar), tbar = smem_u32(&s_tbar);
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(NCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  int4 ch = chunks[j0];
  int q = (int)threadIdx.x < ch.z ? sval[ch.y + threadIdx.x] : -1;
  s_src[threadIdx.x] = q >= 0 ? ssrc[ch.y + threadIdx.x] : -1;
  int cur_cls = -1;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = s_tmem;
  const unsigned a0 = smem_u32(sA), b0 = smem_u32(sB);
  // one chunk's loads: the operator pieces if the class changed (cp.async, all
  // threads), the source pieces by TMA (thread 0); rows past the chunk repeat
  // its first source (their products are not stored)
  auto issue_loads = [&](int cls, int cnt) {
    if (cls != cur_cls) {
      const unsigned short *Kg = Kb + (long long)cls * 3 * B_ELEMS;
      for (int i = threadIdx.x; i < 3 * B_ELEMS / 8; i += 128) cp_async16(sB + 8 * i, Kg + 8 * i);
      cur_cls = cls;
    }
    cp_async_commit();
    if (threadIdx.x < 32) {  // warp 0: lane g issues row group g of every piece and K-block
      if (threadIdx.x == 0) mbar_expect_tx(tbar, A_BYTES);
      __syncwarp();
      const int g = threadIdx.x, f = s_src[0];
      int y[4];
#pragma unroll
      for (int u = 0; u < 4; u++) y[u] = 4 * g + u < cnt ? s_src[4 * g + u] : f;
#pragma unroll
      for (int p = 0; p < 3; p++)
#pragma unroll
        for (int kb = 0; kb < KB; kb++)
          tma_gather4(a0 + (unsigned)(p * A_ELEMS * 2 + kb * kChunk * 128 + g * 512), &msb_map, tbar,
                      p * NDP + 64 * kb, y[0], y[1], y[2], y[3]);
    }
  };
  issue_loads(ch.x, ch.z);
  // the next chunk's descriptor, list positions and sources, loaded one chunk
  // ahead of their use (so the three dependent loads are not waited for
  // between the products and the next gather)
  int4 chn = ch;
  int qn = -1, scn = -1;
  if (j0 + 1 < j1) {
    chn = chunks[j0 + 1];
    qn = (int)threadIdx.x < chn.z ? sval[chn.y + threadIdx.x] : -1;
    scn = (int)threadIdx.x < chn.z ? ssrc[chn.y + threadIdx.x] : -1;
  }
  bool ok = true;
  for (int j = j0; j < j1; j++) {
    const int cnt = ch.z, qc = q, it = j - j0;
    // this chunk's tiles: the source pieces (TMA) and the operator (cp.async)
    bool got = true;
    if ((threadIdx.x & 31) == 0) got = mbar_wait_bounded(tbar, (unsigned)(it & 1));
    got = __shfl_sync(0xffffffffu, got, 0);
    cp_async_wait_all();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    if (!__syncthreads_and(got)) {
      ok = false;
      break;
    }
    tc_fence_after();
    if (threadIdx.x == 0) {
      const int pa[6] = {0, 0, 2, 1, 0, 1}, pb[6] = {0, 2, 0, 1, 1, 0};
#pragma unroll
      for (int t = 0; t < 6; t++)
#pragma unroll
        for (int k = 0; k < NDP / 16; k++) {  // 16 inputs = 32 bytes along the swizzled rows of K-block k / 4
          const int kb = k >> 2, kk = k & 3;
          const unsigned long long da =
              umma_desc_sw128(a0 + (unsigned)(pa[t] * A_ELEMS * 2 + kb * kChunk * 128 + kk * 32));
          const unsigned long long db =
              umma_desc_sw128(b0 + (unsigned)(pb[t] * B_ELEMS * 2 + kb * NDP * 128 + kk * 32));
          umma_bf16(tmem + (t == 0 ? 0u : D1), da, db, IDESC, (t > 1 || k > 0) ? 1u : 0u);
        }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                   : "memory");
    }
    int sc = -1;
    if (j + 1 < j1) {
      ch = chn;
      q = qn;
      sc = scn;
    }
    if (j + 2 < j1) {  // the chunk after, while the products run
      chn = chunks[j + 2];
      qn = (int)threadIdx.x < chn.z ? sval[chn.y + threadIdx.x] : -1;
      scn = (int)threadIdx.x < chn.z ? ssrc[chn.y + threadIdx.x] : -1;
    }
    bool done = true;
    if ((threadIdx.x & 31) == 0) done = mbar_wait_bounded(bar, (unsigned)(it & 1));
    done = __shfl_sync(0xffffffffu, done, 0);
    tc_fence_after();
    if (!__syncthreads_and(done)) {  // products done: the tiles and s_src are free
      ok = false;
      break;
    }
    if (j + 1 < j1) {
      s_src[threadIdx.x] = sc;
      __syncthreads();
      issue_loads(ch.x, ch.z);
    }
    {  // chunk j's accumulators -> Y, while the next loads are in flight
      const int warp = threadIdx.x >> 5;
      const unsigned taddr = tmem + ((unsigned)(warp * 32) << 16);
      float *yrow = (int)threadIdx.x < cnt ? Y + (long long)qc * NDP : nullptr;
#pragma unroll
      for (int c0 = 0; c0 < NDP; c0 += 16) {
        unsigned r[16], v[16];
        tmem_ld16(taddr + (unsigned)c0, r);
        tmem_ld16(taddr + D1 + (unsigned)c0, v);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (yrow) {
#pragma unroll
          for (int h = 0; h < 2; h++) {
            float o[8];
#pragma unroll
            for (int e = 0; e < 8; e++) o[e] = __uint_as_float(r[8 * h + e]) + __uint_as_float(v[8 * h + e]);
            st_global_v8(yrow + c0 + 8 * h, o);
          }
        }
      }
    }
  }
  if (!ok && (threadIdx.x & 31) == 0) atomicOr(err, kErrMmaTimeout);
  cp_async_wait_all();
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOLS) : "memory");
  }
}

// 7. Per target cell, in list order: the sum of its taken pairs' columns of
// Y (FP64), scaled by (-1)^j A_j^k R_t^{-(j+1)}, added to L.  Lane l holds
// entries VEC l .. VEC l + VEC - 1 of a column (VEC = 4 floats, one 16-byte
// load per lane and pair, for NDP > 64; else 2).  A group's rows are loaded
// together with its taken flags (the rows of pairs not taken hold whatever is
// there and are dropped by a select, so the loads do not wait for the flags),
// and the next group's loads are in flight while this one is added.
template <int NDP>
__global__ void k_m2l_class_reduce(const int *off, long long ncells, const unsigned char *taken, const float *Y,
                                   const double4 *cell_x, DevTables t, int P, double2 *L) {
  constexpr int VEC = NDP > 64 ? 4 : 2;
  constexpr int LANES = NDP / VEC;  // lanes that hold entries
  static_assert(NDP % VEC == 0 && LANES <= 32, "one row per warp-wide load");
  constexpr int G = 8;
  using V = typename std::conditional<VEC == 4, float4, float2>::type;
  const int lane = threadIdx.x & 31;
  const bool active = lane < LANES;
  const int NT = t.nterm, ND = nd_of(P);
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  auto load = [&](int q, int e, bool &tk, V &v) {
    tk = false;
    v = V{};
    if (q < e) {
      tk = taken[q] != 0;
      if (active) v = reinterpret_cast<const V *>(Y + (long long)q * NDP)[lane];
    }
  };
  for (long long c = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < ncells; c += warps) {
    const int b = off[c], e = off[c + 1];
    double acc[VEC];
#pragma unroll
    for (int i = 0; i < VEC; i++) acc[i] = 0.0;
    bool any = false;
    bool tk[G], tk2[G];
    V v[G], v2[G];
#pragma unroll
    for (int i = 0; i < G; i++) load(b + i, e, tk[i], v[i]);
    for (int q0 = b; q0 < e; q0 += G) {
#pragma unroll
      for (int i = 0; i < G; i++) load(q0 + G + i, e, tk2[i], v2[i]);  // the next group, in flight
#pragma unroll
      for (int i = 0; i < G; i++) {
        if (!tk[i]) continue;
        any = true;
        const float *f = reinterpret_cast<const float *>(&v[i]);
#pragma unroll
        for (int k = 0; k < VEC; k++) acc[k] += (double)f[k];
      }
#pragma unroll
      for (int i = 0; i < G; i++) {
        tk[i] = tk2[i];
        v[i] = v2[i];
      }
    }
    if (!any || !active) continue;
    const double rt = cell_x[c].w;
#pragma unroll
    for (int h = 0; h < VEC; h++) {
      const int d = VEC * lane + h;
      if (d >= ND) continue;
      int j, k, part;
      dof_decode(d, NT, j, k, part);
      const int o = tri(j) + k;
      const double val = acc[h] * sgn_pow(j) * t.anm[o] * pow(rt, -(double)(j + 1));
      double2 *dst = &L[c * NT + o];
      if (part == 0) dst->x += val;
      else dst->y += val;
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

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled from the driver (no link-time dependency on libcuda).
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// The bf16 source pieces Msb[cell][3 x NDP] as a 2-D tensor (3 NDP x ncells),
// read in boxes of one row x 64 elements (128 bytes) into the 128-byte-swizzled
// layout.
bool msb_tensor_map(CUtensorMap *map, const unsigned short *Msb, long long ncells, int NDP) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn || ncells <= 0 || ncells > 0x7fffffffLL) return false;
  if ((reinterpret_cast<unsigned long long>(Msb) & 15ull) != 0) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)(3 * NDP), (cuuint64_t)ncells};
  const cuuint64_t strides[1] = {(cuuint64_t)(3 * NDP * sizeof(unsigned short))};
  const cuuint32_t box[2] = {64, 1};
  const cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)Msb, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int NDP>
void tma_launch(const CUtensorMap &map, M2LGemmBufs &g, const int *sv, long long chunks_max, int ncls, int *err,
                cudaStream_t st) {
  if constexpr (NDP == 64) {  // the two-K-block form (NDP = 112) measured slower than cp.async at P = 10
    constexpr size_t smem = tma_smem_bytes(NDP);
    set_smem(k_m2l_class_mma_tma<NDP>, smem);
    const int per_sm = (int)(233472 / (smem + 640 + 1024));
    const long long grid = std::min<long long>(chunks_max, (long long)kNumSMs * per_sm);
    k_m2l_class_mma_tma<NDP><<<(unsigned)grid, 128, smem, st>>>(map, g.chunks.p, g.cbase.p + ncls, sv, g.ssrc.p,
                                                                g.Kb.p, g.Y.p, err);
  }
}

}  // namespace

bool m2l_gemm_supported(int P) { return P == 4 || P == 6 || P == 8 || P == 10; }

// Where the class products beat the pair-by-pair kernel for one solve on a
// B200, measured on cube and Plummer systems of 20K-1M bodies (theta 0.4,
// ncrit 64): from about 0.15M pairs at P = 10, 1M at P = 8 and 8M at P = 6
// (at P = 4 the pair-by-pair code always wins), and only when the classes
// hold at least kMinPairsPerClass pairs on average, since every class costs
// an operator build: a 50K-body Plummer system at P = 10 (510K pairs, 73 per
// class) solved in 5.1 ms pair by pair and 6.6 ms with the products, a
// 100K-body cube (597K pairs, 89 per class) in 5.9 and 5.4 ms.
bool m2l_gemm_worthwhile(int P, long long n_m2l) {
  if (P == 6) return n_m2l >= 8000000;
  if (P == 8) return n_m2l >= 1000000;
  if (P == 10) return n_m2l >= 150000;
  return false;
}
constexpr long long kMinPairsPerClass = 80;

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
  g.hid.ensure(hcap);
  g.pair_slot.ensure(n_m2l);
  g.cnt.ensure(4);
  EXA_CUDA(cudaMemsetAsync(g.hk.p, 0xff, hcap * sizeof(unsigned long long), st));
  EXA_CUDA(cudaMemsetAsync(g.hid.p, 0xff, hcap * sizeof(int), st));
  EXA_CUDA(cudaMemsetAsync(g.cnt.p, 0, 4 * sizeof(int), st));
  k_pair_class<<<kNumSMs * 8, 256, 0, st>>>(a.m2l_off, a.m2l_src, nc, a.cell_x, a.cell_pl, min_level, max_dl, g.hk.p,
                                            hcap - 1, g.pair_slot.p);
  EXA_CHECK_LAUNCH();
  const int ccap = (int)std::min<long long>(hcap, (1LL << kClsBits) - 1);
  g.ck.ensure(ccap);
  g.ck_alt.ensure(ccap);
  g.cs.ensure(ccap);
  g.cs_alt.ensure(ccap);
  k_class_compact<<<kNumSMs * 4, 256, 0, st>>>(g.hk.p, hcap, g.ck.p, g.cs.p, g.cnt.p, ccap);
  EXA_CHECK_LAUNCH();
  int *ncls_h = reinterpret_cast<int *>(C.pin + kPinScratch);  // the context's pinned staging
  EXA_CUDA(cudaMemcpyAsync(ncls_h, g.cnt.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  EXA_CUDA(cudaStreamSynchronize(st));
  int ncls = *ncls_h;
  if (ncls <= 0) return false;
  if (!g.force && n_m2l < kMinPairsPerClass * (long long)ncls) return false;  // too many classes for their pairs
  if (ncls > ccap) ncls = ccap;  // the overflow classes' pairs stay per-pair
  bool alt = radix_sort_u64((uint64_t *)g.ck.p, g.cs.p, (uint64_t *)g.ck_alt.p, g.cs_alt.p, ncls, 0, 64, C.sort,
                            C.err.p, st);
  unsigned long long *ck = alt ? g.ck_alt.p : g.ck.p;
  int *cs = alt ? g.cs_alt.p : g.cs.p;
  k_class_ids<<<(ncls + 255) / 256, 256, 0, st>>>(cs, ncls, g.hid.p);
  EXA_CHECK_LAUNCH();
  const bool tc = g.tensor_cores;
  // P = 8 on the tensor cores: source pieces gathered by TMA (its tensor map made below).
  // At P = 10 (two 128-byte K-blocks, one CTA per SM either way) the cp.async
  // form is a little faster (M2L 16.4 vs 16.8 ms on a 1M-charge periodic box).
  CUtensorMap msb_map;
  bool use_tma = tc && NDP == 64 && g.tma && encode_tiled() != nullptr;
  if (tc) g.Kb.ensure((long long)ncls * 3 * (use_tma ? tma_kblocks(NDP) * NDP * 64 : NDP * NDP));
  else g.K.ensure((long long)ncls * NDP * NDP);
  {
    const size_t smem = tri(2 * P - 1) * sizeof(double2);
    float *Kt = tc ? nullptr : g.K.p;
    unsigned short *Kb = tc ? g.Kb.p : nullptr;
    auto build = [&](auto kernel) {
      kernel<<<ncls, 256, smem, st>>>(t, ck, P, Kt, Kb, a.cell_x, a.cycle);
      EXA_CHECK_LAUNCH();
    };
    switch (NDP) {
#define EXA_BUILD_K_CASE(N)                                      \
  case N:                                                        \
    if (!tc) build(k_build_K<N, kKFp32>);                        \
    else if (use_tma) build(k_build_K<N, kKSwizzled>);           \
    else build(k_build_K<N, kKCore>);                            \
    break;
      EXA_BUILD_K_CASE(16)
      EXA_BUILD_K_CASE(48)
      EXA_BUILD_K_CASE(64)
      EXA_BUILD_K_CASE(112)
#undef EXA_BUILD_K_CASE
      default: return false;
    }
  }
  if (tc) g.Msb.ensure(nc * 3 * NDP);
  else g.Msr.ensure(nc * NDP);
  if (use_tma && !msb_tensor_map(&msb_map, g.Msb.p, nc, NDP))
    throw std::runtime_error("TMA tensor map of the multipoles");
  k_scale_M_real<<<kNumSMs * 8, 256, 0, st>>>(t, a.M64, a.cell_x, nc, P, tc ? nullptr : g.Msr.p,
                                              tc ? g.Msb.p : nullptr);
  EXA_CHECK_LAUNCH();
  // ---- pairs of classes with an operator, sorted by class
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
  launch_scan<1024, 8>(ls, nullptr, nc, nc, C.scan, C.err.p, st);
  k_left_fill<<<kNumSMs * 8, 256, 0, st>>>(a.m2l_off, a.m2l_src, nc, g.taken.p, a.cell_pl, min_level, max_dl,
                                           g.left_off.p, g.left_src.p);
  EXA_CHECK_LAUNCH();
  const int end_bit = std::min(32, bits_for(ncls + 1));  // class ids; the untaken key 0xffffffff sorts last
  alt = radix_sort_u32(g.skey.p, g.pval.p, g.skey_alt.p, g.pval_alt.p, n_m2l, 0, end_bit, C.sort, C.err.p, st);
  const unsigned *sk = alt ? g.skey_alt.p : g.skey.p;
  const int *sv = alt ? g.pval_alt.p : g.pval.p;
  g.cstart.ensure(ncls + 1);
  g.cbase.ensure(ncls + 1);
  k_class_ranges<<<(ncls + 256) / 256, 256, 0, st>>>(sk, n_m2l, ncls, g.cstart.p);
  EXA_CHECK_LAUNCH();
  ChunkScan cs2{g.cstart.p, g.cbase.p, ncls};
  launch_scan<1024, 8>(cs2, nullptr, ncls, ncls, C.scan, C.err.p, st);
  const long long chunks_max = n_m2l / kChunk + ncls + 1;
  if (tc) {
    g.chunks.ensure(chunks_max);
    g.ssrc.ensure(n_m2l);
    k_chunk_table<<<(ncls + 255) / 256, 256, 0, st>>>(g.cstart.p, g.cbase.p, ncls, g.chunks.p);
    EXA_CHECK_LAUNCH();
    const int grid = (int)std::min<long long>(kNumSMs * 8, (n_m2l + 255) / 256);
    k_sorted_sources<<<grid, 256, 0, st>>>(sv, a.m2l_src, g.cstart.p + ncls, g.ssrc.p);
    EXA_CHECK_LAUNCH();
  }
  // ---- products per class chunk, then per-target sums
  g.Y.ensure(n_m2l * NDP);
  switch (NDP) {
#define EXA_GEMM_CASE(N)                                                                                      \
  case N: {                                                                                                   \
    if (use_tma) {                                                                                            \
      tma_launch<N>(msb_map, g, sv, chunks_max, ncls, C.err.p, st);                                           \
    } else if (tc) {                                                                                          \
      const size_t smem = mma_smem_bytes(N);                                                                  \
      set_smem(k_m2l_class_mma<N>, smem);                                                                     \
      const long long grid = std::min<long long>(chunks_max, (long long)kNumSMs * mma_ctas_per_sm(N));        \
      k_m2l_class_mma<N><<<(unsigned)grid, 128, smem, st>>>(g.chunks.p, g.cbase.p + ncls, sv, g.ssrc.p,       \
                                                            g.Kb.p, g.Msb.p, g.Y.p, C.err.p);                 \
    } else {                                                                                                  \
      const size_t smem = (size_t)(N * N + kChunk * (N + 4)) * sizeof(float);                                 \
      set_smem(k_m2l_class_gemm<N>, smem);                                                                    \
      k_m2l_class_gemm<N><<<(unsigned)chunks_max, 128, smem, st>>>(sk, sv, g.cstart.p, g.cbase.p, ncls,      \
                                                                   a.m2l_src, g.K.p, g.Msr.p, g.Y.p);         \
    }                                                                                                         \
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

long long m2l_complement(Context &C, const FmmArgs &a, M2LGemmBufs &g, long long n_m2l, int min_level, int max_dl) {
  const long long nc = a.ncells;
  cudaStream_t st = a.stream;
  g.comp_cnt.ensure(nc);
  g.comp_off.ensure(nc + 1);
  g.comp_src.ensure(n_m2l > 0 ? n_m2l : 1);
  const int grid = (int)std::max<long long>(1, std::min<long long>(kNumSMs * 8, (nc + 7) / 8));
  k_complement_count<<<grid, 256, 0, st>>>(a.m2l_off, a.m2l_src, nc, a.cell_pl, min_level, max_dl, g.comp_cnt.p);
  EXA_CHECK_LAUNCH();
  LeftScan ls{g.comp_cnt.p, g.comp_off.p, nc};
  launch_scan<1024, 8>(ls, nullptr, nc, nc, C.scan, C.err.p, st);
  k_complement_fill<<<grid, 256, 0, st>>>(a.m2l_off, a.m2l_src, nc, a.cell_pl, min_level, max_dl, g.comp_off.p,
                                          g.comp_src.p);
  EXA_CHECK_LAUNCH();
  return nc;
}

}  // namespace exafmm_b200
