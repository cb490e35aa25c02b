// Mixed-precision P2P (kernels/laplace.h:150-235) in FP32.
//
// Each body is stored relative to the center of its own leaf as a two-float
// pair (hi + lo, about 48 significant bits), and each target is re-expressed
// relative to the source leaf in FP64 once per source leaf.  The separation of
// a pair is then (t_hi - s_hi) + (t_lo - s_lo): the hi difference is exact for
// close bodies, so close pairs keep their relative accuracy, and the rest of
// the interaction (r^2, rsqrt, the sums) is plain FP32.  Each target
// accumulates one source leaf at a time in FP32 and adds that partial into its
// running sums with Kahan compensation (include/kahan.h:34-48 semantics), so
// the error does not grow with the number of neighbour leaves.  Results are
// added to the FP64 outputs.
#include "fmm.h"

namespace exafmm_b200 {
namespace {

constexpr int kWarps = 4;

// x32[2i] = (hi of x - X_leaf, q), x32[2i+1] = (lo parts, 0).
__global__ void k_rel32(const int4 *cell_b, const double4 *cell_x, long long ncells, const double4 *xt, float4 *x32) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (long long c = (long long)blockIdx.x * kWarps + warp; c < ncells; c += (long long)gridDim.x * kWarps) {
    const int4 cb = cell_b[c];
    if (cb.w != 0) continue;
    const double4 X = cell_x[c];
    for (int i = lane; i < cb.y; i += 32) {
      const double4 b = xt[cb.x + i];
      const double dx = b.x - X.x, dy = b.y - X.y, dz = b.z - X.z;
      const float hx = (float)dx, hy = (float)dy, hz = (float)dz;
      x32[2 * (long long)(cb.x + i)] = make_float4(hx, hy, hz, (float)b.w);
      x32[2 * (long long)(cb.x + i) + 1] =
          make_float4((float)(dx - (double)hx), (float)(dy - (double)hy), (float)(dz - (double)hz), 0.f);
    }
  }
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

template <int TPL>
__global__ void __launch_bounds__(32 * kWarps)
k_p2p32(const int *off, const int *src, long long ncells, const int4 *cell_b, const double4 *cell_x,
        const float4 *x32, double4 *trg, double cycle) {
  __shared__ float4 shi[kWarps][32], slo[kWarps][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (long long c = (long long)blockIdx.x * kWarps + warp; c < ncells; c += (long long)gridDim.x * kWarps) {
    const int b = off[c], e = off[c + 1];
    if (b == e) continue;
    const int4 ci = cell_b[c];
    const double4 Xc = cell_x[c];
    for (int tb = 0; tb < ci.y; tb += 32 * TPL) {
      double xi[TPL], yi[TPL], zi[TPL];  // target offset from its own leaf center
      Kahan pot[TPL], ax[TPL], ay[TPL], az[TPL];
#pragma unroll
      for (int u = 0; u < TPL; u++) {
        const int i = tb + lane + 32 * u;
        float4 h = make_float4(0.f, 0.f, 0.f, 0.f), l = h;
        if (i < ci.y) {
          h = x32[2 * (long long)(ci.x + i)];
          l = x32[2 * (long long)(ci.x + i) + 1];
        }
        xi[u] = (double)h.x + (double)l.x;
        yi[u] = (double)h.y + (double)l.y;
        zi[u] = (double)h.z + (double)l.z;
      }
      for (int q = b; q < e; q++) {
        const int packed = src[q];
        const int cj = packed & 0x3ffffff, img = packed >> 26;
        const double4 Xj = cell_x[cj];
        const double Dx = Xj.x + (double)(img / 9 - 1) * cycle - Xc.x;
        const double Dy = Xj.y + (double)((img / 3) % 3 - 1) * cycle - Xc.y;
        const double Dz = Xj.z + (double)(img % 3 - 1) * cycle - Xc.z;
        const int4 cjb = cell_b[cj];
        // target relative to the source leaf center, as hi + lo floats
        float thx[TPL], thy[TPL], thz[TPL], tlx[TPL], tly[TPL], tlz[TPL];
        float pp[TPL], px[TPL], py[TPL], pz[TPL];
#pragma unroll
        for (int u = 0; u < TPL; u++) {
          const double tx = xi[u] - Dx, ty = yi[u] - Dy, tz = zi[u] - Dz;
          thx[u] = (float)tx;
          thy[u] = (float)ty;
          thz[u] = (float)tz;
          tlx[u] = (float)(tx - (double)thx[u]);
          tly[u] = (float)(ty - (double)thy[u]);
          tlz[u] = (float)(tz - (double)thz[u]);
          pp[u] = px[u] = py[u] = pz[u] = 0.f;
        }
        for (int sb = 0; sb < cjb.y; sb += 32) {
          const int ns = min(32, cjb.y - sb);
          if (lane < ns) {
            shi[warp][lane] = x32[2 * (long long)(cjb.x + sb + lane)];
            slo[warp][lane] = x32[2 * (long long)(cjb.x + sb + lane) + 1];
          }
          __syncwarp();
          for (int s = 0; s < ns; s++) {
            const float4 sh = shi[warp][s], sl = slo[warp][s];
#pragma unroll
            for (int u = 0; u < TPL; u++) {
              const float dx = (thx[u] - sh.x) + (tlx[u] - sl.x);
              const float dy = (thy[u] - sh.y) + (tly[u] - sl.y);
              const float dz = (thz[u] - sh.z) + (tlz[u] - sl.z);
              const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
              const float inv = (r2 > 0.f) ? rsqrtf(r2) : 0.f;
              const float qr = sh.w * inv;
              const float qr3 = qr * inv * inv;
              pp[u] += qr;
              px[u] = fmaf(dx, qr3, px[u]);
              py[u] = fmaf(dy, qr3, py[u]);
              pz[u] = fmaf(dz, qr3, pz[u]);
            }
          }
          __syncwarp();
        }
#pragma unroll
        for (int u = 0; u < TPL; u++) {
          pot[u].add(pp[u]);
          ax[u].add(px[u]);
          ay[u].add(py[u]);
          az[u].add(pz[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < TPL; u++) {
        const int i = tb + lane + 32 * u;
        if (i < ci.y) {
          double4 r = trg[ci.x + i];
          r.x += (double)pot[u].s - (double)pot[u].c;
          r.y -= (double)ax[u].s - (double)ax[u].c;
          r.z -= (double)ay[u].s - (double)ay[u].c;
          r.w -= (double)az[u].s - (double)az[u].c;
          trg[ci.x + i] = r;
        }
      }
    }
  }
}

int blocks_for(long long items) {
  long long g = (items + kWarps - 1) / kWarps;
  if (g > kNumSMs * 32) g = kNumSMs * 32;
  return g < 1 ? 1 : (int)g;
}

}  // namespace

void rel_bodies32(const FmmArgs &a, float4 *x32) {
  k_rel32<<<blocks_for(a.ncells), 32 * kWarps, 0, a.stream>>>(a.cell_b, a.cell_x, a.ncells, a.xt, x32);
  EXA_CHECK_LAUNCH();
}

void p2p_mixed(const FmmArgs &a, const float4 *x32) {
  const int tpl = (a.ncrit + 31) / 32;
  if (tpl <= 1)
    k_p2p32<1><<<blocks_for(a.ncells), 32 * kWarps, 0, a.stream>>>(a.p2p_off, a.p2p_src, a.ncells, a.cell_b,
                                                                   a.cell_x, x32, a.trg64, a.cycle);
  else if (tpl <= 2)
    k_p2p32<2><<<blocks_for(a.ncells), 32 * kWarps, 0, a.stream>>>(a.p2p_off, a.p2p_src, a.ncells, a.cell_b,
                                                                   a.cell_x, x32, a.trg64, a.cycle);
  else
    k_p2p32<4><<<blocks_for(a.ncells), 32 * kWarps, 0, a.stream>>>(a.p2p_off, a.p2p_src, a.ncells, a.cell_b,
                                                                   a.cell_x, x32, a.trg64, a.cycle);
  EXA_CHECK_LAUNCH();
}

}  // namespace exafmm_b200
