// Ewald summation (include/ewald.h:7-197) on the GPU, FP64: the periodic
// reference the lattice FMM is checked against.
//
//   wave part  (ewald.h:27-66, 160-176): S(k) = sum_j q_j exp(i 2 pi k.x_j / L)
//              over integer k with |k| <= ksize in the half space of
//              Ewald::initWaves (ewald.h:69-95); each S(k) scaled by
//              2 / (sigma L^3) exp(-K^2 / (4 alpha^2)) / K^2, K = 2 pi k / L; then
//              pot_i += Re S cos + Im S sin, grad_i -= (Re S sin - Im S cos) K.
//   real part  (ewald.h:98-145): pairs with 0 < r < cutoff under the minimum
//              image: pot += q erfc(alpha r) / r, grad -= dX q alpha^3
//              (2/sqrt(pi) e^{-(alpha r)^2} / (alpha r)^2 + erfc(alpha r) / (alpha r)^3).
//   self term  (ewald.h:150-155): pot_i -= 2/sqrt(pi) q_i alpha.
//
// The reference finds real-part neighbors by walking the source tree with the
// periodic image of each cell pair taken from their wrapped centers; here the
// bodies are binned on a periodic grid whose bins are at least a cutoff wide
// and each pair is taken at its nearest image.  For a cutoff below L/2 minus
// the leaf size the two select the same pairs.  Boxes too small for three bins
// a side use an all-pairs pass instead.
//
// DFT partial sums per (wave, body chunk) and every per-body loop run in a
// fixed order, so results are reproducible.
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/exafmm_b200.h"
#include "common.cuh"

namespace exafmm_b200 {
namespace {

constexpr int kThreads = 256;
constexpr long long kDftChunk = 8192;  // bodies per DFT block row

// Forward DFT, one thread per wave; blockIdx.y selects a chunk of bodies.
__global__ void k_dft(const double4 *x, long long n, const int4 *waves, int nw, double two_over_L, double2 *part) {
  __shared__ double4 sb[kThreads];
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  const long long b0 = (long long)blockIdx.y * kDftChunk;
  const long long b1 = min(n, b0 + kDftChunk);
  const int4 k = w < nw ? waves[w] : make_int4(0, 0, 0, 0);
  double re = 0.0, im = 0.0;
  for (long long base = b0; base < b1; base += kThreads) {
    __syncthreads();
    if (base + threadIdx.x < b1) sb[threadIdx.x] = x[base + threadIdx.x];
    __syncthreads();
    const int cnt = (int)min((long long)kThreads, b1 - base);
    for (int j = 0; j < cnt; j++) {
      const double4 b = sb[j];
      double s, c;
      sincospi((k.x * b.x + k.y * b.y + k.z * b.z) * two_over_L, &s, &c);
      re = fma(b.w, c, re);
      im = fma(b.w, s, im);
    }
  }
  if (w < nw) part[(long long)blockIdx.y * nw + w] = make_double2(re, im);
}

// S(k) = sum over chunks (in order), times the wave factor.
__global__ void k_wave_factor(const double2 *part, int nchunks, const int4 *waves, int nw, double scale, double coef,
                              double coef2, double2 *S) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nw) return;
  double re = 0.0, im = 0.0;
  for (int c = 0; c < nchunks; c++) {
    const double2 v = part[(long long)c * nw + w];
    re += v.x;
    im += v.y;
  }
  const int4 k = waves[w];
  const double kx = k.x * scale, ky = k.y * scale, kz = k.z * scale;
  const double K2 = kx * kx + ky * ky + kz * kz;
  const double f = coef * exp(-K2 * coef2) / K2;
  S[w] = make_double2(re * f, im * f);
}

// Inverse DFT, one thread per body; waves staged through shared memory.
__global__ void k_idft(const double4 *x, long long n, const int4 *waves, const double2 *S, int nw, double two_over_L,
                       double scale, double4 *trg) {
  __shared__ int4 sk[kThreads];
  __shared__ double2 ss[kThreads];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const double4 b = i < n ? x[i] : make_double4(0, 0, 0, 0);
  double pot = 0.0, f0 = 0.0, f1 = 0.0, f2 = 0.0;
  for (int base = 0; base < nw; base += kThreads) {
    __syncthreads();
    if (base + threadIdx.x < nw) {
      sk[threadIdx.x] = waves[base + threadIdx.x];
      ss[threadIdx.x] = S[base + threadIdx.x];
    }
    __syncthreads();
    const int cnt = min(kThreads, nw - base);
    for (int w = 0; w < cnt; w++) {
      const int4 k = sk[w];
      const double2 v = ss[w];
      double s, c;
      sincospi((k.x * b.x + k.y * b.y + k.z * b.z) * two_over_L, &s, &c);
      pot += v.x * c + v.y * s;
      const double d = v.x * s - v.y * c;
      f0 -= d * k.x;
      f1 -= d * k.y;
      f2 -= d * k.z;
    }
  }
  if (i < n) {
    double4 r = trg[i];
    r.x += pot;
    r.y += f0 * scale;
    r.z += f1 * scale;
    r.w += f2 * scale;
    trg[i] = r;
  }
}

__device__ __forceinline__ void real_pair(double dx, double dy, double dz, double q, double alpha, double rc2,
                                          double &pot, double &g0, double &g1, double &g2) {
  const double r2 = dx * dx + dy * dy + dz * dz;
  if (r2 > 0.0 && r2 < rc2) {
    const double r2s = r2 * alpha * alpha;
    const double rs = sqrt(r2s);
    const double inv = 1.0 / rs;
    const double inv2 = inv * inv;
    const double ec = erfc(rs);
    const double t = q * (M_2_SQRTPI * exp(-r2s) * inv2 + ec * inv2 * inv) * alpha * alpha * alpha;
    pot += q * ec * inv * alpha;
    g0 -= dx * t;
    g1 -= dy * t;
    g2 -= dz * t;
  }
}

// Real part over a periodic bin grid (nb >= 3 bins a side, bins >= cutoff wide);
// bodies sorted by bin, bin_start[nb^3 + 1].  xs = bodies wrapped into the box,
// in bin order; out index = caller index via order[].
__global__ void k_real_bins(const double4 *xs, const int *bin_of, const int *bin_start, const int *order, long long n,
                            int nb, double L, double alpha, double cutoff, double4 *trg) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 b = xs[i];
  const int bi = bin_of[i];
  const int ix = bi / (nb * nb), iy = (bi / nb) % nb, iz = bi % nb;
  const double rc2 = cutoff * cutoff;
  double pot = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
  for (int dx = -1; dx <= 1; dx++) {
    int jx = ix + dx;
    double sx = 0.0;
    if (jx < 0) { jx += nb; sx = -L; } else if (jx >= nb) { jx -= nb; sx = L; }
    for (int dy = -1; dy <= 1; dy++) {
      int jy = iy + dy;
      double sy = 0.0;
      if (jy < 0) { jy += nb; sy = -L; } else if (jy >= nb) { jy -= nb; sy = L; }
      for (int dz = -1; dz <= 1; dz++) {
        int jz = iz + dz;
        double sz = 0.0;
        if (jz < 0) { jz += nb; sz = -L; } else if (jz >= nb) { jz -= nb; sz = L; }
        const int bj = (jx * nb + jy) * nb + jz;
        for (int j = bin_start[bj]; j < bin_start[bj + 1]; j++) {
          const double4 s = xs[j];
          real_pair(b.x - s.x - sx, b.y - s.y - sy, b.z - s.z - sz, s.w, alpha, rc2, pot, g0, g1, g2);
        }
      }
    }
  }
  const int o = order[i];
  double4 r = trg[o];
  r.x += pot - M_2_SQRTPI * b.w * alpha;  // with the self term
  r.y += g0;
  r.z += g1;
  r.w += g2;
  trg[o] = r;
}

// All pairs at the nearest image (small boxes).
__global__ void k_real_all(const double4 *xs, long long n, double L, double alpha, double cutoff, double4 *trg) {
  __shared__ double4 tile[kThreads];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const double4 b = i < n ? xs[i] : make_double4(0, 0, 0, 0);
  const double rc2 = cutoff * cutoff;
  double pot = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
  for (long long base = 0; base < n; base += kThreads) {
    __syncthreads();
    if (base + threadIdx.x < n) tile[threadIdx.x] = xs[base + threadIdx.x];
    __syncthreads();
    const int cnt = (int)min((long long)kThreads, n - base);
    for (int j = 0; j < cnt; j++) {
      const double4 s = tile[j];
      double dx = b.x - s.x, dy = b.y - s.y, dz = b.z - s.z;
      dx -= L * rint(dx / L);
      dy -= L * rint(dy / L);
      dz -= L * rint(dz / L);
      real_pair(dx, dy, dz, s.w, alpha, rc2, pot, g0, g1, g2);
    }
  }
  if (i < n) {
    double4 r = trg[i];
    r.x += pot - M_2_SQRTPI * b.w * alpha;
    r.y += g0;
    r.z += g1;
    r.w += g2;
    trg[i] = r;
  }
}

struct Stage {
  cudaStream_t st = nullptr;
  std::vector<void *> bufs;
  Stage() { EXA_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)); }
  ~Stage() {
    cudaStreamSynchronize(st);
    for (void *p : bufs) cudaFree(p);
    cudaStreamDestroy(st);
  }
  template <typename T>
  T *alloc(size_t n) {
    void *p = nullptr;
    EXA_CUDA(cudaMalloc(&p, (n ? n : 1) * sizeof(T)));
    bufs.push_back(p);
    return (T *)p;
  }
  template <typename T>
  T *up(const T *h, size_t n) {
    T *p = alloc<T>(n);
    if (n) EXA_CUDA(cudaMemcpyAsync(p, h, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return p;
  }
};

thread_local std::string g_ewald_err;

// Ewald::initWaves (ewald.h:69-95): l >= 0; m >= 0 when l = 0; n >= 1 when l = m = 0.
std::vector<int4> init_waves(int ksize) {
  std::vector<int4> w;
  const int kmax2 = ksize * ksize;
  for (int l = 0; l <= ksize; l++) {
    const int mmin = l == 0 ? 0 : -ksize;
    for (int m = mmin; m <= ksize; m++) {
      const int nmin = (l == 0 && m == 0) ? 1 : -ksize;
      for (int n = nmin; n <= ksize; n++)
        if (l * l + m * m + n * n <= kmax2) w.push_back(make_int4(l, m, n, 0));
    }
  }
  return w;
}

}  // namespace
}  // namespace exafmm_b200

using namespace exafmm_b200;

extern "C" {

const char *exafmm_ewald_error(void) { return g_ewald_err.c_str(); }

int exafmm_ewald(const double *xyzq, long long n, int ksize, double alpha, double sigma, double cutoff, double cycle,
                 double *trg) {
  try {
    if (n < 0 || (n > 0 && (!xyzq || !trg))) throw std::runtime_error("bad body arrays");
    if (ksize < 0 || !(alpha > 0) || !(sigma > 0) || !(cutoff > 0) || !(cycle > 0))
      throw std::runtime_error("bad Ewald parameters");
    if (n == 0) return 0;
    const double L = cycle;
    // bodies wrapped into [-L/2, L/2): both parts are invariant under lattice shifts
    std::vector<double4> xw(n);
    for (long long i = 0; i < n; i++) {
      double v[3];
      for (int d = 0; d < 3; d++) {
        v[d] = xyzq[4 * i + d];
        v[d] -= L * std::floor(v[d] / L + 0.5);
      }
      xw[i] = make_double4(v[0], v[1], v[2], xyzq[4 * i + 3]);
    }
    Stage s;
    const double4 *dx = s.up(xw.data(), n);
    double4 *dtrg = s.up((const double4 *)trg, n);
    // ---- wave part
    const std::vector<int4> waves = init_waves(ksize);
    const int nw = (int)waves.size();
    if (nw > 0) {
      const int4 *dw = s.up(waves.data(), nw);
      const int nchunks = (int)((n + kDftChunk - 1) / kDftChunk);
      double2 *part = s.alloc<double2>((size_t)nchunks * nw);
      double2 *S = s.alloc<double2>(nw);
      dim3 g((nw + kThreads - 1) / kThreads, nchunks);
      k_dft<<<g, kThreads, 0, s.st>>>(dx, n, dw, nw, 2.0 / L, part);
      EXA_CHECK_LAUNCH();
      const double scale = 2 * M_PI / L;
      k_wave_factor<<<(nw + kThreads - 1) / kThreads, kThreads, 0, s.st>>>(
          part, nchunks, dw, nw, scale, 2 / sigma / (L * L * L), 1 / (4 * alpha * alpha), S);
      EXA_CHECK_LAUNCH();
      k_idft<<<(int)((n + kThreads - 1) / kThreads), kThreads, 0, s.st>>>(dx, n, dw, S, nw, 2.0 / L, scale, dtrg);
      EXA_CHECK_LAUNCH();
    }
    // ---- real part and self term
    const int nb = (int)std::floor(L / cutoff);
    if (nb >= 3) {
      const long long nbins = (long long)nb * nb * nb;
      if (nbins > (1LL << 30)) throw std::runtime_error("Ewald cutoff too small for the bin grid");
      std::vector<int> bin(n), start(nbins + 1, 0), order(n);
      for (long long i = 0; i < n; i++) {
        int c[3];
        const double v[3] = {xw[i].x, xw[i].y, xw[i].z};
        for (int d = 0; d < 3; d++) c[d] = std::min(nb - 1, std::max(0, (int)std::floor((v[d] + L / 2) / L * nb)));
        bin[i] = (c[0] * nb + c[1]) * nb + c[2];
        start[bin[i] + 1]++;
      }
      for (long long b = 0; b < nbins; b++) start[b + 1] += start[b];
      std::vector<int> fill(start.begin(), start.end() - 1);
      for (long long i = 0; i < n; i++) order[fill[bin[i]]++] = (int)i;  // stable: caller order within a bin
      std::vector<double4> xs(n);
      std::vector<int> bs(n);
      for (long long j = 0; j < n; j++) {
        xs[j] = xw[order[j]];
        bs[j] = bin[order[j]];
      }
      const double4 *dxs = s.up(xs.data(), n);
      const int *dbin = s.up(bs.data(), n);
      const int *dstart = s.up(start.data(), nbins + 1);
      const int *dorder = s.up(order.data(), n);
      k_real_bins<<<(int)((n + kThreads - 1) / kThreads), kThreads, 0, s.st>>>(dxs, dbin, dstart, dorder, n, nb, L,
                                                                             alpha, cutoff, dtrg);
      EXA_CHECK_LAUNCH();
    } else {
      k_real_all<<<(int)((n + kThreads - 1) / kThreads), kThreads, 0, s.st>>>(dx, n, L, alpha, cutoff, dtrg);
      EXA_CHECK_LAUNCH();
    }
    EXA_CUDA(cudaMemcpyAsync(trg, dtrg, n * sizeof(double4), cudaMemcpyDeviceToHost, s.st));
    EXA_CUDA(cudaStreamSynchronize(s.st));
    return 0;
  } catch (const std::exception &e) {
    g_ewald_err = e.what();
    return 1;
  }
}

}  // extern "C"
