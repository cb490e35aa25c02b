// Per-operator entry points (the examples/kernel.cxx known-answer chain) and the
// FP64 direct sum (Traversal::direct, include/traversal.h:355-377).  Each
// operator runs the same device kernel the solver uses, on a two- or few-cell
// tree assembled from the caller's arrays.
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/exafmm_b200.h"
#include "fmm.h"
#include "harmonics.cuh"

namespace exafmm_b200 {

namespace {

__global__ void k_direct(const double4 *tgt, long long nt, const double4 *src, long long ns, int prange,
                         double cycle, double4 *trg) {
  __shared__ double4 tile[256];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double4 xi = make_double4(0, 0, 0, 0);
  if (i < nt) xi = tgt[i];
  double pot = 0, ax = 0, ay = 0, az = 0;
  for (int ix = -prange; ix <= prange; ix++)
    for (int iy = -prange; iy <= prange; iy++)
      for (int iz = -prange; iz <= prange; iz++) {
        const double sx = ix * cycle, sy = iy * cycle, sz = iz * cycle;
        for (long long base = 0; base < ns; base += 256) {
          __syncthreads();
          if (base + threadIdx.x < ns) tile[threadIdx.x] = src[base + threadIdx.x];
          __syncthreads();
          const int cnt = (int)min((long long)256, ns - base);
          for (int s = 0; s < cnt; s++) {
            const double4 sj = tile[s];
            const double dx = xi.x - sj.x - sx, dy = xi.y - sj.y - sy, dz = xi.z - sj.z - sz;
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 != 0.0) {
              const double inv2 = 1.0 / r2;
              const double qr = sj.w * sqrt(inv2);
              const double s3 = inv2 * qr;
              pot += qr;
              ax += dx * s3;
              ay += dy * s3;
              az += dz * s3;
            }
          }
        }
      }
  if (i < nt) {
    double4 r = trg[i];
    r.x += pot;
    r.y -= ax;
    r.z -= ay;
    r.w -= az;
    trg[i] = r;
  }
}

// The MD wrappers' cutoff sum (wrappers/md_distributed.cxx:407-461): every
// source at every image -prange..prange whose separation is below the cutoff;
// image shifts rounded to float as the reference's Xperiodic[3] is.
__global__ void k_direct_cutoff(const double4 *tgt, long long nt, const double4 *src, long long ns, int prange,
                                double3 cycle, double cutoff2, double4 *trg) {
  __shared__ double4 tile[256];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double4 xi = make_double4(0, 0, 0, 0);
  if (i < nt) xi = tgt[i];
  double pot = 0, ax = 0, ay = 0, az = 0;
  for (int ix = -prange; ix <= prange; ix++)
    for (int iy = -prange; iy <= prange; iy++)
      for (int iz = -prange; iz <= prange; iz++) {
        const double sx = (double)(float)(ix * cycle.x), sy = (double)(float)(iy * cycle.y),
                     sz = (double)(float)(iz * cycle.z);
        for (long long base = 0; base < ns; base += 256) {
          __syncthreads();
          if (base + threadIdx.x < ns) tile[threadIdx.x] = src[base + threadIdx.x];
          __syncthreads();
          const int cnt = (int)min((long long)256, ns - base);
          for (int s = 0; s < cnt; s++) {
            const double4 sj = tile[s];
            const double dx = xi.x - sj.x - sx, dy = xi.y - sj.y - sy, dz = xi.z - sj.z - sz;
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < cutoff2 && r2 != 0.0) {
              const double inv = 1.0 / sqrt(r2);
              const double s3 = sj.w * inv * inv * inv;
              pot += sj.w * inv;
              ax += dx * s3;
              ay += dy * s3;
              az += dz * s3;
            }
          }
        }
      }
  if (i < nt) {
    double4 r = trg[i];
    r.x += pot;
    r.y -= ax;
    r.z -= ay;
    r.w -= az;
    trg[i] = r;
  }
}

// Device staging for one operator call.
struct Mini {
  cudaStream_t st = nullptr;
  std::vector<void *> bufs;
  Mini() { EXA_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)); }
  ~Mini() {
    cudaStreamSynchronize(st);
    for (void *p : bufs) cudaFree(p);
    cudaStreamDestroy(st);
  }
  template <typename T>
  T *up(const T *h, size_t n) {
    void *p = nullptr;
    EXA_CUDA(cudaMalloc(&p, (n ? n : 1) * sizeof(T)));
    bufs.push_back(p);
    if (n) EXA_CUDA(cudaMemcpyAsync(p, h, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return (T *)p;
  }
  template <typename T>
  void down(T *h, const T *d, size_t n) {
    if (n) EXA_CUDA(cudaMemcpyAsync(h, d, n * sizeof(T), cudaMemcpyDeviceToHost, st));
    EXA_CUDA(cudaStreamSynchronize(st));
  }
};

std::vector<long long> level_table(int level, long long count, long long start) {
  std::vector<long long> v(2 * (kMaxLevels + 1) + 4, 0);
  v[level] = count;
  v[kMaxLevels + 1 + level] = start;
  return v;
}

thread_local std::string g_err;

template <typename F>
int run(F &&f) {
  try {
    f();
    return 0;
  } catch (const std::exception &e) {
    g_err = e.what();
    return 1;
  }
}

void check_P(int P) {
  if (P < 2 || P > kMaxP) throw std::runtime_error("P must be in [2, 20]");
}

}  // namespace

void direct_fp64(const double4 *tgt, long long nt, const double4 *src, long long ns, int prange, double cycle,
                 double4 *trg, cudaStream_t st) {
  if (nt == 0) return;
  k_direct<<<(int)((nt + 255) / 256), 256, 0, st>>>(tgt, nt, src, ns, prange, cycle, trg);
  EXA_CHECK_LAUNCH();
}

}  // namespace exafmm_b200

using namespace exafmm_b200;

extern "C" {

const char *exafmm_kernel_error(void) { return g_err.c_str(); }

int exafmm_direct(const double *targets, long long nt, const double *sources, long long ns, int images,
                  double theta, double cycle, double *trg) {
  return run([&] {
    Mini m;
    int neighbor = (int)(2 * (0.5 / theta + 1) + 1);
    int prange = 0;
    for (int i = 0; i < images; i++) {
      int p = 1;
      for (int k = 0; k < i; k++) p *= neighbor;
      prange += p;
    }
    const double4 *t = m.up((const double4 *)targets, nt);
    const double4 *s = m.up((const double4 *)sources, ns);
    double4 *r = m.up((const double4 *)trg, nt);
    direct_fp64(t, nt, s, ns, prange, cycle, r, m.st);
    m.down((double4 *)trg, r, nt);
  });
}

int exafmm_direct_range(const double *targets, long long nt, const double *sources, long long ns, int prange,
                        double cycle, double *trg) {
  return run([&] {
    if (prange < 0) throw std::runtime_error("negative image range");
    Mini m;
    const double4 *t = m.up((const double4 *)targets, nt);
    const double4 *s = m.up((const double4 *)sources, ns);
    double4 *r = m.up((const double4 *)trg, nt);
    direct_fp64(t, nt, s, ns, prange, cycle, r, m.st);
    m.down((double4 *)trg, r, nt);
  });
}

int exafmm_direct_cutoff(const double *targets, long long nt, const double *sources, long long ns, int prange,
                         const double *cycle3, double cutoff, double *trg) {
  return run([&] {
    if (prange < 0) throw std::runtime_error("negative image range");
    if (!cycle3) throw std::runtime_error("null cycle");
    if (!(cutoff >= 0)) throw std::runtime_error("negative cutoff");
    if (nt == 0) return;
    Mini m;
    const double4 *t = m.up((const double4 *)targets, nt);
    const double4 *s = m.up((const double4 *)sources, ns);
    double4 *r = m.up((const double4 *)trg, nt);
    k_direct_cutoff<<<(int)((nt + 255) / 256), 256, 0, m.st>>>(t, nt, s, ns, prange,
                                                              make_double3(cycle3[0], cycle3[1], cycle3[2]),
                                                              cutoff * cutoff, r);
    EXA_CHECK_LAUNCH();
    m.down((double4 *)trg, r, nt);
  });
}

int exafmm_kernel_p2m(int P, const double *X, long long n, const double *xyzq, double *Mh) {
  return run([&] {
    check_P(P);
    Mini m;
    const int NT = tri(P);
    int4 cb = make_int4(0, (int)n, 0, 0);
    double4 cx = make_double4(X[0], X[1], X[2], 1.0);
    FmmArgs a;
    a.P = P;
    a.ncells = 1;
    a.stream = m.st;
    a.cell_b = m.up(&cb, 1);
    a.cell_x = m.up(&cx, 1);
    a.xt = m.up((const double4 *)xyzq, n);
    std::vector<double2> Mv(NT);
    a.M64 = m.up(Mv.data(), NT);
    p2m_fp64(a);
    m.down(Mv.data(), a.M64, NT);
    for (int o = 0; o < NT; o++) {
      Mh[2 * o] += Mv[o].x;
      Mh[2 * o + 1] += Mv[o].y;
    }
  });
}

int exafmm_kernel_m2m(int P, const double *Xp, int nchild, const double *Xc, const double *Mc, double *Mp) {
  return run([&] {
    check_P(P);
    Mini m;
    const int NT = tri(P);
    std::vector<int4> cb(nchild + 1, make_int4(0, 0, 0, 0));
    std::vector<double4> cx(nchild + 1);
    cb[0] = make_int4(0, 0, 1, nchild);
    cx[0] = make_double4(Xp[0], Xp[1], Xp[2], 1.0);
    for (int c = 0; c < nchild; c++) cx[c + 1] = make_double4(Xc[3 * c], Xc[3 * c + 1], Xc[3 * c + 2], 0.5);
    std::vector<double2> Mv((size_t)(nchild + 1) * NT, make_double2(0, 0));
    std::memcpy(Mv.data() + NT, Mc, (size_t)nchild * NT * sizeof(double2));
    auto lvl = level_table(0, 1, 0);
    int nd0 = 0;
    FmmArgs a;
    a.P = P;
    a.ncells = nchild + 1;
    a.stream = m.st;
    a.cell_b = m.up(cb.data(), cb.size());
    a.cell_x = m.up(cx.data(), cx.size());
    a.lvl = m.up(lvl.data(), lvl.size());
    a.nd_cell = m.up(&nd0, 1);
    a.M64 = m.up(Mv.data(), Mv.size());
    m2m_fp64(a, 0, 1);
    m.down(Mv.data(), a.M64, NT);
    for (int o = 0; o < NT; o++) {
      Mp[2 * o] += Mv[o].x;
      Mp[2 * o + 1] += Mv[o].y;
    }
  });
}

int exafmm_kernel_m2l(int P, const double *Xi, const double *Xj, const double *Mj, double *Li,
                      const double *Xper) {
  return run([&] {
    check_P(P);
    Mini m;
    const int NT = tri(P);
    double s[3] = {0, 0, 0};
    if (Xper) std::memcpy(s, Xper, sizeof(s));
    double4 cx[2] = {make_double4(Xi[0], Xi[1], Xi[2], 1.0),
                     make_double4(Xj[0] + s[0], Xj[1] + s[1], Xj[2] + s[2], 1.0)};
    int off[3] = {0, 1, 1};
    int src[1] = {1 | (13 << 26)};
    std::vector<double2> Mv(2 * NT, make_double2(0, 0)), Lv(2 * NT);
    std::memcpy(Mv.data() + NT, Mj, NT * sizeof(double2));
    std::memcpy(Lv.data(), Li, NT * sizeof(double2));
    FmmArgs a;
    a.P = P;
    a.ncells = 2;
    a.stream = m.st;
    a.cell_x = m.up(cx, 2);
    a.m2l_off = m.up(off, 3);
    a.m2l_src = m.up(src, 1);
    a.M64 = m.up(Mv.data(), Mv.size());
    a.L64 = m.up(Lv.data(), Lv.size());
    m2l_fp64(a);
    m.down((double2 *)Li, a.L64, NT);
  });
}

int exafmm_kernel_l2l(int P, const double *Xc, const double *Xp, const double *Lp, double *Lc) {
  return run([&] {
    check_P(P);
    Mini m;
    const int NT = tri(P);
    double4 cx[2] = {make_double4(Xp[0], Xp[1], Xp[2], 1.0), make_double4(Xc[0], Xc[1], Xc[2], 0.5)};
    int2 pl[2] = {make_int2(0, 0), make_int2(0, 1)};
    int ndc[2] = {0, 1};
    auto lvl = level_table(1, 1, 1);
    std::vector<double2> Lv(2 * NT);
    std::memcpy(Lv.data(), Lp, NT * sizeof(double2));
    std::memcpy(Lv.data() + NT, Lc, NT * sizeof(double2));
    FmmArgs a;
    a.P = P;
    a.ncells = 2;
    a.stream = m.st;
    a.cell_x = m.up(cx, 2);
    a.cell_pl = m.up(pl, 2);
    a.nd_cell = m.up(ndc, 2);
    a.lvl = m.up(lvl.data(), lvl.size());
    a.L64 = m.up(Lv.data(), Lv.size());
    l2l_fp64(a, 1, 1);
    m.down((double2 *)Lc, a.L64 + NT, NT);
  });
}

int exafmm_kernel_l2p(int P, const double *X, const double *L, long long n, const double *xyzq, double *trg) {
  return run([&] {
    check_P(P);
    Mini m;
    const int NT = tri(P);
    int4 cb = make_int4(0, (int)n, 0, 0);
    double4 cx = make_double4(X[0], X[1], X[2], 1.0);
    FmmArgs a;
    a.P = P;
    a.ncells = 1;
    a.stream = m.st;
    a.cell_b = m.up(&cb, 1);
    a.cell_x = m.up(&cx, 1);
    a.xt = m.up((const double4 *)xyzq, n);
    a.L64 = m.up((const double2 *)L, NT);
    a.trg64 = m.up((const double4 *)trg, n);
    l2p_fp64(a);
    m.down((double4 *)trg, a.trg64, n);
  });
}

int exafmm_kernel_p2p(long long ni, const double *xi, long long nj, const double *xj, const double *Xper,
                      double *trg) {
  return run([&] {
    Mini m;
    double s[3] = {0, 0, 0};
    if (Xper) std::memcpy(s, Xper, sizeof(s));
    std::vector<double4> x(ni + nj);
    std::memcpy(x.data(), xi, ni * sizeof(double4));
    for (long long j = 0; j < nj; j++)
      x[ni + j] = make_double4(xj[4 * j] + s[0], xj[4 * j + 1] + s[1], xj[4 * j + 2] + s[2], xj[4 * j + 3]);
    int4 cb[2] = {make_int4(0, (int)ni, 0, 0), make_int4((int)ni, (int)nj, 0, 0)};
    int off[3] = {0, 1, 1};
    int src[1] = {1 | (13 << 26)};
    std::vector<double4> t(ni + nj, make_double4(0, 0, 0, 0));
    std::memcpy(t.data(), trg, ni * sizeof(double4));
    FmmArgs a;
    a.ncrit = (int)(ni < 128 ? ni : 128);
    a.ncells = 2;
    a.stream = m.st;
    a.cell_b = m.up(cb, 2);
    a.xt = m.up(x.data(), x.size());
    a.p2p_off = m.up(off, 3);
    a.p2p_src = m.up(src, 1);
    a.trg64 = m.up(t.data(), t.size());
    p2p_fp64(a);
    m.down((double4 *)trg, a.trg64, ni);
  });
}

}  // extern "C"
