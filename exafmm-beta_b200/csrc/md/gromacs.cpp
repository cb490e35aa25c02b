// MD-code ABI in the shape of the reference's GROMACS wrapper
// (wrappers/gromacs.cxx:39-363), one process and one GPU; declared in
// include/exafmm_md.h, built as libexafmm_md_gromacs.so.  Host code over the
// engine's own C ABI: one solve context holds the tree, expansions and lists of
// the periodic system.
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/exafmm_b200.h"
#include "../../../include/exafmm_md.h"
#include "md_common.h"

namespace {

// FMM_Init's fixed parameters (wrappers/gromacs.cxx:40-43)
constexpr int kP = 10;
constexpr int kNcrit = 32;
constexpr int kNspawn = 1000;
constexpr double kTheta = 0.5;
// wrap codes ride in the top bits of Body::IBODY (wrappers/gromacs.cxx:96-97)
constexpr int kShift = 29;
constexpr int kMask = (int)~(0x7u << kShift);

struct MdState {
  exafmm_ctx *ctx = nullptr;
  int images = 0;
  bool verbose = false;
  std::string path = "./";
  double bounds[6] = {0, 0, 0, 0, 0, 0};  // local bounds of the last FMM_Partition
  bool have_bounds = false;
};

MdState *g_md = nullptr;
std::string g_error;

// vec.h:534-553 wrap / unwrap with a scalar period.
int wrap3(double v[3], double w) {
  const double ww[3] = {w, w, w};
  return exafmm_md::wrap3(v, ww);
}
void unwrap3(double v[3], double w, int iw) {
  const double ww[3] = {w, w, w};
  exafmm_md::unwrap3(v, ww, iw);
}

void check(int rc, const char *what) { exafmm_md::check(g_md ? g_md->ctx : nullptr, rc, what); }

MdState &state() {
  if (!g_md || !g_md->ctx) throw std::runtime_error("FMM_Init has not been called");
  return *g_md;
}

template <typename F>
void guarded(const char *name, F &&f) {
  exafmm_md::guarded(g_error, name, f);
}

// Bodies of FMM_Partition / FMM_Coulomb: X = x - cycle / 2, wrapped into the box.
std::vector<double> shifted_bodies(int n, const float *x, const float *q, double cycle, std::vector<int> *iwrap) {
  std::vector<double> b(4 * (size_t)n);
  if (iwrap) iwrap->resize(n);
  for (int i = 0; i < n; i++) {
    double X[3] = {(double)x[3 * i + 0] - cycle / 2, (double)x[3 * i + 1] - cycle / 2,
                   (double)x[3 * i + 2] - cycle / 2};
    const int w = wrap3(X, cycle);
    if (iwrap) (*iwrap)[i] = w;
    b[4 * i + 0] = X[0];
    b[4 * i + 1] = X[1];
    b[4 * i + 2] = X[2];
    b[4 * i + 3] = (double)q[i];
  }
  return b;
}

}  // namespace

extern "C" {

void FMM_Init(int images, int threads, bool verbose, const char *path) {
  (void)threads;
  guarded("FMM_Init", [&] {
    if (images < 0) throw std::runtime_error("images must be >= 0");
    if (g_md) {
      if (g_md->ctx) exafmm_destroy(g_md->ctx);
      delete g_md;
      g_md = nullptr;
    }
    MdState *s = new MdState;
    if (exafmm_create(&s->ctx, kP, kTheta, kNcrit, kNspawn, images, 2 * M_PI, EXAFMM_FP64, -1) != 0) {
      const std::string m = exafmm_create_error();
      delete s;
      throw std::runtime_error(m);
    }
    s->images = images;
    s->verbose = verbose;
    s->path = path ? path : "./";
    g_md = s;
  });
}

void FMM_Finalize(void) {
  guarded("FMM_Finalize", [&] {
    if (!g_md) return;
    if (g_md->ctx) exafmm_destroy(g_md->ctx);
    delete g_md;
    g_md = nullptr;
  });
}

void FMM_Partition(int *n, int *ibody, int *icell, float *x, float *q, float cycle) {
  guarded("FMM_Partition", [&] {
    MdState &s = state();
    if (!n || *n < 0) throw std::runtime_error("bad body count");
    const int N = *n;
    if (N > 0 && (!ibody || !icell || !x || !q)) throw std::runtime_error("null body array");
    for (int i = 0; i < N; i++)
      if (icell[i] < 0) throw std::runtime_error("residual groups (ICELL < 0) are not supported");
    const double c = (double)cycle;
    std::vector<int> iwrap;
    std::vector<double> b = shifted_bodies(N, x, q, c, &iwrap);
    check(exafmm_set_params(s.ctx, kP, kTheta, kNcrit, kNspawn, s.images, c), "set_params");
    check(exafmm_set_bodies(s.ctx, b.data(), N), "set_bodies");
    // BoundBox::getBounds, then Partition::octsection with one rank
    // (include/partition.h:185-207): Xmin stays, Xmax = Xmin + 1 * (Xmax - Xmin)
    double g[6];
    check(exafmm_get_bounds(s.ctx, g), "get_bounds");
    exafmm_md::octsection_one_rank(g, s.bounds);
    s.have_bounds = true;
    check(exafmm_build_tree(s.ctx, s.bounds), "build_tree");
    std::vector<int> perm(N);
    if (N) check(exafmm_get_perm(s.ctx, perm.data()), "get_perm");
    // bodies back in tree order, IBODY's wrap bits undone (wrappers/gromacs.cxx:125-135)
    const std::vector<int> ib(ibody, ibody + N), ic(icell, icell + N);
    const std::vector<float> qq(q, q + N);
    for (int i = 0; i < N; i++) {
      const int j = perm[i];
      double X[3] = {b[4 * j + 0], b[4 * j + 1], b[4 * j + 2]};
      unwrap3(X, c, iwrap[j]);
      ibody[i] = (ib[j] | (iwrap[j] << kShift)) & kMask;
      icell[i] = ic[j];
      for (int d = 0; d < 3; d++) x[3 * i + d] = (float)(X[d] + c / 2);
      q[i] = qq[j];
    }
  });
}

void FMM_Coulomb(int n, int *index, float *x, float *q, float *p, float *f, float cycle) {
  (void)index;
  guarded("FMM_Coulomb", [&] {
    MdState &s = state();
    if (!s.have_bounds) throw std::runtime_error("FMM_Partition has not been called");
    if (n < 0) throw std::runtime_error("bad body count");
    if (n > 0 && (!x || !q || !p || !f)) throw std::runtime_error("null body array");
    const double c = (double)cycle;
    std::vector<double> b = shifted_bodies(n, x, q, c, nullptr);
    check(exafmm_set_params(s.ctx, kP, kTheta, kNcrit, kNspawn, s.images, c), "set_params");
    check(exafmm_set_bodies(s.ctx, b.data(), n), "set_bodies");
    check(exafmm_build_tree(s.ctx, s.bounds), "build_tree");
    check(exafmm_upward(s.ctx), "upward");
    check(exafmm_traverse(s.ctx), "traverse");
    check(exafmm_downward(s.ctx), "downward");
    // UpDownPass::getDipole(bodies, 0) and dipoleCorrection(bodies, dipole, n, cycles)
    double dip[3];
    const double origin[3] = {0.0, 0.0, 0.0};
    check(exafmm_get_dipole(s.ctx, origin, dip), "get_dipole");
    check(exafmm_dipole_correction(s.ctx, dip, n), "dipole_correction");
    std::vector<double> trg(4 * (size_t)n);
    check(exafmm_get_results(s.ctx, trg.data()), "get_results");
    for (int i = 0; i < n; i++) {  // TRG starts from p, f (wrappers/gromacs.cxx:156-160)
      p[i] = (float)((double)p[i] + trg[4 * i + 0]);
      for (int d = 0; d < 3; d++) f[3 * i + d] = (float)((double)f[3 * i + d] + trg[4 * i + 1 + d]);
    }
  });
}

void Ewald_Coulomb(int n, float *x, float *q, float *p, float *f, int ksize, float alpha, float sigma, float cutoff,
                   float cycle) {
  guarded("Ewald_Coulomb", [&] {
    state();
    if (n < 0) throw std::runtime_error("bad body count");
    if (n > 0 && (!x || !q || !p || !f)) throw std::runtime_error("null body array");
    const double c = (double)cycle;
    std::vector<double> b(4 * (size_t)n), trg(4 * (size_t)n);
    for (int i = 0; i < n; i++) {  // wrappers/gromacs.cxx:230-243: X wrapped, TRG from p, f
      double X[3] = {(double)x[3 * i + 0], (double)x[3 * i + 1], (double)x[3 * i + 2]};
      wrap3(X, c);
      for (int d = 0; d < 3; d++) b[4 * i + d] = X[d];
      b[4 * i + 3] = (double)q[i];
      trg[4 * i + 0] = (double)p[i];
      for (int d = 0; d < 3; d++) trg[4 * i + 1 + d] = (double)f[3 * i + d];
    }
    if (exafmm_ewald(b.data(), n, ksize, alpha, sigma, cutoff, c, trg.data()) != 0)
      throw std::runtime_error(exafmm_ewald_error());
    for (int i = 0; i < n; i++) {
      p[i] = (float)trg[4 * i + 0];
      for (int d = 0; d < 3; d++) f[3 * i + d] = (float)trg[4 * i + 1 + d];
    }
  });
}

void Direct_Coulomb(int n, float *x, float *q, float *p, float *f, float cycle) {
  guarded("Direct_Coulomb", [&] {
    MdState &s = state();
    if (n < 0) throw std::runtime_error("bad body count");
    if (n > 0 && (!x || !q || !p || !f)) throw std::runtime_error("null body array");
    int prange = 0;  // wrappers/gromacs.cxx:292-296
    for (int i = 0, pw = 1; i < s.images; i++, pw *= 3) prange += pw;
    std::vector<double> b(4 * (size_t)n), trg(4 * (size_t)n, 0.0);
    for (int i = 0; i < n; i++) {
      for (int d = 0; d < 3; d++) b[4 * i + d] = (double)x[3 * i + d];
      b[4 * i + 3] = (double)q[i];
    }
    if (exafmm_direct_range(b.data(), n, b.data(), n, prange, (double)cycle, trg.data()) != 0)
      throw std::runtime_error(exafmm_kernel_error());
    // p += sum q/r; f -= sum dx q/r^3 (wrappers/gromacs.cxx:331-334), then the dipole
    // correction with the float dipole and coefficient of wrappers/gromacs.cxx:336-360
    for (int i = 0; i < n; i++) {
      p[i] = (float)((double)p[i] + trg[4 * i + 0]);
      for (int d = 0; d < 3; d++) f[3 * i + d] = (float)((double)f[3 * i + d] + trg[4 * i + 1 + d]);
    }
    float dipole[3] = {0, 0, 0};
    for (int i = 0; i < n; i++)
      for (int d = 0; d < 3; d++) dipole[d] += x[3 * i + d] * q[i];
    double norm = 0;
    for (int d = 0; d < 3; d++) norm += dipole[d] * dipole[d];
    const double cyc = (double)cycle;
    const float coef = (float)(4 * M_PI / (3 * cyc * cyc * cyc));
    for (int i = 0; i < n; i++) {
      p[i] -= coef * norm / n / q[i];
      for (int d = 0; d < 3; d++) f[3 * i + d] -= coef * dipole[d];
    }
  });
}

const char *FMM_Error(void) { return g_error.c_str(); }

}  // extern "C"
