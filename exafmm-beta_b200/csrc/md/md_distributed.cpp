// MD-code ABI in the shape of the reference's distributed MD wrapper
// (wrappers/md_distributed.cxx:36-461), one process and one GPU; declared in
// include/exafmm_md_distributed.h, built as libexafmm_md_distributed.so.  Host
// code over the engine's own C ABI.  With one process the MPI steps (bounds
// all-reduce, octsection across ranks, body and LET exchange, the ring shifts
// of the direct sums) take their one-rank form, so the solve is the local tree
// alone and the ghost bodies come from the 26 periodic images of the bodies.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/exafmm_b200.h"
#include "../../../include/exafmm_md_distributed.h"
#include "md_common.h"

namespace {

// FMM_Init's fixed parameters (wrappers/md_distributed.cxx:37-39)
constexpr int kP = 10;
constexpr int kNcrit = 32;
constexpr int kNspawn = 1000;

struct MdState {
  exafmm_ctx *ctx = nullptr;
  int images = 0;
  double theta = 0.5;
  double cutoff = 0;
  bool verbose = false;
  std::string path = "./";
  double bounds[6] = {0, 0, 0, 0, 0, 0};  // localBounds of the last Set_Index / FMM_Partition
  bool have_bounds = false;
};

MdState *g_md = nullptr;
std::string g_error;

MdState &state() {
  if (!g_md || !g_md->ctx) throw std::runtime_error("FMM_Init has not been called");
  return *g_md;
}

void check(int rc, const char *what) { exafmm_md::check(g_md ? g_md->ctx : nullptr, rc, what); }

template <typename F>
void guarded(const char *name, F &&f) {
  exafmm_md::guarded(g_error, name, f);
}

double cubic(const double *cycle) {
  if (!cycle) throw std::runtime_error("null cycle");
  if (cycle[0] != cycle[1] || cycle[0] != cycle[2])
    throw std::runtime_error("the periodic solve needs a cubic box (cycle[0] == cycle[1] == cycle[2])");
  return cycle[0];
}

void need_bodies(int n, const void *a, const void *b, const void *c, const void *d) {
  if (n < 0) throw std::runtime_error("bad body count");
  if (n > 0 && (!a || !b || !c || !d)) throw std::runtime_error("null body array");
}

// The bodies of Set_Index / FMM_Partition / FMM_FMM: x wrapped into the box
// (md_distributed.cxx:97-109), the wrap codes kept.
std::vector<double> wrapped_bodies(int n, const double *x, const double *q, const double *cycle,
                                   std::vector<int> &iwrap) {
  std::vector<double> b(4 * (size_t)n);
  iwrap.resize(n);
  for (int i = 0; i < n; i++) {
    double X[3] = {x[3 * i + 0], x[3 * i + 1], x[3 * i + 2]};
    iwrap[i] = exafmm_md::wrap3(X, cycle);
    b[4 * i + 0] = X[0];
    b[4 * i + 1] = X[1];
    b[4 * i + 2] = X[2];
    b[4 * i + 3] = q[i];
  }
  return b;
}

// Tree order back to the caller's arrays (md_distributed.cxx:125-141,
// 171-187): res_index from Body::ICELL, x unwrapped, q and v moved with their
// bodies.
void write_back(int n, const std::vector<int> &perm, const std::vector<double> &b, const std::vector<int> &iwrap,
                const std::vector<int> &icell, const double *cycle, int *res_index, double *x, double *q, double *v) {
  const std::vector<double> v0(v, v + 3 * (size_t)n);
  for (int i = 0; i < n; i++) {
    const int j = perm[i];
    double X[3] = {b[4 * j + 0], b[4 * j + 1], b[4 * j + 2]};
    exafmm_md::unwrap3(X, cycle, iwrap[j]);
    res_index[i] = icell[i];
    for (int d = 0; d < 3; d++) {
      x[3 * i + d] = X[d];
      v[3 * i + d] = v0[3 * j + d];
    }
    q[i] = b[4 * j + 3];
  }
}

// getBounds, optionally the one-rank octsection, buildTree; returns the tree
// order (perm[i] = caller index of tree slot i).
std::vector<int> build(MdState &s, const std::vector<double> &b, int n, double cycle, bool octsection) {
  check(exafmm_set_params(s.ctx, kP, s.theta, kNcrit, kNspawn, s.images, cycle), "set_params");
  check(exafmm_set_bodies(s.ctx, b.data(), n), "set_bodies");
  double g[6];
  check(exafmm_get_bounds(s.ctx, g), "get_bounds");
  if (octsection) exafmm_md::octsection_one_rank(g, s.bounds);
  else
    for (int k = 0; k < 6; k++) s.bounds[k] = g[k];
  s.have_bounds = true;
  check(exafmm_build_tree(s.ctx, s.bounds), "build_tree");
  std::vector<int> perm(n);
  if (n) check(exafmm_get_perm(s.ctx, perm.data()), "get_perm");
  return perm;
}

}  // namespace

extern "C" {

void FMM_Init(int images, int threads, double theta, double cutoff, bool verbose, const char *path) {
  (void)threads;
  guarded("FMM_Init", [&] {
    if (images < 0) throw std::runtime_error("images must be >= 0");
    if (!(theta > 0)) throw std::runtime_error("theta must be > 0");
    if (g_md) {
      if (g_md->ctx) exafmm_destroy(g_md->ctx);
      delete g_md;
      g_md = nullptr;
    }
    MdState *s = new MdState;
    if (exafmm_create(&s->ctx, kP, theta, kNcrit, kNspawn, images, 2 * M_PI, EXAFMM_FP64, -1) != 0) {
      const std::string m = exafmm_create_error();
      delete s;
      throw std::runtime_error(m);
    }
    s->images = images;
    s->theta = theta;
    s->cutoff = cutoff;
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

void Set_Index(int *ni, int nimax, int *res_index, double *x, double *q, double *v, double *cycle) {
  guarded("Set_Index", [&] {
    MdState &s = state();
    if (!ni) throw std::runtime_error("bad body count");
    const int n = *ni;
    need_bodies(n, res_index, x, q, v);
    if (!cycle) throw std::runtime_error("null cycle");
    std::vector<int> iwrap;
    const std::vector<double> b = wrapped_bodies(n, x, q, cycle, iwrap);
    // getBounds then buildTree (md_distributed.cxx:110-111); the upward pass
    // there leaves nothing these outputs read.
    const std::vector<int> perm = build(s, b, n, cycle[0], false);
    long long nc = 0;
    check(exafmm_tree_info(s.ctx, &nc, nullptr, nullptr, nullptr), "tree_info");
    std::vector<int> ci(5 * (size_t)nc);
    if (nc) check(exafmm_get_cells(s.ctx, ci.data(), nullptr), "get_cells");
    // Group labels (md_distributed.cxx:113-124): every cell, in cell order,
    // walks the bodies it spans; a group starts at its first body and closes
    // after 3..5 bodies at random (one drand48 draw a body, from the process's
    // drand48 sequence) or after 6.  A group's first body gets the next id,
    // the others -(place in the group).  Leaves come after their ancestors, so
    // the last label a body gets is its leaf's.
    std::vector<int> icell(n);
    int id = 0;
    for (long long c = 0; c < nc; c++) {
      int ic = 0;
      for (int k = ci[5 * c + 3]; k < ci[5 * c + 3] + ci[5 * c + 4]; k++) {
        const bool draw = drand48() > 0.5;
        if ((draw && ic > 2) || ic > 5) ic = 0;
        icell[k] = (ic == 0) ? id++ : -ic;
        ic++;
      }
    }
    if (n < nimax) write_back(n, perm, b, iwrap, icell, cycle, res_index, x, q, v);
  });
}

void FMM_Partition(int *ni, int nimax, int *res_index, double *x, double *q, double *v, double *cycle) {
  guarded("FMM_Partition", [&] {
    MdState &s = state();
    if (!ni) throw std::runtime_error("bad body count");
    const int n = *ni;
    need_bodies(n, res_index, x, q, v);
    if (!cycle) throw std::runtime_error("null cycle");
    std::vector<int> iwrap;
    const std::vector<double> b = wrapped_bodies(n, x, q, cycle, iwrap);
    // getBounds, octsection with one rank, buildTree (md_distributed.cxx:162-166)
    const std::vector<int> perm = build(s, b, n, cycle[0], true);
    std::vector<int> icell(n);
    for (int i = 0; i < n; i++) icell[i] = res_index[perm[i]];
    if (n < nimax) write_back(n, perm, b, iwrap, icell, cycle, res_index, x, q, v);
  });
}

void FMM_FMM(int ni, int *nj, int *res_index, double *x, double *q, double *p, double *f, double *cycle) {
  guarded("FMM_FMM", [&] {
    MdState &s = state();
    if (!s.have_bounds) throw std::runtime_error("FMM_Partition or Set_Index has not been called");
    need_bodies(ni, res_index, x, q, p);
    if (ni > 0 && !f) throw std::runtime_error("null body array");
    if (!nj) throw std::runtime_error("null nj");
    const double c = cubic(cycle);
    std::vector<int> iwrap;
    const std::vector<double> b = wrapped_bodies(ni, x, q, cycle, iwrap);
    // buildTree in the partition's bounds, up, traverse, down, dipole
    // correction about the origin (md_distributed.cxx:220-266)
    check(exafmm_set_params(s.ctx, kP, s.theta, kNcrit, kNspawn, s.images, c), "set_params");
    check(exafmm_set_bodies(s.ctx, b.data(), ni), "set_bodies");
    check(exafmm_build_tree(s.ctx, s.bounds), "build_tree");
    check(exafmm_upward(s.ctx), "upward");
    check(exafmm_traverse(s.ctx), "traverse");
    check(exafmm_downward(s.ctx), "downward");
    double dip[3];
    const double origin[3] = {0.0, 0.0, 0.0};
    check(exafmm_get_dipole(s.ctx, origin, dip), "get_dipole");
    check(exafmm_dipole_correction(s.ctx, dip, ni), "dipole_correction");
    std::vector<double> trg(4 * (size_t)ni);
    std::vector<int> perm(ni);
    if (ni) {
      check(exafmm_get_results(s.ctx, trg.data()), "get_results");
      check(exafmm_get_perm(s.ctx, perm.data()), "get_perm");
    }
    // Ghosts (md_distributed.cxx:274-298): every body, in tree order, at each
    // of the 26 neighbouring images that lands strictly inside the local
    // bounds widened by the cutoff.
    const double *lb = s.bounds;
    std::vector<int> gb;
    std::vector<double> gx;
    for (int ix = -1; ix <= 1; ix++)
      for (int iy = -1; iy <= 1; iy++)
        for (int iz = -1; iz <= 1; iz++) {
          if (ix == 0 && iy == 0 && iz == 0) continue;
          const int sh[3] = {ix, iy, iz};
          for (int i = 0; i < ni; i++) {
            const int j = perm[i];
            double X[3];
            bool in = true;
            for (int d = 0; d < 3; d++) {
              X[d] = b[4 * j + d] + sh[d] * cycle[d];
              in = in && (lb[d] - s.cutoff < X[d]) && (X[d] < lb[3 + d] + s.cutoff);
            }
            if (in) {
              gb.push_back(j);
              gx.insert(gx.end(), X, X + 3);
            }
          }
        }
    const int njmax = *nj;
    const long long total = (long long)ni + (long long)gb.size();
    if (total > 0x7fffffffLL) throw std::runtime_error("too many ghost bodies");
    // TRG started from p and f; the results go out in the tree's body order
    // (md_distributed.cxx:267-272), which is the caller's order after
    // FMM_Partition.
    const std::vector<double> p0(p, p + ni), f0(f, f + 3 * (size_t)ni);
    const std::vector<int> r0(res_index, res_index + ni);
    for (int i = 0; i < ni; i++) {
      const int j = perm[i];
      p[i] = p0[j] + trg[4 * j + 0];
      for (int d = 0; d < 3; d++) f[3 * i + d] = f0[3 * j + d] + trg[4 * j + 1 + d];
    }
    *nj = (int)total;
    if (*nj < njmax) {
      for (size_t k = 0; k < gb.size(); k++) {
        const size_t i = (size_t)ni + k;
        res_index[i] = r0[gb[k]];
        for (int d = 0; d < 3; d++) x[3 * i + d] = gx[3 * k + d];
        q[i] = b[4 * gb[k] + 3];
      }
    }
  });
}

void FMM_Ewald(int ni, double *x, double *q, double *p, double *f, int ksize, double alpha, double sigma,
               double cutoff, double *cycle) {
  guarded("FMM_Ewald", [&] {
    state();
    need_bodies(ni, x, q, p, f);
    const double c = cubic(cycle);
    std::vector<double> b(4 * (size_t)ni), trg(4 * (size_t)ni);
    for (int i = 0; i < ni; i++) {  // md_distributed.cxx:323-336: X wrapped, TRG from p, f
      double X[3] = {x[3 * i + 0], x[3 * i + 1], x[3 * i + 2]};
      exafmm_md::wrap3(X, cycle);
      for (int d = 0; d < 3; d++) b[4 * i + d] = X[d];
      b[4 * i + 3] = q[i];
      trg[4 * i + 0] = p[i];
      for (int d = 0; d < 3; d++) trg[4 * i + 1 + d] = f[3 * i + d];
    }
    if (exafmm_ewald(b.data(), ni, ksize, alpha, sigma, cutoff, c, trg.data()) != 0)
      throw std::runtime_error(exafmm_ewald_error());
    for (int i = 0; i < ni; i++) {  // written back by IBODY: the caller's order
      p[i] = trg[4 * i + 0];
      for (int d = 0; d < 3; d++) f[3 * i + d] = trg[4 * i + 1 + d];
    }
  });
}

void Dipole_Correction(int ni, double *x, double *q, double *p, double *f, double *cycle) {
  guarded("Dipole_Correction", [&] {
    need_bodies(ni, x, q, p, f);
    if (!cycle) throw std::runtime_error("null cycle");
    // md_distributed.cxx:383-405: the dipole summed in float, |d|^2 in double
    // of float squares, the coefficient in float
    float dipole[3] = {0, 0, 0};
    for (int i = 0; i < ni; i++)
      for (int d = 0; d < 3; d++) dipole[d] += x[3 * i + d] * q[i];
    double norm = 0;
    for (int d = 0; d < 3; d++) norm += dipole[d] * dipole[d];
    const float coef = 4 * M_PI / (3 * cycle[0] * cycle[1] * cycle[2]);
    for (int i = 0; i < ni; i++) {
      p[i] -= coef * norm / ni / q[i];
      for (int d = 0; d < 3; d++) f[3 * i + d] -= coef * dipole[d];
    }
  });
}

void FMM_Cutoff(int ni, double *x, double *q, double *p, double *f, double cutoff, double *cycle) {
  guarded("FMM_Cutoff", [&] {
    need_bodies(ni, x, q, p, f);
    if (!cycle) throw std::runtime_error("null cycle");
    // md_distributed.cxx:407-461: images out to the cutoff, every pair closer
    // than the cutoff; p += sum q/r, f -= sum dx q/r^3
    const double cmin = std::fmin(cycle[0], std::fmin(cycle[1], cycle[2]));
    const int prange = int(cutoff / cmin * 0.999999) + 1;
    std::vector<double> b(4 * (size_t)ni), trg(4 * (size_t)ni, 0.0);
    for (int i = 0; i < ni; i++) {
      for (int d = 0; d < 3; d++) b[4 * i + d] = x[3 * i + d];
      b[4 * i + 3] = q[i];
    }
    if (exafmm_direct_cutoff(b.data(), ni, b.data(), ni, prange, cycle, cutoff, trg.data()) != 0)
      throw std::runtime_error(exafmm_kernel_error());
    for (int i = 0; i < ni; i++) {
      p[i] += trg[4 * i + 0];
      for (int d = 0; d < 3; d++) f[3 * i + d] += trg[4 * i + 1 + d];
    }
  });
}

const char *FMM_Error(void) { return g_error.c_str(); }

}  // extern "C"
