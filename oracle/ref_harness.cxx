// Reference harness: the UNMODIFIED exafmm-beta Laplace headers, compiled in
// place (-I into the reference tree, nothing copied) and exposed through a small
// extern "C" surface so the tests and the CPU-baseline leg of bench.py can drive
// them with ctypes.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
// calls this file; it is the checker.  Built by oracle/Makefile into
// oracle/_ref/libexafmm_ref.so.
//
// What it runs is the examples/fmm.cxx solve sequence (examples/fmm.cxx:61-77):
//   BoundBox::getBounds -> BuildTree::buildTree -> UpDownPass::upwardPass ->
//   Traversal::traverse -> UpDownPass::downwardPass
// plus, for list parity, a thin Kernel subclass that records which (Ci, Cj)
// pairs the reference traversal hands to M2L and P2P (include/traversal.h:121,168).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>
#include <omp.h>

#include "types.h"
#include "logger.h"
// Rename the reference Kernel class so a recording subclass can take its name;
// Traversal and UpDownPass call kernel.M2L / kernel.P2P on a `Kernel &`, so the
// subclass's (hiding) methods are the ones they invoke.
#define Kernel RefKernelBase
#include "laplace.h"
#undef Kernel

namespace exafmm_laplace {
  struct PairLog {
    std::vector<int> m2l;
    std::vector<int> p2p;
  };

  class Kernel : public RefKernelBase {
  public:
    PairLog * log = nullptr;
    C_iter C0;    // first target cell
    C_iter Cj0;   // first source cell (C0 unless the sources have their own tree)
    Kernel(int P, real_t eps2, complex_t wavek) : RefKernelBase(P, eps2, wavek) {}
    // the traversal's tasks call these from several threads when threads > 1
    std::mutex log_mutex;
    void M2L(C_iter Ci, C_iter Cj) {
      if (log) {
        std::lock_guard<std::mutex> lock(log_mutex);
        log->m2l.push_back(int(Ci - C0));
        log->m2l.push_back(int(Cj - Cj0));
      }
      RefKernelBase::M2L(Ci, Cj);
    }
    void P2P(C_iter Ci, C_iter Cj) {
      if (log) {
        std::lock_guard<std::mutex> lock(log_mutex);
        log->p2p.push_back(int(Ci - C0));
        log->p2p.push_back(int(Cj - Cj0));
      }
      RefKernelBase::P2P(Ci, Cj);
    }
  };
}

#include "bound_box.h"
#include "build_tree.h"
#include "up_down_pass.h"
#include "traversal.h"
#include "ewald.h"

using namespace exafmm_laplace;

namespace {
  // Kernel tables are O(P^4); build one object per P and reuse it.
  std::mutex g_kernel_mutex;
  std::map<int, Kernel *> g_kernels;

  Kernel & kernelFor(int P) {
    std::lock_guard<std::mutex> lock(g_kernel_mutex);
    auto it = g_kernels.find(P);
    if (it != g_kernels.end()) return *it->second;
    Kernel * k = new Kernel(P, 0.0, complex_t(10., 1.) / real_t(2 * M_PI));
    g_kernels[P] = k;
    return *k;
  }

  // Dataset::initTarget semantics (include/dataset.h:220-227).
  void loadBodies(Bodies & bodies, int n, const double * xyzq) {
    bodies.resize(n);
    for (int i = 0; i < n; i++) {
      for (int d = 0; d < 3; d++) bodies[i].X[d] = xyzq[4 * i + d];
      bodies[i].SRC = xyzq[4 * i + 3];
      bodies[i].TRG = 0;
      bodies[i].IBODY = i;
      bodies[i].IRANK = 0;
      bodies[i].ICELL = 0;
      bodies[i].WEIGHT = 1;
    }
  }

  struct Run {
    int n = 0, P = 0;
    Bounds bounds;
    Bodies bodies;            // tree order after buildTree
    Cells cells;
    Bodies jbodies;           // separate sources (IneJ), tree order
    Cells jcells;
    PairLog log;
    double times[8] = {0};    // bounds, grow, link, up, traverse, down, total, dipole
  };
}

extern "C" {

// Full solve.  xyzq is n x 4 (x, y, z, q) in the caller's order.  bounds_in may be
// null, in which case BoundBox::getBounds computes them as examples/fmm.cxx:163 does.
// threads > 1 runs the reference's own OpenMP task tree (include/thread.h:31-43,
// include/traversal.h:208-225) inside one parallel region; threads == 1 is what
// examples/fmm.cxx does (its tasks run with no enclosing parallel region).
void * ref_run(int n, const double * xyzq, int P, double theta, int ncrit, int nspawn,
               int images, double cycle, int threads, int record_lists,
               const double * bounds_in, int dipole_correction) {
  Run * run = new Run;
  run->n = n;
  run->P = P;
  Kernel & kernel = kernelFor(P);
  loadBodies(run->bodies, n, xyzq);
  Bodies buffer;
  buffer.reserve(n);
  BoundBox boundBox;
  BuildTree buildTree(ncrit);
  UpDownPass upDownPass(kernel);
  Traversal traversal(kernel, theta, nspawn, images, "./");
  vec3 vcycle = cycle;
  double t0 = logger::get_time();
  if (bounds_in) {
    for (int d = 0; d < 3; d++) {
      run->bounds.Xmin[d] = bounds_in[d];
      run->bounds.Xmax[d] = bounds_in[3 + d];
    }
  } else {
    run->bounds = boundBox.getBounds(run->bodies);
  }
  double t1 = logger::get_time();
  run->cells = buildTree.buildTree(run->bodies, buffer, run->bounds);
  double t2 = logger::get_time();
  upDownPass.upwardPass(run->cells);
  traversal.initListCount(run->cells);  // examples/fmm.cxx:67
  double t3 = logger::get_time();
  kernel.C0 = run->cells.begin();
  kernel.Cj0 = run->cells.begin();
  kernel.log = record_lists ? &run->log : nullptr;
  if (threads > 1) {
    omp_set_num_threads(threads);
#pragma omp parallel
#pragma omp single
    traversal.traverse(run->cells, run->cells, vcycle, true);
  } else {
    traversal.traverse(run->cells, run->cells, vcycle, true);
  }
  kernel.log = nullptr;
  double t4 = logger::get_time();
  upDownPass.downwardPass(run->cells);
  double t5 = logger::get_time();
  double t6 = t5;
  if (images > 0 && dipole_correction) {
    // examples/ewald.cxx recipe: dipole about the origin, corrected per body.
    vec3 dipole = upDownPass.getDipole(run->bodies, 0);
    upDownPass.dipoleCorrection(run->bodies, dipole, n, vcycle);
    t6 = logger::get_time();
  }
  run->times[0] = t1 - t0;
  run->times[1] = t2 - t1;  // grow + link (buildTree)
  run->times[2] = 0;
  run->times[3] = t3 - t2;
  run->times[4] = t4 - t3;
  run->times[5] = t5 - t4;
  run->times[6] = t5 - t0;
  run->times[7] = t6 - t5;
  return run;
}

// Separate source bodies (examples/fmm.cxx -j IneJ, :61-73): bounds of the
// targets extended by the sources (BoundBox::getBounds(jbodies, bounds)), a
// tree for each on those bounds, both upward passes, traverse(cells, jcells),
// downward pass of the targets.  Free space.
void * ref_run_inej(int n, const double * xyzq, int nj, const double * jxyzq, int P, double theta, int ncrit,
                    int nspawn, int record_lists) {
  Run * run = new Run;
  run->n = n;
  run->P = P;
  Kernel & kernel = kernelFor(P);
  loadBodies(run->bodies, n, xyzq);
  loadBodies(run->jbodies, nj, jxyzq);
  Bodies buffer;
  buffer.reserve(std::max(n, nj));
  BoundBox boundBox;
  BuildTree buildTree(ncrit);
  UpDownPass upDownPass(kernel);
  Traversal traversal(kernel, theta, nspawn, 0, "./");
  vec3 vcycle = 2 * M_PI;
  run->bounds = boundBox.getBounds(run->bodies);
  run->bounds = boundBox.getBounds(run->jbodies, run->bounds);
  run->cells = buildTree.buildTree(run->bodies, buffer, run->bounds);
  upDownPass.upwardPass(run->cells);
  traversal.initListCount(run->cells);
  run->jcells = buildTree.buildTree(run->jbodies, buffer, run->bounds);
  upDownPass.upwardPass(run->jcells);
  kernel.C0 = run->cells.begin();
  kernel.Cj0 = run->jcells.begin();
  kernel.log = record_lists ? &run->log : nullptr;
  traversal.traverse(run->cells, run->jcells, vcycle, true);
  kernel.log = nullptr;
  upDownPass.downwardPass(run->cells);
  return run;
}

int ref_num_jcells(void * h) { return int(((Run *)h)->jcells.size()); }

void ref_get_jcells(void * h, int * ints, double * reals, int * jperm) {
  Run * run = (Run *)h;
  int c = 0;
  for (auto & C : run->jcells) {
    ints[5 * c + 0] = C.IPARENT;
    ints[5 * c + 1] = C.ICHILD;
    ints[5 * c + 2] = C.NCHILD;
    ints[5 * c + 3] = C.IBODY;
    ints[5 * c + 4] = C.NBODY;
    for (int d = 0; d < 3; d++) reals[4 * c + d] = C.X[d];
    reals[4 * c + 3] = C.R;
    c++;
  }
  for (size_t i = 0; i < run->jbodies.size(); i++) jperm[i] = run->jbodies[i].IBODY;
}

int ref_num_cells(void * h) { return int(((Run *)h)->cells.size()); }
int ref_num_m2l(void * h) { return int(((Run *)h)->log.m2l.size() / 2); }
int ref_num_p2p(void * h) { return int(((Run *)h)->log.p2p.size() / 2); }

void ref_get_bounds(void * h, double * out) {
  Run * run = (Run *)h;
  for (int d = 0; d < 3; d++) {
    out[d] = run->bounds.Xmin[d];
    out[3 + d] = run->bounds.Xmax[d];
  }
}

// Per-body (pot, ax, ay, az) scattered back to the caller's order by IBODY.
void ref_get_trg(void * h, double * trg) {
  Run * run = (Run *)h;
  for (auto & B : run->bodies) {
    for (int k = 0; k < 4; k++) trg[4 * B.IBODY + k] = B.TRG[k];
  }
}

// Tree-order permutation: perm[i] = original index of the body at tree slot i.
void ref_get_perm(void * h, int * perm) {
  Run * run = (Run *)h;
  for (int i = 0; i < run->n; i++) perm[i] = run->bodies[i].IBODY;
}

// ints: C x 5 (IPARENT, ICHILD, NCHILD, IBODY, NBODY); reals: C x 4 (X, Y, Z, R).
void ref_get_cells(void * h, int * ints, double * reals, unsigned long long * icell) {
  Run * run = (Run *)h;
  int c = 0;
  for (auto & C : run->cells) {
    ints[5 * c + 0] = C.IPARENT;
    ints[5 * c + 1] = C.ICHILD;
    ints[5 * c + 2] = C.NCHILD;
    ints[5 * c + 3] = C.IBODY;
    ints[5 * c + 4] = C.NBODY;
    for (int d = 0; d < 3; d++) reals[4 * c + d] = C.X[d];
    reals[4 * c + 3] = C.R;
    if (icell) icell[c] = C.ICELL;
    c++;
  }
}

void ref_get_lists(void * h, int * m2l, int * p2p) {
  Run * run = (Run *)h;
  if (m2l) std::copy(run->log.m2l.begin(), run->log.m2l.end(), m2l);
  if (p2p) std::copy(run->log.p2p.begin(), run->log.p2p.end(), p2p);
}

// Expansions as interleaved (re, im), C x NTERM x 2.
void ref_get_expansions(void * h, double * M, double * L) {
  Run * run = (Run *)h;
  int nterm = run->P * (run->P + 1) / 2;
  int c = 0;
  for (auto & C : run->cells) {
    for (int k = 0; k < nterm; k++) {
      if (M) { M[2 * (c * nterm + k)] = C.M[k].real(); M[2 * (c * nterm + k) + 1] = C.M[k].imag(); }
      if (L) { L[2 * (c * nterm + k)] = C.L[k].real(); L[2 * (c * nterm + k) + 1] = C.L[k].imag(); }
    }
    c++;
  }
}

// Traversal::writeList (include/traversal.h:412-421) of the run's cells into
// path + "list%06d.dat" (rank 0), as examples/fmm.cxx:88 calls it.
void ref_write_list(void * h, const char * path) {
  Run * run = (Run *)h;
  Traversal traversal(kernelFor(run->P), 0.4, 0, 0, path);
  traversal.writeList(run->cells, 0);
}

// logger::writeTime (include/logger.h:116-127) of the given events into
// path + "time%06d.dat" (rank 0).
void ref_write_time(int count, const char * const * names, const double * seconds, const char * path) {
  logger::timer.clear();
  for (int i = 0; i < count; i++) logger::timer[names[i]] = seconds[i];
  const char * saved = logger::path;
  logger::path = path;
  logger::writeTime(0);
  logger::path = saved;
}

void ref_get_times(void * h, double * t) {
  std::memcpy(t, ((Run *)h)->times, sizeof(((Run *)h)->times));
}

void ref_free(void * h) { delete (Run *)h; }

// ---- Per-operator wrappers (the examples/kernel.cxx known-answer chain) ----
// Expansions are interleaved (re, im) arrays of NTERM = P(P+1)/2 entries.

static void toComplex(const double * in, std::vector<complex_t> & out, int nterm) {
  out.assign(nterm, 0.0);
  if (in) for (int k = 0; k < nterm; k++) out[k] = complex_t(in[2 * k], in[2 * k + 1]);
}
static void fromComplex(const std::vector<complex_t> & in, double * out) {
  for (size_t k = 0; k < in.size(); k++) { out[2 * k] = in[k].real(); out[2 * k + 1] = in[k].imag(); }
}

void ref_p2m(int P, const double * X, double R, int n, const double * xyzq, double * M) {
  Kernel & kernel = kernelFor(P);
  Bodies bodies; loadBodies(bodies, n, xyzq);
  Cells cells(1);
  C_iter C = cells.begin();
  for (int d = 0; d < 3; d++) C->X[d] = X[d];
  C->R = R; C->BODY = bodies.begin(); C->NBODY = n;
  toComplex(M, C->M, kernel.NTERM);
  kernel.P2M(C);
  fromComplex(C->M, M);
}

// Parent at Xp accumulates children (nchild, centers Xc[nchild][3], M[nchild][NTERM][2]).
void ref_m2m(int P, const double * Xp, int nchild, const double * Xc, const double * Mc, double * Mp) {
  Kernel & kernel = kernelFor(P);
  Cells cells(nchild + 1);
  for (int c = 0; c < nchild; c++) {
    for (int d = 0; d < 3; d++) cells[c].X[d] = Xc[3 * c + d];
    toComplex(Mc + 2 * c * kernel.NTERM, cells[c].M, kernel.NTERM);
  }
  C_iter Ci = cells.begin() + nchild;
  for (int d = 0; d < 3; d++) Ci->X[d] = Xp[d];
  Ci->ICHILD = 0; Ci->NCHILD = nchild;
  toComplex(Mp, Ci->M, kernel.NTERM);
  kernel.M2M(Ci, cells.begin());
  fromComplex(Ci->M, Mp);
}

void ref_m2l(int P, const double * Xi, const double * Xj, const double * Mj, double * Li,
             const double * Xperiodic) {
  Kernel & kernel = kernelFor(P);
  Cells cells(2);
  C_iter Ci = cells.begin(), Cj = cells.begin() + 1;
  for (int d = 0; d < 3; d++) { Ci->X[d] = Xi[d]; Cj->X[d] = Xj[d]; }
  toComplex(Mj, Cj->M, kernel.NTERM);
  toComplex(Li, Ci->L, kernel.NTERM);
  vec3 saved = kernel.Xperiodic;
  for (int d = 0; d < 3; d++) kernel.Xperiodic[d] = Xperiodic ? Xperiodic[d] : 0.0;
  kernel.RefKernelBase::M2L(Ci, Cj);
  kernel.Xperiodic = saved;
  fromComplex(Ci->L, Li);
}

void ref_l2l(int P, const double * Xc, const double * Xp, const double * Lp, double * Lc) {
  Kernel & kernel = kernelFor(P);
  Cells cells(2);
  C_iter Cp = cells.begin(), Cc = cells.begin() + 1;
  for (int d = 0; d < 3; d++) { Cp->X[d] = Xp[d]; Cc->X[d] = Xc[d]; }
  toComplex(Lp, Cp->L, kernel.NTERM);
  toComplex(Lc, Cc->L, kernel.NTERM);
  Cc->IPARENT = 0;
  kernel.L2L(Cc, cells.begin());
  fromComplex(Cc->L, Lc);
}

// trg (n x 4) accumulates.
void ref_l2p(int P, const double * X, const double * L, int n, const double * xyzq, double * trg) {
  Kernel & kernel = kernelFor(P);
  Bodies bodies; loadBodies(bodies, n, xyzq);
  for (int i = 0; i < n; i++) for (int k = 0; k < 4; k++) bodies[i].TRG[k] = trg[4 * i + k];
  Cells cells(1);
  C_iter C = cells.begin();
  for (int d = 0; d < 3; d++) C->X[d] = X[d];
  C->BODY = bodies.begin(); C->NBODY = n;
  toComplex(L, C->L, kernel.NTERM);
  kernel.L2P(C);
  for (int i = 0; i < n; i++) for (int k = 0; k < 4; k++) trg[4 * i + k] = bodies[i].TRG[k];
}

// trg_i (ni x 4) accumulates.
void ref_p2p(int ni, const double * xi, int nj, const double * xj, const double * Xperiodic, double * trg_i) {
  Kernel & kernel = kernelFor(4);
  Bodies bi, bj; loadBodies(bi, ni, xi); loadBodies(bj, nj, xj);
  for (int i = 0; i < ni; i++) for (int k = 0; k < 4; k++) bi[i].TRG[k] = trg_i[4 * i + k];
  Cells cells(2);
  C_iter Ci = cells.begin(), Cj = cells.begin() + 1;
  Ci->BODY = bi.begin(); Ci->NBODY = ni; Cj->BODY = bj.begin(); Cj->NBODY = nj;
  vec3 saved = kernel.Xperiodic;
  for (int d = 0; d < 3; d++) kernel.Xperiodic[d] = Xperiodic ? Xperiodic[d] : 0.0;
  kernel.RefKernelBase::P2P(Ci, Cj);
  kernel.Xperiodic = saved;
  for (int i = 0; i < ni; i++) for (int k = 0; k < 4; k++) trg_i[4 * i + k] = bi[i].TRG[k];
}

// Ewald summation (include/ewald.h) driven as examples/ewald.cxx:122-136 does for one
// rank: a tree of the bodies, wavePart(bodies, bodies), realPart(cells, cells),
// selfTerm(bodies).  Results (potential, gradient) overwrite trg in caller order.
void ref_ewald(int n, const double * xyzq, int ksize, double alpha, double sigma, double cutoff,
               double cycle, int ncrit, double * trg) {
  Bodies bodies, buffer;
  loadBodies(bodies, n, xyzq);
  buffer.reserve(n);
  BoundBox boundBox;
  BuildTree buildTree(ncrit);
  Bounds bounds = boundBox.getBounds(bodies);
  Cells cells = buildTree.buildTree(bodies, buffer, bounds);
  Ewald ewald(ksize, alpha, sigma, cutoff, vec3(cycle));
  ewald.wavePart(bodies, bodies);
  ewald.realPart(cells, cells);
  ewald.selfTerm(bodies);
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 4; k++) trg[4 * bodies[i].IBODY + k] = bodies[i].TRG[k];
}

// Traversal::direct (include/traversal.h:355-377): targets accumulate over all sources
// and over the periodic image range implied by images and theta.
void ref_direct(int ni, const double * xi, int nj, const double * xj, int images, double theta,
                double cycle, double * trg_i) {
  Kernel & kernel = kernelFor(4);
  Bodies bi, bj; loadBodies(bi, ni, xi); loadBodies(bj, nj, xj);
  for (int i = 0; i < ni; i++) for (int k = 0; k < 4; k++) bi[i].TRG[k] = trg_i[4 * i + k];
  Traversal traversal(kernel, theta, 5000, images, "./");
  vec3 saved = kernel.Xperiodic;
  traversal.direct(bi, bj, vec3(cycle));
  kernel.Xperiodic = saved;
  for (int i = 0; i < ni; i++) for (int k = 0; k < 4; k++) trg_i[4 * i + k] = bi[i].TRG[k];
}

}  // extern "C"
