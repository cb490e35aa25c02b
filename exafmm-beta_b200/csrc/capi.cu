// extern "C" surface of the engine (include/exafmm_b200.h) and the solve driver.
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <vector>

#include "../../include/exafmm_b200.h"
#include "drift.cuh"
#include "fmm.h"
#include "harmonics.cuh"
#include "records.h"

namespace exafmm_b200 {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void throw_cuda(cudaError_t e, const char *what, const char *file, int line) {
  std::string m = std::string(cudaGetErrorString(e)) + " in " + what + " (" + file + ":" + std::to_string(line) + ")";
  throw CudaError(m);
}
void throw_msg(const char *msg) { throw std::runtime_error(msg); }

static std::atomic<long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

void direct_fp64(const double4 *tgt, long long nt, const double4 *src, long long ns, int prange, double cycle,
                 double4 *trg, cudaStream_t st);

namespace {

// Phase events of the last solve: ev[0..7] bound bounds, tree, upward, lists,
// m2l, p2p, downward; link splits the tree build (growTree / linkTree), lat
// brackets the periodic lattice.  Each phase, once complete, is flagged in
// `done`; fold() adds the flagged phases' times under the reference's logger
// event names to `timer` (before their events are recorded again), which
// exafmm_write_time writes out and exafmm_take_timers hands to the caller.
struct Timing {
  enum : unsigned { kBounds = 1, kGrow = 2, kLink = 4, kUp = 8, kTrav = 16, kPer = 32, kDown = 64 };
  cudaEvent_t ev[8] = {};
  cudaEvent_t link = nullptr, lat[2] = {};
  bool live = false;
  unsigned done = 0;       // phases complete whose times are not in `timer` yet
  std::map<std::string, double> timer;
  void init() {
    if (live) return;
    for (auto &e : ev) EXA_CUDA(cudaEventCreate(&e));
    EXA_CUDA(cudaEventCreate(&link));
    for (auto &e : lat) EXA_CUDA(cudaEventCreate(&e));
    live = true;
  }
  double seconds(cudaEvent_t a, cudaEvent_t b) {
    EXA_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    EXA_CUDA(cudaEventElapsedTime(&ms, a, b));
    return 1e-3 * ms;
  }
  // Event names of include/bound_box.h:12, build_tree.h:187-207, up_down_pass.h:50-74,
  // traversal.h:234-350 ("Traverse" includes "Traverse periodic", as there).
  void fold() {
    if (!done) return;
    if (done & kBounds) timer["Get bounds"] += seconds(ev[0], ev[1]);
    if (done & kGrow) timer["Grow tree"] += seconds(ev[1], link);
    if (done & kLink) timer["Link tree"] += seconds(link, ev[2]);
    if (done & kUp) timer["Upward pass"] += seconds(ev[2], ev[3]);
    if (done & kTrav) timer["Traverse"] += seconds(ev[3], ev[6]);
    if (done & kPer) timer["Traverse periodic"] += seconds(lat[0], lat[1]);
    if (done & kDown) timer["Downward pass"] += seconds(ev[6], ev[7]);
    done = 0;
  }
  // Before a phase records its events again, the last run of it is folded.
  void reuse(unsigned phases) {
    if (done & phases) fold();
  }
  ~Timing() {
    if (live) {
      for (auto &e : ev) cudaEventDestroy(e);
      cudaEventDestroy(link);
      for (auto &e : lat) cudaEventDestroy(e);
    }
  }
};

}  // namespace

struct Engine {
  Context C;
  ListBufs lists;
  DBuf<double2> M, L;
  DBuf<unsigned char> Ms;  // scaled multipoles for the unrolled M2L (FP32 or FP64)
  DBuf<unsigned char> Ms64;  // FP64 scaled multipoles for the FP64 part of the mixed form
  DBuf<float4> x32;        // bodies as two-float pairs relative to the root center (mixed P2P)
  DBuf<float4> x32j;       // the same for separate source bodies
  M2LGemmBufs gemm;         // class-grouped tile M2L (mixed form)
  DBuf<double2> lat;        // periodic lattice: supercell multipoles and warp partials
  DBuf<double> dip;         // dipole reduction scratch and result
  P2PWork p2pw;               // work counters and order of the mixed P2P kernels
  DBuf<double4> trg, out;
  Timing tm;
  bool tree_ok = false, up_ok = false, lists_ok = false;
  // Separate source bodies (examples/fmm.cxx -j IneJ, :61-73): their own tree
  // and multipoles, on the same stream as the targets.
  std::unique_ptr<Engine> jsrc;
  bool is_source = false;  // this engine is another one's source tree

  ~Engine() {
    if (C.pin) pinned_block_release(C.pin);  // its copies ended with the call that made them
  }

  FmmArgs args() {
    FmmArgs a;
    a.P = C.prm.P;
    a.ncrit = C.prm.ncrit;
    a.ncells = C.tree.ncells;
    a.n = C.tree.n;
    a.cycle = C.prm.cycle;
    a.stream = C.stream;
    a.lvl = C.tree.lvl.p;
    a.nd_cell = C.tree.nd_cell.p;
    a.cell_b = C.tree.cell_b.p;
    a.cell_pl = C.tree.cell_pl.p;
    a.cell_x = C.tree.cell_x.p;
    a.xt = C.tree.xyzq_tree.p;
    a.m2l_off = lists.m2l_off.p;
    a.m2l_src = lists.m2l_src.p;
    a.p2p_off = lists.p2p_off.p;
    a.p2p_src = lists.p2p_src.p;
    a.M64 = M.p;
    a.L64 = L.p;
    a.trg64 = trg.p;
    if (C.tree.nsys) {
      a.nsys = C.tree.nsys;
      a.sys_off = C.tree.sys_off.p;
      a.sys_box = C.tree.sys_box.p;
    }
    return a;
  }

  void check_err(const char *phase) {
    EXA_CUDA(cudaMemcpyAsync(C.err_host, C.err.p, sizeof(int), cudaMemcpyDeviceToHost, C.stream));
    EXA_CUDA(cudaStreamSynchronize(C.stream));
    int e = *C.err_host;
    if (e) {
      EXA_CUDA(cudaMemsetAsync(C.err.p, 0, sizeof(int), C.stream));
      std::string m = std::string(phase) + ": device error flags " + std::to_string(e);
      if (e & kErrTreeTooDeep) m += " (tree deeper than 21 levels: more than ncrit coincident bodies?)";
      throw std::runtime_error(m);
    }
  }

  void set_bodies(const double *xyzq, long long n, cudaMemcpyKind kind) {
    if (n < 0) throw std::runtime_error("negative body count");
    if (n >= (1LL << 26)) throw std::runtime_error("more than 2^26 bodies per context is not supported");
    C.tree.nsys = 0;  // one system
    C.tree.nroots = 0;
    C.tree.n = n;
    C.tree.xyzq.ensure(n);
    if (n) EXA_CUDA(cudaMemcpyAsync(C.tree.xyzq.p, xyzq, n * sizeof(double4), kind, C.stream));
    tree_ok = up_ok = lists_ok = false;
  }

  // A forest of count independent systems, bodies concatenated in system
  // order (system s: n[s] bodies).  Every system gets its own bounds, tree,
  // lists and expansions, as a solo solve of it would; they run together.
  // parts (optional): one pointer per system instead of the concatenation,
  // host or device memory (copied with cudaMemcpyDefault, one copy each).
  void set_systems(int count, const long long *n, const double *xyzq, cudaMemcpyKind kind,
                   const double *const *parts = nullptr) {
    if (count < 1) throw std::runtime_error("a forest needs at least one system");
    if (!n) throw std::runtime_error("null system sizes");
    if (jsrc) throw std::runtime_error("a forest of systems cannot have separate sources");
    if (C.prm.images != 0) throw std::runtime_error("a forest of systems is solved in free space (images = 0)");
    TreeBufs &T = C.tree;
    std::vector<long long> off(count + 1, 0);
    std::vector<int> sys_root(count, -1), root_sys;
    std::vector<int> tile_sys;
    std::vector<long long> tile_beg;
    for (int s = 0; s < count; s++) {
      if (n[s] < 0) throw std::runtime_error("negative body count");
      off[s + 1] = off[s] + n[s];
      if (off[s + 1] >= (1LL << 26)) throw std::runtime_error("more than 2^26 bodies per context is not supported");
      if (n[s] > 0) {
        sys_root[s] = (int)root_sys.size();
        root_sys.push_back(s);
        for (long long b = off[s]; b < off[s + 1]; b += kForestTile) {
          tile_sys.push_back(s);
          tile_beg.push_back(b);
        }
      }
    }
    const long long total = off[count];
    if (T.nsys == count && T.sys_off_host == off) {  // same layout as before: only the bodies change
      T.n = total;
      copy_systems(xyzq, kind, parts);
      tree_ok = up_ok = lists_ok = false;
      return;
    }
    T.nsys = count;
    T.nroots = (int)root_sys.size();
    T.ntiles = (long long)tile_sys.size();
    T.sys_off_host = off;
    T.sys_off.ensure(count + 1);
    T.sys_root.ensure(count);
    T.root_sys.ensure(std::max<size_t>(1, root_sys.size()));
    T.tile_sys.ensure(std::max<size_t>(1, tile_sys.size()));
    T.tile_beg.ensure(std::max<size_t>(1, tile_beg.size()));
    // on the context's stream (its buffers are stream-ordered allocations);
    // pageable host vectors, so the stream is synchronized before they go
    cudaStream_t st = C.stream;
    EXA_CUDA(cudaMemcpyAsync(T.sys_off.p, off.data(), (count + 1) * sizeof(long long), cudaMemcpyHostToDevice, st));
    EXA_CUDA(cudaMemcpyAsync(T.sys_root.p, sys_root.data(), count * sizeof(int), cudaMemcpyHostToDevice, st));
    if (!root_sys.empty())
      EXA_CUDA(cudaMemcpyAsync(T.root_sys.p, root_sys.data(), root_sys.size() * sizeof(int), cudaMemcpyHostToDevice,
                               st));
    if (!tile_sys.empty()) {
      EXA_CUDA(cudaMemcpyAsync(T.tile_sys.p, tile_sys.data(), tile_sys.size() * sizeof(int), cudaMemcpyHostToDevice,
                               st));
      EXA_CUDA(cudaMemcpyAsync(T.tile_beg.p, tile_beg.data(), tile_beg.size() * sizeof(long long),
                               cudaMemcpyHostToDevice, st));
    }
    EXA_CUDA(cudaStreamSynchronize(st));
    T.n = total;
    T.xyzq.ensure(total);
    copy_systems(xyzq, kind, parts);
    tree_ok = up_ok = lists_ok = false;
  }

  void copy_systems(const double *xyzq, cudaMemcpyKind kind, const double *const *parts) {
    TreeBufs &T = C.tree;
    if (!parts) {
      if (T.n) EXA_CUDA(cudaMemcpyAsync(T.xyzq.p, xyzq, T.n * sizeof(double4), kind, C.stream));
      return;
    }
    for (int s = 0; s < T.nsys; s++) {
      const long long k = T.sys_off_host[s + 1] - T.sys_off_host[s];
      if (!k) continue;
      if (!parts[s]) throw std::runtime_error("null bodies of system " + std::to_string(s));
      EXA_CUDA(cudaMemcpyAsync(T.xyzq.p + T.sys_off_host[s], parts[s], k * sizeof(double4), cudaMemcpyDefault,
                               C.stream));
    }
  }

  void set_sources(const double *xyzq, long long n) {
    if (xyzq && C.tree.nsys) throw std::runtime_error("a forest of systems cannot have separate sources");
    if (!xyzq) {  // back to sources == targets
      jsrc.reset();
    } else {
      if (n <= 0) throw std::runtime_error("separate sources need at least one body");
      if (!jsrc) {
        std::unique_ptr<Engine> e(new Engine);
        e->is_source = true;
        e->C.device = C.device;
        e->C.stream = C.stream;
        e->C.err.ensure(1);
        EXA_CUDA(cudaMemsetAsync(e->C.err.p, 0, sizeof(int), C.stream));
        e->C.pin = pinned_block_acquire();
        e->C.err_host = reinterpret_cast<int *>(e->C.pin);
        jsrc = std::move(e);
      }
      jsrc->C.prm = C.prm;
      jsrc->set_bodies(xyzq, n, cudaMemcpyHostToDevice);
    }
    tree_ok = up_ok = lists_ok = false;
  }

  // The source tree on the targets' bounds (examples/fmm.cxx:69).
  void build_sources(const double *d_bounds6, const Params &prm) {
    tm.init();
    C.prm = prm;
    C.tree.bounds.ensure(6);
    EXA_CUDA(cudaMemcpyAsync(C.tree.bounds.p, d_bounds6, 6 * sizeof(double), cudaMemcpyDeviceToDevice, C.stream));
    grow_tree();
    tree_ok = true;
    up_ok = lists_ok = false;
  }

  void build(const double *bounds6) {
    tm.fold();  // the previous solve's times, before its events are reused
    tm.init();
    C.ev_link = tm.link;
    EXA_CUDA(cudaEventRecord(tm.ev[0], C.stream));
    if (C.tree.nsys && bounds6) throw std::runtime_error("a forest computes each system's own bounds");
    if (bounds6) {
      set_bounds(C, bounds6);
    } else {
      compute_bounds(C);
      if (jsrc) extend_bounds(C, jsrc->C.tree.xyzq.p, jsrc->C.tree.n);  // examples/fmm.cxx:62-64
    }
    EXA_CUDA(cudaEventRecord(tm.ev[1], C.stream));
    grow_tree();
    if (jsrc) jsrc->build_sources(C.tree.bounds.p, C.prm);
    EXA_CUDA(cudaEventRecord(tm.ev[2], C.stream));
    tm.done |= Timing::kBounds | Timing::kGrow | Timing::kLink;
    tree_ok = true;
    up_ok = lists_ok = false;
  }

  void grow_tree() {
    for (int attempt = 0;; attempt++) {
      build_tree(C);
      sync_tree(C);
      int e = *C.err_host;
      if ((e & kErrCellOverflow) && attempt < 8) {
        EXA_CUDA(cudaMemsetAsync(C.err.p, 0, sizeof(int), C.stream));
        build_tree_grow(2 * C.tree.node_cap);
        continue;
      }
      break;
    }
    check_err("build_tree");
  }

  void build_tree_grow(long long cap) {
    TreeBufs &T = C.tree;
    T.nd_begin.ensure(cap);
    T.nd_count.ensure(cap);
    T.nd_nchild.ensure(cap);
    T.nd_childbeg.ensure(cap);
    T.nd_nnode.ensure(cap);
    T.nd_cell.ensure(cap);
    T.nd_pcell.ensure(cap);
    T.nd_ichild.ensure(cap);
    T.nd_x.ensure(cap);
    T.cell_b.ensure(cap);
    T.cell_pl.ensure(cap);
    T.cell_x.ensure(cap);
    T.cell_node.ensure(cap);
    T.node_cap = cap;
    T.cell_cap = cap;
  }

  void upward() {
    if (!tree_ok) throw std::runtime_error("upward pass before build_tree");
    const long long nc = C.tree.ncells;
    const int NT = tri(C.prm.P);
    M.ensure(nc * NT);
    L.ensure(nc * NT);
    if (nc > 0) {
      FmmArgs a = args();
      p2m_fp64(a);
      for (int l = C.tree.depth - 1; l >= 0; l--) m2m_fp64(a, l, C.tree.lvl_host[l]);
    }
    if (jsrc) jsrc->upward();  // examples/fmm.cxx:70
    tm.reuse(Timing::kUp | Timing::kTrav);
    EXA_CUDA(cudaEventRecord(tm.ev[3], C.stream));
    tm.done |= Timing::kUp;
    up_ok = true;
  }

  // Traversal::traverse(cells, jcells) and the operators across the two trees:
  // FP64, or in the mixed form the FP32 pair-by-pair M2L for the pairs of the
  // mixed policy (the source tree's scaled multipoles), FP64 for the rest, and
  // the FP32 P2P over the source tree's bodies (two-float offsets from the
  // common root center: both trees are built on the same bounds).
  void traverse_separate_sources() {
    if (C.prm.images != 0) throw std::runtime_error("separate sources: free space only (images = 0)");
    const long long nc = C.tree.ncells;
    const int NT = tri(C.prm.P);
    for (int attempt = 0; !traverse(C, lists, &jsrc->C.tree); attempt++)
      if (attempt > 8) throw std::runtime_error("traversal capacity growth did not converge");
    check_err("traverse");
    EXA_CUDA(cudaEventRecord(tm.ev[4], C.stream));
    EXA_CUDA(cudaMemsetAsync(L.p, 0, nc * NT * sizeof(double2), C.stream));
    FmmArgs a = args();
    a.src_cell_b = jsrc->C.tree.cell_b.p;
    a.src_cell_pl = jsrc->C.tree.cell_pl.p;
    a.src_cell_x = jsrc->C.tree.cell_x.p;
    a.src_xt = jsrc->C.tree.xyzq_tree.p;
    a.src_M64 = jsrc->M.p;
    const bool mixed = C.prm.precision == kMixed;
    if (mixed && C.prm.mixed_m2l && m2l_fast_supported(C.prm.P, true)) {
      const long long ncj = jsrc->C.tree.ncells;
      Ms.ensure(std::max<long long>(1, ncj) * NT * sizeof(float2));
      scale_multipoles(C.prm.P, jsrc->M.p, jsrc->C.tree.cell_x.p, ncj, true, Ms.p, C.stream);
      m2l_fast(a, true, Ms.p, C.prm.mixed_min_level, C.prm.mixed_max_dl);
      m2l_fp64(a, C.prm.mixed_min_level, C.prm.mixed_max_dl);  // the pairs outside the policy
    } else {
      m2l_fp64(a);
    }
    EXA_CUDA(cudaEventRecord(tm.lat[0], C.stream));
    EXA_CUDA(cudaEventRecord(tm.lat[1], C.stream));
    EXA_CUDA(cudaEventRecord(tm.ev[5], C.stream));
    if (mixed && C.prm.mixed_p2p) {
      const long long ns = jsrc->C.tree.n;
      x32.ensure(2 * C.tree.n);
      x32j.ensure(std::max<long long>(1, 2 * ns));
      rel_bodies32(a, x32.p);
      rel_bodies32(a, jsrc->C.tree.xyzq_tree.p, ns, x32j.p);
      p2p_mixed(C, a, x32.p, false, p2pw, x32j.p);
    } else {
      p2p_fp64(a);
    }
  }

  void traverse_and_evaluate() {
    if (!up_ok) throw std::runtime_error("traverse before the upward pass");
    const long long nc = C.tree.ncells;
    const int NT = tri(C.prm.P);
    tm.reuse(Timing::kTrav | Timing::kPer | Timing::kDown);
    trg.ensure(C.tree.n);
    if (C.tree.n) EXA_CUDA(cudaMemsetAsync(trg.p, 0, C.tree.n * sizeof(double4), C.stream));
    if (nc > 0 && jsrc) {
      traverse_separate_sources();
    } else if (nc > 0) {
      for (int attempt = 0; !traverse(C, lists); attempt++)
        if (attempt > 8) throw std::runtime_error("traversal capacity growth did not converge");
      check_err("traverse");
      EXA_CUDA(cudaEventRecord(tm.ev[4], C.stream));
      EXA_CUDA(cudaMemsetAsync(L.p, 0, nc * NT * sizeof(double2), C.stream));
      FmmArgs a = args();
      const bool mixed = C.prm.precision == kMixed;
      const bool m2l32 = mixed && C.prm.mixed_m2l && m2l_fast_supported(C.prm.P, true);
      if (m2l32) {
        FmmArgs left = a;  // the pairs the pair-by-pair FP32 kernel takes
        // periodic boxes (neutral MD systems: their potentials cancel strongly)
        // take the per-class products at any size; pair by pair, FP32 sums over
        // a lane's sources lose more there (1.5e-6 against the plain method on
        // a 36K-charge water box at P = 8, against 6.8e-7 for the products)
        gemm.force = C.prm.mixed_gemm == 2 || (C.prm.mixed_gemm == 1 && C.prm.images > 0);
        gemm.tensor_cores = C.prm.mixed_gemm_tc != 0;
        if (C.prm.mixed_gemm && m2l_gemm(C, a, gemm, lists.n_m2l, C.prm.mixed_min_level, C.prm.mixed_max_dl)) {
          left.m2l_off = gemm.left_off.p;
          left.m2l_src = gemm.left_src.p;
        }
        Ms.ensure(nc * NT * sizeof(float2));
        scale_multipoles(a, true, Ms.p);
        m2l_fast(left, true, Ms.p, C.prm.mixed_min_level, C.prm.mixed_max_dl);
        // root levels and large size ratios in FP64: few target cells with many
        // sources each, which the unrolled kernel's lanes-over-sources form spreads out
        if (m2l_fast_supported(C.prm.P, false)) {
          m2l_complement(C, a, gemm, lists.n_m2l, C.prm.mixed_min_level, C.prm.mixed_max_dl);
          FmmArgs comp = a;
          comp.m2l_off = gemm.comp_off.p;
          comp.m2l_src = gemm.comp_src.p;
          Ms64.ensure(nc * NT * sizeof(double2));
          scale_multipoles(a, false, Ms64.p);
          m2l_fast(comp, false, Ms64.p);
        } else {
          m2l_fp64(a, C.prm.mixed_min_level, C.prm.mixed_max_dl);
        }
      } else if (m2l_fast_supported(C.prm.P, false)) {
        Ms.ensure(nc * NT * sizeof(double2));
        scale_multipoles(a, false, Ms.p);
        m2l_fast(a, false, Ms.p);
      } else {
        m2l_fp64(a);
      }
      EXA_CUDA(cudaEventRecord(tm.lat[0], C.stream));
      if (C.prm.images > 1) {  // Traversal::traversePeriodic
        lat.ensure(lattice_scratch_terms(C.prm.P));
        lattice_fp64(a, C.prm.images, C.prm.theta, lat.p);
      }
      EXA_CUDA(cudaEventRecord(tm.lat[1], C.stream));
      EXA_CUDA(cudaEventRecord(tm.ev[5], C.stream));
      if (mixed && C.prm.mixed_p2p) {
        x32.ensure(2 * C.tree.n);  // hi and lo float4 per body
        rel_bodies32(a, x32.p);
        p2p_mixed(C, a, x32.p, C.prm.images > 0, p2pw);
      } else {
        p2p_fp64(a);
      }
    } else {
      EXA_CUDA(cudaEventRecord(tm.ev[4], C.stream));
      EXA_CUDA(cudaEventRecord(tm.lat[0], C.stream));
      EXA_CUDA(cudaEventRecord(tm.lat[1], C.stream));
      EXA_CUDA(cudaEventRecord(tm.ev[5], C.stream));
    }
    EXA_CUDA(cudaEventRecord(tm.ev[6], C.stream));
    tm.done |= Timing::kTrav | (C.prm.images > 0 ? Timing::kPer : 0u);
    lists_ok = true;
  }

  void downward() {
    if (!lists_ok) throw std::runtime_error("downward pass before traverse");
    const long long nc = C.tree.ncells;
    if (nc > 0) {
      FmmArgs a = args();
      for (int l = 1; l <= C.tree.depth; l++) l2l_fp64(a, l, C.tree.lvl_host[l]);
      l2p_fp64(a);
    }
    tm.reuse(Timing::kDown);
    EXA_CUDA(cudaEventRecord(tm.ev[7], C.stream));
    tm.done |= Timing::kDown;
  }

  void results(double *dst, cudaMemcpyKind kind, double *const *parts = nullptr);
  void displace(double sigma, unsigned long long seed);
  long long p2p_interactions();
  void bodies(double *dst, cudaMemcpyKind kind);

  void get_dipole(const double *X0, double *dipole3) {
    const double zero[3] = {0.0, 0.0, 0.0};
    dip.ensure(3 * 256 + 3);
    dipole_fp64(C.tree.xyzq.p, C.tree.n, X0 ? X0 : zero, dip.p, dip.p + 3 * 256, C.stream);
    EXA_CUDA(cudaMemcpyAsync(dipole3, dip.p + 3 * 256, 3 * sizeof(double), cudaMemcpyDeviceToHost, C.stream));
    EXA_CUDA(cudaStreamSynchronize(C.stream));
  }

  void dipole_correction(const double *dipole3, long long num_bodies) {
    if (!lists_ok) throw std::runtime_error("dipole correction before a solve");
    if (num_bodies <= 0) throw std::runtime_error("dipole correction needs num_bodies > 0");
    dipole_correction_fp64(C.tree.xyzq_tree.p, trg.p, C.tree.n, C.prm.cycle, dipole3, (double)num_bodies,
                           C.stream);
  }
};

namespace {
__global__ void k_unsort(const double4 *trg, const int *perm, long long n, double4 *out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[perm[i]] = trg[i];
}

// SplitMix64 (Steele, Lea and Flood 2014; Vigna's constants): a counter-based
// stream, one 64-bit word per (seed, counter).
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
// uniform in (0, 1]: the top 53 bits, plus one ulp
__device__ __forceinline__ double unit53(unsigned long long w) { return ((w >> 11) + 1) * 0x1.0p-53; }

// Body i moves by sigma times three standard normals drawn by the Box-Muller
// transform from four uniforms of the stream at counters 4i..4i+3 (the fourth
// normal is dropped), so a displacement depends only on (seed, i).
__global__ void k_displace(double4 *x, long long n, double sigma, unsigned long long seed) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long c = seed * 0x2545f4914f6cdd1dull + 4ull * (unsigned long long)i;
    const double u0 = unit53(splitmix64(c)), u1 = unit53(splitmix64(c + 1));
    const double u2 = unit53(splitmix64(c + 2)), u3 = unit53(splitmix64(c + 3));
    const double r0 = sqrt(-2.0 * log(u0)), r1 = sqrt(-2.0 * log(u2));
    double s0, c0, s1, c1;
    sincospi(2.0 * u1, &s0, &c0);
    sincospi(2.0 * u3, &s1, &c1);
    double4 b = x[i];
    b.x += sigma * r0 * c0;
    b.y += sigma * r0 * s0;
    b.z += sigma * r1 * c1;
    x[i] = b;
  }
}
}  // namespace

namespace {
// Pair interactions of the P2P lists, sum over list entries (i, j) of
// NBODY(i) * NBODY(j): each block sums its target cells and adds once.
__global__ void k_list_work(const int *off, const int *src, long long nc, const int4 *cell_b,
                            const int4 *src_cell_b, unsigned long long *out) {
  unsigned long long acc = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nc; i += (long long)gridDim.x * blockDim.x) {
    unsigned long long nj = 0;
    for (int q = off[i]; q < off[i + 1]; q++) nj += (unsigned)src_cell_b[src[q] & 0x3ffffff].y;
    acc += nj * (unsigned)cell_b[i].y;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  __shared__ unsigned long long part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[w];
    atomicAdd(out, t);
  }
}
}  // namespace

long long Engine::p2p_interactions() {
  if (!lists_ok) throw std::runtime_error("no interaction lists (solve first)");
  const long long nc = C.tree.ncells;
  dip.ensure(1);  // one word of the dipole scratch
  unsigned long long *d = (unsigned long long *)dip.p;
  EXA_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), C.stream));
  if (nc > 0) {
    const int4 *sb = jsrc ? jsrc->C.tree.cell_b.p : C.tree.cell_b.p;
    const int grid = (int)std::max<long long>(1, std::min<long long>(kNumSMs * 4, (nc + 255) / 256));
    k_list_work<<<grid, 256, 0, C.stream>>>(lists.p2p_off.p, lists.p2p_src.p, nc, C.tree.cell_b.p, sb, d);
    EXA_CHECK_LAUNCH();
  }
  unsigned long long h = 0;
  EXA_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, C.stream));
  EXA_CUDA(cudaStreamSynchronize(C.stream));
  return (long long)h;
}

void Engine::displace(double sigma, unsigned long long seed) {
  const long long n = C.tree.n;
  if (n) {
    k_displace<<<kNumSMs * 4, 256, 0, C.stream>>>(C.tree.xyzq.p, n, sigma, seed);
    EXA_CHECK_LAUNCH();
  }
  tree_ok = up_ok = lists_ok = false;
}

void Engine::bodies(double *dst, cudaMemcpyKind kind) {
  if (C.tree.n) EXA_CUDA(cudaMemcpyAsync(dst, C.tree.xyzq.p, C.tree.n * sizeof(double4), kind, C.stream));
  EXA_CUDA(cudaStreamSynchronize(C.stream));
}

// parts (a forest only): one destination per system, host or device memory.
void Engine::results(double *dst, cudaMemcpyKind kind, double *const *parts) {
  if (!lists_ok) throw std::runtime_error("results before a solve");
  const long long n = C.tree.n;
  out.ensure(n);
  if (n) {
    k_unsort<<<kNumSMs * 4, 256, 0, C.stream>>>(trg.p, C.tree.perm.p, n, out.p);
    EXA_CHECK_LAUNCH();
    if (!parts) {
      EXA_CUDA(cudaMemcpyAsync(dst, out.p, n * sizeof(double4), kind, C.stream));
    } else {
      const TreeBufs &T = C.tree;
      for (int s = 0; s < T.nsys; s++) {
        const long long k = T.sys_off_host[s + 1] - T.sys_off_host[s];
        if (!k) continue;
        if (!parts[s]) throw std::runtime_error("null results of system " + std::to_string(s));
        EXA_CUDA(cudaMemcpyAsync(parts[s], out.p + T.sys_off_host[s], k * sizeof(double4), cudaMemcpyDefault,
                                 C.stream));
      }
    }
  }
  EXA_CUDA(cudaStreamSynchronize(C.stream));
}

}  // namespace exafmm_b200

using namespace exafmm_b200;

struct exafmm_ctx {
  Engine E;
};

namespace exafmm_b200 {
thread_local long long *g_dbuf_account = nullptr;
thread_local cudaStream_t g_dbuf_stream = nullptr;

namespace {
std::mutex g_pin_mutex;
std::vector<unsigned char *> g_pin_free;  // blocks of kPinBytes in pinned slabs that live until exit
}  // namespace

unsigned char *pinned_block_acquire() {
  std::lock_guard<std::mutex> lock(g_pin_mutex);
  if (g_pin_free.empty()) {
    constexpr int kBlocks = 64;
    unsigned char *slab = nullptr;
    EXA_CUDA(cudaMallocHost((void **)&slab, kBlocks * kPinBytes));
    for (int i = kBlocks - 1; i >= 0; i--) g_pin_free.push_back(slab + (size_t)i * kPinBytes);
  }
  unsigned char *p = g_pin_free.back();
  g_pin_free.pop_back();
  return p;
}

void pinned_block_release(unsigned char *p) {
  if (!p) return;
  std::lock_guard<std::mutex> lock(g_pin_mutex);
  g_pin_free.push_back(p);
}
}

namespace {
thread_local std::string g_create_error;

// Charges the buffers a call allocates to one context's byte counter and
// orders their allocation on its stream.
struct AccountScope {
  long long *prev;
  cudaStream_t prev_st;
  AccountScope(long long *a, cudaStream_t s) : prev(g_dbuf_account), prev_st(g_dbuf_stream) {
    g_dbuf_account = a;
    g_dbuf_stream = s;
  }
  ~AccountScope() {
    g_dbuf_account = prev;
    g_dbuf_stream = prev_st;
  }
};

template <typename F>
int guarded(exafmm_ctx *ctx, F &&f) {
  if (!ctx) return 2;
  AccountScope scope(&ctx->E.C.dev_bytes, ctx->E.C.stream);
  try {
    f();
    return 0;
  } catch (const std::exception &e) {
    ctx->E.C.last_error = e.what();
    return 1;
  }
}

template <typename F>
int guarded_free(F &&f, std::string &err) {
  try {
    f();
    return 0;
  } catch (const std::exception &e) {
    err = e.what();
    return 1;
  }
}
thread_local std::string g_kernel_error;

// Cell table in the reference's layout: ints (IPARENT, ICHILD, NCHILD, IBODY, NBODY),
// reals (X, Y, Z, R).
void copy_cells(Engine &E, int *ints, double *reals) {
  {
    const long long nc = E.C.tree.ncells;
    std::vector<int4> b(nc);
    std::vector<int2> pl(nc);
    std::vector<double4> x(nc);
    if (nc) {
      EXA_CUDA(cudaMemcpy(b.data(), E.C.tree.cell_b.p, nc * sizeof(int4), cudaMemcpyDeviceToHost));
      EXA_CUDA(cudaMemcpy(pl.data(), E.C.tree.cell_pl.p, nc * sizeof(int2), cudaMemcpyDeviceToHost));
      EXA_CUDA(cudaMemcpy(x.data(), E.C.tree.cell_x.p, nc * sizeof(double4), cudaMemcpyDeviceToHost));
    }
    for (long long c = 0; c < nc; c++) {
      if (ints) {
        ints[5 * c + 0] = pl[c].x;
        ints[5 * c + 1] = b[c].z;
        ints[5 * c + 2] = b[c].w;
        ints[5 * c + 3] = b[c].x;
        ints[5 * c + 4] = b[c].y;
      }
      if (reals) {
        reals[4 * c + 0] = x[c].x;
        reals[4 * c + 1] = x[c].y;
        reals[4 * c + 2] = x[c].z;
        reals[4 * c + 3] = x[c].w;
      }
    }
  }
}

}  // namespace

extern "C" {

int exafmm_create(exafmm_ctx **out, int P, double theta, int ncrit, int nspawn, int images, double cycle,
                  int precision, int device) {
  if (!out) return 2;
  *out = nullptr;
  try {
    if (P < 2 || P > kMaxP) throw std::runtime_error("P must be in [2, 20]");
    if (ncrit < 1 || ncrit > 1024) throw std::runtime_error("ncrit must be in [1, 1024]");
    if (!(theta > 0)) throw std::runtime_error("theta must be positive");
    if (images < 0) throw std::runtime_error("images must be >= 0");
    if (precision != EXAFMM_FP64 && precision != EXAFMM_MIXED) throw std::runtime_error("unknown precision");
    int ndev = 0;
    EXA_CUDA(cudaGetDeviceCount(&ndev));
    if (ndev == 0) throw std::runtime_error("no CUDA device");
    if (device >= 0) EXA_CUDA(cudaSetDevice(device));
    std::unique_ptr<exafmm_ctx> c(new exafmm_ctx);
    Context &C = c->E.C;
    AccountScope scope(&C.dev_bytes, nullptr);  // the stream is made below
    EXA_CUDA(cudaGetDevice(&C.device));
    C.prm.P = P;
    C.prm.theta = theta;
    C.prm.ncrit = ncrit;
    C.prm.nspawn = nspawn;
    C.prm.images = images;
    C.prm.cycle = cycle;
    C.prm.precision = precision;
    EXA_CUDA(cudaStreamCreateWithFlags(&C.stream, cudaStreamNonBlocking));
    {
      // Buffers come from the device's stream-ordered pool; keep what contexts
      // free in the pool for reuse instead of handing it back to the driver at
      // every synchronization.
      cudaMemPool_t pool;
      EXA_CUDA(cudaDeviceGetDefaultMemPool(&pool, C.device));
      unsigned long long keep = ~0ull;
      EXA_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    g_dbuf_stream = C.stream;
    C.err.ensure(1);
    EXA_CUDA(cudaMemsetAsync(C.err.p, 0, sizeof(int), C.stream));
    C.pin = pinned_block_acquire();
    C.err_host = reinterpret_cast<int *>(C.pin);
    device_tables(P);
    *out = c.release();
    return 0;
  } catch (const std::exception &e) {
    g_create_error = e.what();
    return 1;
  }
}

int exafmm_destroy(exafmm_ctx *ctx) {
  if (!ctx) return 0;
  cudaSetDevice(ctx->E.C.device);
  cudaStreamSynchronize(ctx->E.C.stream);
  cudaStream_t st = ctx->E.C.stream;
  delete ctx;
  if (st) cudaStreamDestroy(st);
  return 0;
}

const char *exafmm_last_error(const exafmm_ctx *ctx) { return ctx ? ctx->E.C.last_error.c_str() : "null context"; }
const char *exafmm_create_error(void) { return g_create_error.c_str(); }

int exafmm_set_params(exafmm_ctx *ctx, int P, double theta, int ncrit, int nspawn, int images, double cycle) {
  return guarded(ctx, [&] {
    Engine &E = ctx->E;
    Params &p = E.C.prm;
    if (P < 2 || P > kMaxP) throw std::runtime_error("P must be in [2, 20]");
    if (ncrit < 1 || ncrit > 1024) throw std::runtime_error("ncrit must be in [1, 1024]");
    if (!(theta > 0)) throw std::runtime_error("theta must be positive");
    if (images < 0) throw std::runtime_error("images must be >= 0");
    cudaSetDevice(E.C.device);
    device_tables(P);
    if (ncrit != p.ncrit) E.tree_ok = false;
    if (ncrit != p.ncrit || P != p.P) E.up_ok = false;
    if (ncrit != p.ncrit || P != p.P || theta != p.theta || nspawn != p.nspawn || images != p.images ||
        cycle != p.cycle)
      E.lists_ok = false;
    p.P = P;
    p.theta = theta;
    p.ncrit = ncrit;
    p.nspawn = nspawn;
    p.images = images;
    p.cycle = cycle;
  });
}

int exafmm_set_mixed_policy(exafmm_ctx *ctx, int m2l_fp32, int p2p_fp32, int min_level, int max_dl) {
  return guarded(ctx, [&] {
    Params &p = ctx->E.C.prm;
    if (min_level < 0 || max_dl < 0) throw std::runtime_error("min_level and max_dl must be >= 0");
    if (m2l_fp32 < 0 || m2l_fp32 > 5) throw std::runtime_error("m2l_fp32 must be in 0..5");
    p.mixed_m2l = m2l_fp32 != 0;
    p.mixed_gemm = (m2l_fp32 == 1 || m2l_fp32 == 4) ? 1 : ((m2l_fp32 == 3 || m2l_fp32 == 5) ? 2 : 0);
    p.mixed_gemm_tc = m2l_fp32 <= 3;
    p.mixed_p2p = p2p_fp32 != 0;
    p.mixed_min_level = min_level;
    p.mixed_max_dl = max_dl;
    ctx->E.lists_ok = false;
  });
}

int exafmm_set_p2p_targets_per_lane(exafmm_ctx *ctx, int tpl) {
  return guarded(ctx, [&] {
    if (tpl != 0 && tpl != 2 && tpl != 3) throw std::runtime_error("targets per lane: 0 (by leaf size), 2 or 3");
    ctx->E.C.prm.p2p_tpl = tpl;
    ctx->E.lists_ok = false;
  });
}

int exafmm_set_bodies(exafmm_ctx *ctx, const double *xyzq, long long n) {
  return guarded(ctx, [&] {
    cudaSetDevice(ctx->E.C.device);
    ctx->E.set_bodies(xyzq, n, cudaMemcpyHostToDevice);
    EXA_CUDA(cudaStreamSynchronize(ctx->E.C.stream));
  });
}

int exafmm_set_bodies_device(exafmm_ctx *ctx, const double *d_xyzq, long long n) {
  return guarded(ctx, [&] {
    cudaSetDevice(ctx->E.C.device);
    ctx->E.set_bodies(d_xyzq, n, cudaMemcpyDeviceToDevice);
  });
}

int exafmm_set_systems(exafmm_ctx *ctx, int count, const long long *n, const double *xyzq) {
  return guarded(ctx, [&] {
    cudaSetDevice(ctx->E.C.device);
    ctx->E.set_systems(count, n, xyzq, cudaMemcpyHostToDevice);
    EXA_CUDA(cudaStreamSynchronize(ctx->E.C.stream));
  });
}

int exafmm_set_systems_device(exafmm_ctx *ctx, int count, const long long *n, const double *d_xyzq) {
  return guarded(ctx, [&] {
    cudaSetDevice(ctx->E.C.device);
    ctx->E.set_systems(count, n, d_xyzq, cudaMemcpyDeviceToDevice);
  });
}

int exafmm_displace_bodies(exafmm_ctx *ctx, double sigma, unsigned long long seed) {
  return guarded(ctx, [&] {
    if (!(sigma >= 0) || !std::isfinite(sigma)) throw std::runtime_error("sigma must be finite and >= 0");
    cudaSetDevice(ctx->E.C.device);
    ctx->E.displace(sigma, seed);
  });
}

int exafmm_get_bodies(exafmm_ctx *ctx, double *xyzq) {
  return guarded(ctx, [&] {
    cudaSetDevice(ctx->E.C.device);
    ctx->E.bodies(xyzq, cudaMemcpyDeviceToHost);
  });
}

int exafmm_get_bodies_device(exafmm_ctx *ctx, double *d_xyzq) {
  return guarded(ctx, [&] {
    cudaSetDevice(ctx->E.C.device);
    ctx->E.bodies(d_xyzq, cudaMemcpyDeviceToDevice);
  });
}

int exafmm_set_systems_list(exafmm_ctx *ctx, int count, const long long *n, const double *const *xyzq) {
  return guarded(ctx, [&] {
    if (!xyzq) throw std::runtime_error("null body list");
    cudaSetDevice(ctx->E.C.device);
    ctx->E.set_systems(count, n, nullptr, cudaMemcpyDefault, xyzq);
    EXA_CUDA(cudaStreamSynchronize(ctx->E.C.stream));
  });
}

int exafmm_get_results_list(exafmm_ctx *ctx, double *const *trg) {
  return guarded(ctx, [&] {
    if (!trg) throw std::runtime_error("null result list");
    if (!ctx->E.C.tree.nsys) throw std::runtime_error("the context holds one system (exafmm_set_systems was not called)");
    cudaSetDevice(ctx->E.C.device);
    ctx->E.results(nullptr, cudaMemcpyDefault, trg);
  });
}

int exafmm_get_systems(exafmm_ctx *ctx, long long *cell_base, long long *body_off, double *bounds) {
  return guarded(ctx, [&] {
    Engine &E = ctx->E;
    TreeBufs &T = E.C.tree;
    if (!T.nsys) throw std::runtime_error("the context holds one system (exafmm_set_systems was not called)");
    cudaSetDevice(E.C.device);
    if (body_off)
      for (int s = 0; s <= T.nsys; s++) body_off[s] = T.sys_off_host[s];
    if ((cell_base || bounds) && !E.tree_ok) throw std::runtime_error("no tree");
    if (cell_base)
      for (int s = 0; s <= T.nsys; s++) cell_base[s] = T.sys_cell_host[s];
    if (bounds) {
      EXA_CUDA(cudaMemcpyAsync(bounds, T.sys_bounds.p, 6 * T.nsys * sizeof(double), cudaMemcpyDeviceToHost,
                               E.C.stream));
      EXA_CUDA(cudaStreamSynchronize(E.C.stream));
    }
  });
}

int exafmm_get_bounds(exafmm_ctx *ctx, double *b6) {
  return guarded(ctx, [&] {
    if (ctx->E.C.tree.nsys) throw std::runtime_error("a forest has bounds per system (exafmm_get_systems)");
    cudaSetDevice(ctx->E.C.device);
    compute_bounds(ctx->E.C);
    if (ctx->E.jsrc) extend_bounds(ctx->E.C, ctx->E.jsrc->C.tree.xyzq.p, ctx->E.jsrc->C.tree.n);
    EXA_CUDA(cudaMemcpyAsync(b6, ctx->E.C.tree.bounds.p, 6 * sizeof(double), cudaMemcpyDeviceToHost,
                             ctx->E.C.stream));
    EXA_CUDA(cudaStreamSynchronize(ctx->E.C.stream));
  });
}

int exafmm_build_tree(exafmm_ctx *ctx, const double *bounds6) {
  return guarded(ctx, [&] {
    cudaSetDevice(ctx->E.C.device);
    ctx->E.build(bounds6);
  });
}

int exafmm_upward(exafmm_ctx *ctx) {
  return guarded(ctx, [&] {
    cudaSetDevice(ctx->E.C.device);
    ctx->E.upward();
  });
}

int exafmm_traverse(exafmm_ctx *ctx) {
  return guarded(ctx, [&] {
    cudaSetDevice(ctx->E.C.device);
    ctx->E.traverse_and_evaluate();
  });
}

int exafmm_downward(exafmm_ctx *ctx) {
  return guarded(ctx, [&] {
    cudaSetDevice(ctx->E.C.device);
    ctx->E.downward();
    ctx->E.check_err("downward");
  });
}

int exafmm_solve(exafmm_ctx *ctx) {
  return guarded(ctx, [&] {
    cudaSetDevice(ctx->E.C.device);
    ctx->E.build(nullptr);
    ctx->E.upward();
    ctx->E.traverse_and_evaluate();
    ctx->E.downward();
  });
}

int exafmm_get_results(exafmm_ctx *ctx, double *trg) {
  return guarded(ctx, [&] {
    cudaSetDevice(ctx->E.C.device);
    ctx->E.results(trg, cudaMemcpyDeviceToHost);
  });
}

int exafmm_get_results_device(exafmm_ctx *ctx, double *d_trg) {
  return guarded(ctx, [&] {
    cudaSetDevice(ctx->E.C.device);
    ctx->E.results(d_trg, cudaMemcpyDeviceToDevice);
  });
}

int exafmm_tree_info(exafmm_ctx *ctx, long long *ncells, int *depth, long long *n_m2l, long long *n_p2p) {
  return guarded(ctx, [&] {
    if (ncells) *ncells = ctx->E.C.tree.ncells;
    if (depth) *depth = ctx->E.C.tree.depth;
    if (n_m2l) *n_m2l = ctx->E.lists_ok ? ctx->E.lists.n_m2l : -1;
    if (n_p2p) *n_p2p = ctx->E.lists_ok ? ctx->E.lists.n_p2p : -1;
  });
}

int exafmm_list_work(exafmm_ctx *ctx, long long *p2p_interactions) {
  return guarded(ctx, [&] {
    if (!p2p_interactions) throw std::runtime_error("null output");
    cudaSetDevice(ctx->E.C.device);
    *p2p_interactions = ctx->E.p2p_interactions();
  });
}

int exafmm_get_cells(exafmm_ctx *ctx, int *ints, double *reals) {
  return guarded(ctx, [&] {
    if (!ctx->E.tree_ok) throw std::runtime_error("no tree");
    cudaSetDevice(ctx->E.C.device);
    copy_cells(ctx->E, ints, reals);
  });
}

int exafmm_set_sources(exafmm_ctx *ctx, const double *xyzq, long long n) {
  return guarded(ctx, [&] {
    cudaSetDevice(ctx->E.C.device);
    ctx->E.set_sources(xyzq, n);
  });
}

int exafmm_get_source_cells(exafmm_ctx *ctx, long long *ncells, int *ints, double *reals, int *perm) {
  return guarded(ctx, [&] {
    Engine &E = ctx->E;
    if (!E.jsrc) throw std::runtime_error("no separate sources");
    if (!E.tree_ok || !E.jsrc->tree_ok) throw std::runtime_error("no tree");
    cudaSetDevice(E.C.device);
    if (ncells) *ncells = E.jsrc->C.tree.ncells;
    copy_cells(*E.jsrc, ints, reals);
    if (perm && E.jsrc->C.tree.n)
      EXA_CUDA(cudaMemcpy(perm, E.jsrc->C.tree.perm.p, E.jsrc->C.tree.n * sizeof(int), cudaMemcpyDeviceToHost));
  });
}

int exafmm_get_perm(exafmm_ctx *ctx, int *perm) {
  return guarded(ctx, [&] {
    Engine &E = ctx->E;
    if (!E.tree_ok) throw std::runtime_error("no tree");
    cudaSetDevice(E.C.device);
    if (E.C.tree.n)
      EXA_CUDA(cudaMemcpy(perm, E.C.tree.perm.p, E.C.tree.n * sizeof(int), cudaMemcpyDeviceToHost));
  });
}

int exafmm_get_lists(exafmm_ctx *ctx, int *m2l, int *p2p) {
  return guarded(ctx, [&] {
    Engine &E = ctx->E;
    if (!E.lists_ok) throw std::runtime_error("no lists");
    cudaSetDevice(E.C.device);
    const long long nc = E.C.tree.ncells;
    auto dump = [&](const DBuf<int> &off, const DBuf<int> &src, long long n, int *outp) {
      if (!outp || n == 0) return;
      std::vector<int> o(nc + 1), s(n);
      EXA_CUDA(cudaMemcpy(o.data(), off.p, (nc + 1) * sizeof(int), cudaMemcpyDeviceToHost));
      EXA_CUDA(cudaMemcpy(s.data(), src.p, n * sizeof(int), cudaMemcpyDeviceToHost));
      for (long long c = 0; c < nc; c++)
        for (int q = o[c]; q < o[c + 1]; q++) {
          outp[3 * q + 0] = (int)c;
          outp[3 * q + 1] = s[q] & ((1 << 26) - 1);
          outp[3 * q + 2] = s[q] >> 26;
        }
    };
    dump(E.lists.m2l_off, E.lists.m2l_src, E.lists.n_m2l, m2l);
    dump(E.lists.p2p_off, E.lists.p2p_src, E.lists.n_p2p, p2p);
  });
}

int exafmm_get_expansions(exafmm_ctx *ctx, double *Mh, double *Lh) {
  return guarded(ctx, [&] {
    Engine &E = ctx->E;
    cudaSetDevice(E.C.device);
    const long long cnt = E.C.tree.ncells * (long long)tri(E.C.prm.P);
    EXA_CUDA(cudaStreamSynchronize(E.C.stream));
    if (Mh && E.up_ok && cnt) EXA_CUDA(cudaMemcpy(Mh, E.M.p, cnt * sizeof(double2), cudaMemcpyDeviceToHost));
    if (Lh && E.lists_ok && cnt) EXA_CUDA(cudaMemcpy(Lh, E.L.p, cnt * sizeof(double2), cudaMemcpyDeviceToHost));
  });
}

void *exafmm_stream(exafmm_ctx *ctx) { return ctx ? (void *)ctx->E.C.stream : nullptr; }

int exafmm_write_list(exafmm_ctx *ctx, const char *path, int rank) {
  return guarded(ctx, [&] {
    Engine &E = ctx->E;
    if (!E.lists_ok) throw std::runtime_error("no interaction lists (traverse first)");
    cudaSetDevice(E.C.device);
    const long long nc = E.C.tree.ncells;
    std::vector<int> m2l_off(nc + 1, 0), p2p_off(nc + 1, 0);
    std::vector<int2> pl(nc);
    std::vector<double4> x(nc);
    if (nc) {
      EXA_CUDA(cudaMemcpy(m2l_off.data(), E.lists.m2l_off.p, (nc + 1) * sizeof(int), cudaMemcpyDeviceToHost));
      EXA_CUDA(cudaMemcpy(p2p_off.data(), E.lists.p2p_off.p, (nc + 1) * sizeof(int), cudaMemcpyDeviceToHost));
      EXA_CUDA(cudaMemcpy(pl.data(), E.C.tree.cell_pl.p, nc * sizeof(int2), cudaMemcpyDeviceToHost));
      EXA_CUDA(cudaMemcpy(x.data(), E.C.tree.cell_x.p, nc * sizeof(double4), cudaMemcpyDeviceToHost));
    }
    // BuildTree::nodes2cells (include/build_tree.h:132): getKey(C->X, X0 - R0, 2 C->R, level)
    std::vector<unsigned long long> icell(nc);
    for (long long c = 0; c < nc; c++) {
      const double X[3] = {x[c].x, x[c].y, x[c].z};
      const double Xmin[3] = {x[0].x - x[0].w, x[0].y - x[0].w, x[0].z - x[0].w};
      icell[c] = morton_key(X, Xmin, 2 * x[c].w, pl[c].y);
    }
    write_list_file(path, rank, nc, icell.data(), p2p_off.data(), m2l_off.data());
  });
}

int exafmm_write_time(exafmm_ctx *ctx, const char *path, int rank) {
  return guarded(ctx, [&] {
    Engine &E = ctx->E;
    cudaSetDevice(E.C.device);
    E.tm.fold();
    write_time_file(path, rank, E.tm.timer);
    E.tm.timer.clear();
  });
}

int exafmm_take_timers(exafmm_ctx *ctx, int cap, char *names, double *seconds, int *count) {
  return guarded(ctx, [&] {
    if (!count) throw std::runtime_error("null count");
    Engine &E = ctx->E;
    cudaSetDevice(E.C.device);
    E.tm.fold();
    *count = (int)E.tm.timer.size();
    if (!names || !seconds) return;  // the count only
    if (cap < *count) throw std::runtime_error("timer arrays too short");
    int k = 0;
    for (auto &kv : E.tm.timer) {
      std::snprintf(names + 32 * k, 32, "%s", kv.first.c_str());
      seconds[k++] = kv.second;
    }
    E.tm.timer.clear();
  });
}

int exafmm_phase_times(exafmm_ctx *ctx, double *ms8) {
  return guarded(ctx, [&] {
    Engine &E = ctx->E;
    if (!E.tm.live) throw std::runtime_error("no timed solve");
    EXA_CUDA(cudaStreamSynchronize(E.C.stream));
    float t;
    for (int k = 0; k < 7; k++) {
      EXA_CUDA(cudaEventElapsedTime(&t, E.tm.ev[k], E.tm.ev[k + 1]));
      ms8[k] = t;
    }
    EXA_CUDA(cudaEventElapsedTime(&t, E.tm.ev[0], E.tm.ev[7]));
    ms8[7] = t;
  });
}

long long exafmm_launch_count(void) { return launch_count(); }

int exafmm_get_dipole(exafmm_ctx *ctx, const double *X0, double *dipole3) {
  return guarded(ctx, [&] {
    if (!dipole3) throw std::runtime_error("null dipole output");
    ctx->E.get_dipole(X0, dipole3);
  });
}

int exafmm_dipole_correction(exafmm_ctx *ctx, const double *dipole3, long long num_bodies) {
  return guarded(ctx, [&] {
    if (!dipole3) throw std::runtime_error("null dipole");
    ctx->E.dipole_correction(dipole3, num_bodies);
  });
}

int exafmm_device_bytes(exafmm_ctx *ctx, long long *bytes) {
  if (!ctx || !bytes) return 2;
  *bytes = ctx->E.C.dev_bytes;
  return 0;
}

double exafmm_drift(double x, long long k, int up) { return up ? drift_up(x, k) : drift_down(x, k); }

}  // extern "C"
