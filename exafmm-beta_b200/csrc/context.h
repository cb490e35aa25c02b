// Solve context: every device buffer one FMM solve touches, owned per caller.
#pragma once
#include <vector>

#include "engine.h"

namespace exafmm_b200 {

enum Precision : int { kFP64 = 0, kMixed = 1 };

struct Params {
  int P = 10;
  double theta = 0.4;
  int ncrit = 64;
  int nspawn = 5000;
  int images = 0;
  double cycle = 6.283185307179586;
  int precision = kFP64;
  // Mixed form: which operators run in FP32, and which M2L pairs (target level
  // and source/target level difference) may; the rest stays FP64.
  int mixed_m2l = 1;
  int mixed_p2p = 1;
  int mixed_min_level = 2;
  int mixed_max_dl = 3;
  int mixed_gemm = 1;     // per-class products for frequent offset classes: 0 off, 1 where they pay, 2 always
  int mixed_gemm_tc = 1;  // ... on the tensor cores (bf16x3), else FP32 on the CUDA cores
  int p2p_tpl = 0;        // mixed P2P targets per lane: 0 by leaf size (two or three), 2 or 3 for every leaf
};

// Level-ordered octree nodes plus the reference-layout cell table.
struct TreeBufs {
  long long n = 0;
  DBuf<double4> xyzq;        // bodies, caller order
  DBuf<double4> xyzq_tree;   // bodies, tree order
  DBuf<unsigned long long> keys, keys_alt;
  DBuf<int> perm, perm_alt;  // perm[tree slot] = caller index
  DBuf<double> bounds;       // Xmin[3], Xmax[3]
  DBuf<double> box;          // X0[3], R0
  DBuf<unsigned long long> bounds_enc;
  // nodes (level order)
  long long node_cap = 0;
  DBuf<int> nd_begin, nd_count, nd_nchild, nd_childbeg, nd_nnode, nd_cell, nd_pcell, nd_ichild;
  DBuf<double4> nd_x;
  DBuf<long long> lvl;       // [0, L]: node count per level; [L+1, 2L+1]: level start
  DBuf<int> split_level;     // deepest level with a node of more than ncrit bodies (-1: none)
  // cells (reference layout)
  long long cell_cap = 0;
  DBuf<int4> cell_b;         // ibody, nbody, ichild, nchild
  DBuf<int2> cell_pl;        // iparent, level
  DBuf<double4> cell_x;      // X, Y, Z, R
  DBuf<int> cell_node;       // cell -> node
  // host mirrors (valid after sync_tree)
  int ncells = 0;
  int depth = 0;
  long long lvl_host[2 * (kMaxLevels + 1)];

  // Forest of independent systems (exafmm_set_systems).  nsys == 0 is the
  // plain path: one system, root cell 0.  Otherwise the bodies of system s are
  // [sys_off[s], sys_off[s+1]) in caller order and in tree order alike; each
  // non-empty system has a root node at level 0 (root node k belongs to system
  // root_sys[k]) and its cells are [sys_cell[s], sys_cell[s+1]), laid out as
  // that system's solo tree would be, shifted by sys_cell[s].
  int nsys = 0;
  int nroots = 0;
  long long ntiles = 0;                 // body tiles of at most kForestTile bodies, none across systems
  std::vector<long long> sys_off_host;  // nsys + 1
  std::vector<int> sys_cell_host;       // nsys + 1 (valid after sync_tree)
  DBuf<long long> sys_off;
  DBuf<int> sys_root;                   // per system: its root node, or -1 when it has no bodies
  DBuf<int> root_sys;                   // per root node: its system
  DBuf<int> tile_sys;
  DBuf<long long> tile_beg;
  DBuf<unsigned long long> sys_enc;     // 16 words per system (bounds reduction)
  DBuf<double> sys_bounds;              // Xmin[3], Xmax[3] per system
  DBuf<double4> sys_box;                // X0, R0 per system
  DBuf<int> sys_cell;
  DBuf<int> nd_sys;                     // node -> system
  DBuf<unsigned> fs_key, fs_key_alt;    // second sort pass: system of each key-sorted body
  DBuf<int> fs_idx, fs_idx_alt;
};

// Bodies per tile of the forest's per-system reductions.
constexpr int kForestTile = 4096;

struct Context {
  long long dev_bytes = 0;     // device bytes held by this context's buffers (declared first: outlives them)
  Params prm;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_link = nullptr;  // when set, recorded between growing the octree and linking the cells
  int device = 0;
  DBuf<int> err;               // device error word
  unsigned char *pin = nullptr;  // pinned block (pinned_block_acquire): the error word, then readback staging
  int *err_host = nullptr;     // pinned mirror of the error word (the start of pin)
  TreeBufs tree;
  ScanWork scan;
  SortWork sort;
  std::string last_error;
};

// Pinned host block of a context: its error word at offset 0 and, from
// kPinScratch on, the staging area of a solve's small device-to-host readbacks
// (level counts, traversal counts, the class count), so that a solve copies
// nothing into pageable memory.  Blocks come from a process-wide pinned slab
// and return to it when the context is destroyed: creating and destroying
// contexts neither pins nor unpins host memory (cudaFreeHost waits for the
// whole device, which stalls every other context's stream in a server).
constexpr size_t kPinBytes = 4096, kPinScratch = 64;
unsigned char *pinned_block_acquire();
void pinned_block_release(unsigned char *p);

// Tree construction (tree.cu).
void compute_bounds(Context &C);
void set_bounds(Context &C, const double *bounds6_host);
// BoundBox::getBounds(bodies, bounds): C's bounds extended by n bodies x (device).
void extend_bounds(Context &C, const double4 *x, long long n);
void build_tree(Context &C);
void sync_tree(Context &C);  // reads cell count, depth and the error word

}  // namespace exafmm_b200
