// Host launchers for the expansion operators and the traversal.
#pragma once
#include "context.h"

namespace exafmm_b200 {

struct FmmArgs {
  int P = 10;
  int ncrit = 64;
  long long ncells = 0;
  double cycle = 0;
  cudaStream_t stream = nullptr;
  const long long *lvl = nullptr;
  const int *nd_cell = nullptr;
  const int4 *cell_b = nullptr;
  const int2 *cell_pl = nullptr;
  const double4 *cell_x = nullptr;
  const double4 *xt = nullptr;         // bodies in tree order
  const int *m2l_off = nullptr, *m2l_src = nullptr;
  const int *p2p_off = nullptr, *p2p_src = nullptr;
  double2 *M64 = nullptr, *L64 = nullptr;
  double4 *trg64 = nullptr;            // results in tree order
};

void p2m_fp64(const FmmArgs &a);
void m2m_fp64(const FmmArgs &a, int level, long long nodes_at_level);
void m2l_fp64(const FmmArgs &a);
void l2l_fp64(const FmmArgs &a, int level, long long nodes_at_level);
void l2p_fp64(const FmmArgs &a);
void p2p_fp64(const FmmArgs &a);

// Interaction lists of the dual tree traversal (traverse.cu).
struct ListBufs {
  long long q_cap = 0, m2l_cap = 0, p2p_cap = 0;
  DBuf<int2> q0, q1;                 // pair queues (ci, cj | image << 26)
  DBuf<int2> m2l, p2p;               // emitted pairs, traversal order
  DBuf<unsigned> key, key_alt;       // sort keys (target cell)
  DBuf<int> val, val_alt;            // sort payloads (source | image << 26)
  DBuf<int> m2l_off, p2p_off;        // CSR offsets per target cell (ncells + 1)
  DBuf<int> m2l_src, p2p_src;        // CSR sources
  DBuf<long long> cnt;               // per sweep: queue size, m2l base, p2p base
  long long n_m2l = 0, n_p2p = 0;
  int sweeps = 0;
};

// Runs the traversal into lists (unsorted), then groups them by target cell.
// Returns false when a capacity was exceeded; the capacities are then grown to
// the counts the traversal reported and the caller reruns it.
bool traverse(Context &C, ListBufs &lb);

}  // namespace exafmm_b200
