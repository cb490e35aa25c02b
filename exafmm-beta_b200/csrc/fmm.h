// Host launchers for the expansion operators and the traversal.
#pragma once
#include "context.h"

namespace exafmm_b200 {

struct FmmArgs {
  int P = 10;
  int ncrit = 64;
  long long ncells = 0;
  long long n = 0;                     // bodies
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
  // separate source bodies (their own tree): the source side of M2L and P2P
  // (null: the sources are the targets)
  const int4 *src_cell_b = nullptr;
  const int2 *src_cell_pl = nullptr;
  const double4 *src_cell_x = nullptr;
  const double4 *src_xt = nullptr;
  const double2 *src_M64 = nullptr;
  // forest of systems: bodies of system s are [sys_off[s], sys_off[s+1]) in
  // tree order, its root box sys_box[s] (null: one system, root cell 0)
  int nsys = 0;
  const long long *sys_off = nullptr;
  const double4 *sys_box = nullptr;
};

void p2m_fp64(const FmmArgs &a);
void m2m_fp64(const FmmArgs &a, int level, long long nodes_at_level);
// Generic FP64 M2L.  With skip_min_level >= 0 it leaves out the pairs the
// mixed-precision kernel takes (target level >= skip_min_level and
// |level difference| <= skip_max_dl).
void m2l_fp64(const FmmArgs &a, int skip_min_level = -1, int skip_max_dl = 0);
void l2l_fp64(const FmmArgs &a, int level, long long nodes_at_level);
void l2p_fp64(const FmmArgs &a);
void p2p_fp64(const FmmArgs &a);

// Mixed form: FP32 M2L for targets at level >= kMixedMinLevel and source/target
// level differences of at most kMixedMaxDl; everything else in FP64.
constexpr int kMixedMinLevel = 3;
constexpr int kMixedMaxDl = 3;

// Register-resident unrolled M2L (m2l.cu) for the orders it is built for.
bool m2l_fast_supported(int P, bool mixed);
// Ms = A_n^m M_n^m / R^n per cell, FP32 (mixed) or FP64: of the cells of a,
// or of any cell table (a separate source tree's).
void scale_multipoles(const FmmArgs &a, bool mixed, void *Ms);
void scale_multipoles(int P, const double2 *M, const double4 *cell_x, long long ncells, bool mixed, void *Ms,
                      cudaStream_t st);
// In mixed mode only pairs with target level >= min_level and |level difference|
// <= max_dl are taken (FP64 takes the rest, compacted by m2l_complement).
// taken: pairs another kernel evaluates (skipped here), or null.
bool m2l_fast(const FmmArgs &a, bool mixed, const void *Ms, int min_level = 0, int max_dl = 0,
              const unsigned char *taken = nullptr);

// Class-grouped tile M2L (m2l_gemm.cu): the mixed-regular pairs whose offset
// class is frequent, FP32 products with FP64 accumulation, added to L.  When it
// returns true, left_off / left_src hold the other mixed-regular pairs, grouped
// by target, for the pair-by-pair FP32 kernel.
struct M2LGemmBufs {
  DBuf<unsigned long long> hk;        // class hash table: keys
  DBuf<int> hid;                      // slot -> class id (or -1)
  DBuf<int> pair_slot;                // per list entry: hash slot (or -1)
  DBuf<unsigned long long> ck, ck_alt;
  DBuf<int> cs, cs_alt;
  DBuf<float> K;                      // per class operator, FP32, k-major (CUDA-core engine)
  DBuf<float> Msr;                    // scaled multipoles over real degrees of freedom (CUDA-core engine)
  DBuf<unsigned short> Kb;            // per class operator, three bf16 pieces (tensor-core engine)
  DBuf<unsigned short> Msb;           // scaled multipoles, three bf16 pieces (tensor-core engine)
  DBuf<int4> chunks;                  // per chunk: class, first sorted position, pairs (tensor-core engine)
  DBuf<int> ssrc;                     // per sorted taken pair: its source cell (tensor-core engine)
  DBuf<unsigned char> taken;
  DBuf<unsigned> skey, skey_alt;      // pairs sorted by class
  DBuf<int> pval, pval_alt;           // their list positions
  DBuf<int> cstart, cbase;            // class ranges, chunk offsets per class
  DBuf<float> Y;                      // per list entry: the pair's contribution (real dofs)
  DBuf<int> cnt;
  DBuf<int> left_cnt, left_off, left_src;
  DBuf<int> comp_cnt, comp_off, comp_src;  // pairs outside the mixed policy (FP64), per target
  bool force = false;         // use the class products whatever the size (parity tests)
  bool tensor_cores = true;   // tcgen05 bf16x3 products, else FP32 on the CUDA cores
  bool tma = true;            // P = 8 on the tensor cores: source pieces gathered by TMA
};
bool m2l_gemm_supported(int P);
bool m2l_gemm(Context &C, const FmmArgs &a, M2LGemmBufs &g, long long n_m2l, int min_level, int max_dl);
// The pairs outside the mixed policy compacted into g.comp_off / g.comp_src (CSR by target, list order).
long long m2l_complement(Context &C, const FmmArgs &a, M2LGemmBufs &g, long long n_m2l, int min_level, int max_dl);

// Periodic lattice of root images (traversePeriodic), FP64, into L of the root.
// scratch holds lattice_scratch_terms(P) complex values.
long long lattice_scratch_terms(int P);
void lattice_fp64(const FmmArgs &a, int images, double theta, double2 *scratch);
// getDipole about X0 into out3 (device), scratch: 3 * 256 doubles.
void dipole_fp64(const double4 *x, long long n, const double X0[3], double *scratch, double *out3, cudaStream_t st);
// dipoleCorrection on results in tree order (xt: bodies in the same order).
void dipole_correction_fp64(const double4 *xt, double4 *trg, long long n, double cycle, const double dip[3],
                            double nbodies, cudaStream_t st);

// Mixed-precision P2P (p2p32.cu): bodies as two-float pairs relative to the
// root center; periodic selects the form that tests every pair for r = 0.
void rel_bodies32(const FmmArgs &a, float4 *x32);
// The same for other bodies (a separate source tree's) about the root center of a.
void rel_bodies32(const FmmArgs &a, const double4 *xt, long long n, float4 *x32);
// Scratch of the mixed P2P: the persistent kernels' work counters and their
// work order (target leaves by kind, longest first).
struct P2PWork {
  DBuf<unsigned long long> next;   // [2] work counters
  DBuf<unsigned> key, key_alt;     // order keys
  DBuf<int> order, order_alt;      // cells in work order
  DBuf<int> count;                 // [3] leaves of each kind: two targets per lane, three, no P2P list
  // The three-target kind runs on a stream of its own, forked from and joined
  // back to the solve's stream, so its blocks take the SMs that the
  // two-target kind's last leaves leave idle (made on first use).
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  P2PWork() = default;
  P2PWork(const P2PWork &) = delete;
  P2PWork &operator=(const P2PWork &) = delete;
  ~P2PWork() {
    if (side) cudaStreamSynchronize(side);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    if (side) cudaStreamDestroy(side);
  }
};
// x32j (null: x32) holds the source bodies, whose cells are a.src_cell_b when set.
void p2p_mixed(Context &C, const FmmArgs &a, const float4 *x32, bool periodic, P2PWork &w,
               const float4 *x32j = nullptr);

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
bool traverse(Context &C, ListBufs &lb, const TreeBufs *sources = nullptr);

}  // namespace exafmm_b200
