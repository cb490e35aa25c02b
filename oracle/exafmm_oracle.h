/* CPU restatement of the exafmm-beta Laplace FMM evaluation path, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY: this is the oracle the GPU engine is checked
 * against.  Only tests, __graft_entry__.smoke() and the CPU-baseline leg of
 * bench.py may load it; the product library never links or calls it.
 *
 * Every routine follows the reference file and lines cited beside it.  The
 * restatement is pinned to the reference itself (oracle/_ref, the reference
 * headers compiled in place) by tests/test_oracle.py and by the golden
 * fixtures under tests/golden/.
 *
 * Conventions (shared with the GPU engine and the reference harness):
 *   bodies:      xyzq[4*i + {0,1,2,3}] = x, y, z, charge, caller's order
 *   results:     trg[4*i + {0,1,2,3}]  = potential, d/dx, d/dy, d/dz
 *   expansions:  interleaved (re, im), NTERM = P(P+1)/2 entries, index
 *                n(n+1)/2 + m for 0 <= m <= n < P
 *   cells:       ints  C x 5 = IPARENT, ICHILD, NCHILD, IBODY, NBODY
 *                reals C x 4 = X, Y, Z, R
 *   lists:       pairs (target cell, source cell)
 */
#ifndef EXAFMM_ORACLE_H
#define EXAFMM_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_run oracle_run;

/* BoundBox::getBounds with its sequential drift (include/bound_box.h:11-25). */
void oracle_bounds(int n, const double *xyzq, double *bounds6);
/* One coordinate of the same recurrence: x -/+ 1e-5 applied k times, stepwise. */
double oracle_drift_seq(double x, long long k, int up);

/* Full solve (examples/fmm.cxx:163-179).  bounds6 may be NULL. */
oracle_run *oracle_solve(int n, const double *xyzq, int P, double theta, int ncrit,
                         int nspawn, int images, double cycle, const double *bounds6,
                         int dipole_correction);
int oracle_num_cells(const oracle_run *r);
int oracle_num_m2l(const oracle_run *r);
int oracle_num_p2p(const oracle_run *r);
int oracle_depth(const oracle_run *r);
void oracle_get_bounds(const oracle_run *r, double *bounds6);
void oracle_get_trg(const oracle_run *r, double *trg);
void oracle_get_perm(const oracle_run *r, int *perm);
void oracle_get_cells(const oracle_run *r, int *ints, double *reals);
void oracle_get_lists(const oracle_run *r, int *m2l, int *p2p);
void oracle_get_expansions(const oracle_run *r, double *M, double *L);
void oracle_free(oracle_run *r);

/* Tree only (BuildTree::buildTree, include/build_tree.h:186-209). */
oracle_run *oracle_build_tree(int n, const double *xyzq, int ncrit, const double *bounds6);

/* Per-operator forms, same argument meaning as the reference harness. */
void oracle_p2m(int P, const double *X, int n, const double *xyzq, double *M);
void oracle_m2m(int P, const double *Xp, int nchild, const double *Xc, const double *Mc, double *Mp);
void oracle_m2l(int P, const double *Xi, const double *Xj, const double *Mj, double *Li,
                const double *Xperiodic);
void oracle_l2l(int P, const double *Xc, const double *Xp, const double *Lp, double *Lc);
void oracle_l2p(int P, const double *X, const double *L, int n, const double *xyzq, double *trg);
void oracle_p2p(int ni, const double *xi, int nj, const double *xj, const double *Xperiodic,
                double *trg);
/* Traversal::direct (include/traversal.h:355-377), multithreaded over targets. */
/* Ewald summation (ewald.h): wave part, real part at the nearest image, self term; trg accumulates. */
void oracle_ewald(int n, const double *xyzq, int ksize, double alpha, double sigma, double cutoff, double cycle,
                  double *trg);
void oracle_direct(int ni, const double *xi, int nj, const double *xj, int images, double theta,
                   double cycle, double *trg);

#ifdef __cplusplus
}
#endif
#endif
