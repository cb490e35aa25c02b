/* MD-code ABI in the shape of the reference's GROMACS wrapper
 * (wrappers/gromacs.cxx:39-363, driven by wrappers/test_gromacs.cxx), for one
 * process and one GPU, in libexafmm_md_gromacs.so (the distributed wrapper's
 * ABI, include/exafmm_md_distributed.h, reuses some of these names under other
 * signatures and lives in its own library).  Same names, argument meaning and
 * call order:
 *
 *   FMM_Init(images, threads, verbose, path);
 *   FMM_Partition(&n, ibody, icell, x, q, cycle);   once, or when bodies moved far
 *   FMM_Coulomb(n, icell, x, q, p, f, cycle);        each step
 *   Ewald_Coulomb(...) / Direct_Coulomb(...);        checks
 *   FMM_Finalize();
 *
 * x is n x 3, positions in [0, cycle)^3 (any period image is accepted: they are
 * wrapped), q the charges; p and f (n and n x 3) accumulate the potential and
 * its gradient, in the reference's sign convention.  The solve is the
 * reference's: Laplace FMM with P = 10, theta = 0.5, ncrit = 32, nspawn = 1000,
 * `images` periodic image levels and the dipole correction, computed in FP64
 * on the GPU (the reference in its real_t, double by default).
 *
 * One process holds the whole system, so the MPI steps of the reference
 * (octsection across ranks, body and LET exchange) reduce to their one-rank
 * form.  Bodies with ICELL < 0 (the residual groups of the reference's
 * EXAFMM_CLUSTER build) are not supported.  The reference reports no errors;
 * here a failing call leaves its outputs untouched, prints the reason on
 * stderr and keeps it for FMM_Error(). */
#ifndef EXAFMM_MD_H
#define EXAFMM_MD_H
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

/* wrappers/gromacs.cxx:39-77: parameters of the solves; threads is ignored
 * (the GPU runs them), path is kept for records. */
void FMM_Init(int images, int threads, bool verbose, const char *path);
/* wrappers/gromacs.cxx:79-90. */
void FMM_Finalize(void);
/* wrappers/gromacs.cxx:92-137: wraps the bodies into the box, takes the
 * bounds of the local domain (octsection with one rank) and builds the tree;
 * returns ibody, icell, x and q reordered into the tree's body order (x
 * unwrapped again).  *n is unchanged with one process. */
void FMM_Partition(int *n, int *ibody, int *icell, float *x, float *q, float cycle);
/* wrappers/gromacs.cxx:139-215: one periodic FMM solve in the bounds of the
 * last FMM_Partition, dipole correction about the origin of the shifted box,
 * p and f accumulated in caller order.  index (Body::ICELL) is not used by the
 * solve. */
void FMM_Coulomb(int n, int *index, float *x, float *q, float *p, float *f, float cycle);
/* wrappers/gromacs.cxx:217-266: Ewald summation (wave part over |k| <= ksize,
 * real part within cutoff, self term) on the GPU in FP64, accumulated into p, f. */
void Ewald_Coulomb(int n, float *x, float *q, float *p, float *f, int ksize, float alpha, float sigma,
                   float cutoff, float cycle);
/* wrappers/gromacs.cxx:289-363: direct sum over the image range sum_{i<images} 3^i
 * (FP64 on the GPU), then the dipole correction in float as there. */
void Direct_Coulomb(int n, float *x, float *q, float *p, float *f, float cycle);
/* No counterpart in the reference: the reason the last call failed, or "". */
const char *FMM_Error(void);

#ifdef __cplusplus
}
#endif
#endif
