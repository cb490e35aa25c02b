/* MD-code ABI in the shape of the reference's distributed MD wrapper
 * (wrappers/md_distributed.cxx:36-461, driven by
 * wrappers/test_md_distributed.cxx), for one process and one GPU, in
 * libexafmm_md_distributed.so.  Same names, argument meaning and call order:
 *
 *   FMM_Init(images, threads, theta, cutoff, verbose, path);
 *   Set_Index(&ni, nimax, res_index, x, q, v, cycle);     or
 *   FMM_Partition(&ni, nimax, res_index, x, q, v, cycle);
 *   FMM_FMM(ni, &nj, res_index, x, q, p, f, cycle);        each step
 *   FMM_Ewald(...) / FMM_Cutoff(...) / Dipole_Correction(...);   checks
 *   FMM_Finalize();
 *
 * All arrays are double: x is n x 3 (wrapped into [-cycle/2, cycle/2] per
 * dimension, any image accepted), q the charges, v the velocities that move with
 * their bodies, p and f (n and n x 3) the potential and its gradient in the
 * reference's sign convention.  cycle points to the three box edges.  The solve
 * is the reference's Laplace FMM with P = 10, ncrit = 32, nspawn = 1000, the
 * caller's theta and image levels and the dipole correction, in FP64 on the GPU.
 *
 * One process holds the whole system: the MPI steps of the reference take
 * their one-rank form, and the ghost bodies FMM_FMM appends are the periodic
 * images of the bodies near the box faces.  The periodic solve and the Ewald
 * sum need a cubic box.  The reference's regression-file helpers
 * (FMM_Verify_*, FMM_Only_Accuracy) are not provided.  The reference reports no
 * errors; here a failing call leaves its outputs untouched, prints the reason on
 * stderr and keeps it for FMM_Error().
 *
 * This ABI shares FMM_Init, FMM_Finalize and FMM_Partition with the GROMACS
 * one (include/exafmm_md.h) under other signatures, as the reference's two
 * wrappers do; the two live in separate libraries. */
#ifndef EXAFMM_MD_DISTRIBUTED_H
#define EXAFMM_MD_DISTRIBUTED_H
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

/* md_distributed.cxx:36-74: theta and the ghost cutoff of the solves; threads is
 * ignored (the GPU runs them), path is kept for records. */
void FMM_Init(int images, int threads, double theta, double cutoff, bool verbose, const char *path);
/* md_distributed.cxx:76-87. */
void FMM_Finalize(void);
/* md_distributed.cxx:89-142: wraps the bodies, takes their bounds (no
 * octsection) and builds the tree, then labels bodies in groups of 3 to 6 per
 * cell from the process's drand48 sequence: a group's first body gets the next
 * id, the others -(their place in the group).  When *ni < nimax, returns
 * res_index (the labels), x (unwrapped), q and v in the tree's body order. */
void Set_Index(int *ni, int nimax, int *res_index, double *x, double *q, double *v, double *cycle);
/* md_distributed.cxx:144-188: wraps the bodies, takes the bounds of the local
 * domain (octsection with one rank) and builds the tree; when *ni < nimax,
 * returns res_index, x (unwrapped), q and v in the tree's body order. */
void FMM_Partition(int *ni, int nimax, int *res_index, double *x, double *q, double *v, double *cycle);
/* md_distributed.cxx:190-308: one periodic FMM solve in the bounds of the last
 * FMM_Partition / Set_Index, p and f accumulated and written in the tree's body
 * order (the caller's order after FMM_Partition).  Then *nj = ni + the ghost
 * count (bodies at one of the 26 neighbouring images inside the local bounds
 * widened by the cutoff); when that is below the *nj passed in, their
 * res_index, x and q fill slots ni.. of the arrays. */
void FMM_FMM(int ni, int *nj, int *res_index, double *x, double *q, double *p, double *f, double *cycle);
/* md_distributed.cxx:310-360: Ewald summation (wave part over |k| <= ksize, real
 * part within cutoff at the nearest image, self term), FP64 on the GPU,
 * accumulated into p, f in the caller's order. */
void FMM_Ewald(int ni, double *x, double *q, double *p, double *f, int ksize, double alpha, double sigma,
               double cutoff, double *cycle);
/* md_distributed.cxx:383-405: the dipole correction with the dipole summed in
 * float, on the host as there. */
void Dipole_Correction(int ni, double *x, double *q, double *p, double *f, double *cycle);
/* md_distributed.cxx:407-461: direct sum over every pair closer than cutoff
 * at the images out to the cutoff, FP64 on the GPU; p += sum q/r, f -= sum dx q/r^3. */
void FMM_Cutoff(int ni, double *x, double *q, double *p, double *f, double cutoff, double *cycle);
/* No counterpart in the reference: the reason the last call failed, or "". */
const char *FMM_Error(void);

#ifdef __cplusplus
}
#endif
#endif
