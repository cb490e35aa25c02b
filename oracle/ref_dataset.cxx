// Reference harness for the body generators: the UNMODIFIED exafmm-beta
// Dataset class (include/dataset.h), compiled in place (-I into the reference
// tree, nothing copied) without fast-math, as the reference's default build
// compiles it (plain IEEE arithmetic and scalar libm calls).
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
// calls this file.  Built by oracle/Makefile into
// oracle/_ref/libexafmm_ref_dataset.so.
#include <cstring>

#include "types.h"
#include "dataset.h"

using namespace exafmm_laplace;

extern "C" {

// Dataset::initBodies(numBodies, distribution, mpirank, mpisize, numSplit)
// (include/dataset.h:229-257): positions and charges as n x 4 (x, y, z, q),
// up to cap bodies.  Returns the number of bodies the reference made.
int ref_dataset_init_bodies(int n, const char *distribution, int mpirank, int mpisize, int num_split,
                            double *xyzq, int cap) {
  Dataset data;
  Bodies bodies = data.initBodies(n, distribution, mpirank, mpisize, num_split);
  const int m = int(bodies.size());
  for (int i = 0; i < m && i < cap; i++) {
    for (int d = 0; d < 3; d++) xyzq[4 * i + d] = bodies[i].X[d];
    xyzq[4 * i + 3] = bodies[i].SRC;
  }
  return m;
}

// n draws of drand48 after srand48(seed), the sequence every generator uses.
void ref_drand48(long seed, int n, double *out) {
  srand48(seed);
  for (int i = 0; i < n; i++) out[i] = drand48();
}

}  // extern "C"
