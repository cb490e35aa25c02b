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
#include "verify.h"

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

// Dataset::writeSources / writeTargets (include/dataset.h:186-204, 276-287)
// of n bodies given as n x 4 (x, y, z, q) and n x 4 targets, into the current
// directory as the reference names them (source%04d.dat, target%04d.dat).
void ref_dataset_write(int n, const double *xyzq, const double *trg, int mpirank) {
  Dataset data;
  Bodies bodies(n);
  for (int i = 0; i < n; i++) {
    for (int d = 0; d < 3; d++) bodies[i].X[d] = xyzq[4 * i + d];
    bodies[i].SRC = xyzq[4 * i + 3];
    for (int d = 0; d < 4; d++) bodies[i].TRG[d] = trg[4 * i + d];
  }
  data.writeSources(bodies, mpirank);
  data.writeTargets(bodies, mpirank);
}

// Dataset::readSources twice on one Dataset object, then readTargets twice on
// another (include/dataset.h:162-184, 259-274): successive reads of n bodies
// each from the current directory, each going on from the object's file
// position.  src_out holds 2 x n x (x, y, z, q), trg_out 2 x n x 4.
void ref_dataset_read(int n, int mpirank, double *src_out, double *trg_out) {
  Dataset data, tdata;
  for (int r = 0; r < 2; r++) {
    Bodies bodies(n);
    data.readSources(bodies, mpirank);
    for (int i = 0; i < n; i++) {
      for (int d = 0; d < 3; d++) src_out[(r * n + i) * 4 + d] = bodies[i].X[d];
      src_out[(r * n + i) * 4 + 3] = bodies[i].SRC;
    }
  }
  for (int r = 0; r < 2; r++) {
    Bodies bodies(n);
    tdata.readTargets(bodies, mpirank);
    for (int i = 0; i < n; i++)
      for (int d = 0; d < 4; d++) trg_out[(r * n + i) * 4 + d] = bodies[i].TRG[d];
  }
}

// Verify::regression (include/verify.h:118-175) over a sequence of calls on one
// Verify object whose path is `path`: calls i uses keys[i], time[i],
// iteration[i], value[i], value2[i]; pass[i] receives its result.
void ref_verify_sequence(const char *path, int n, const unsigned long long *keys, const int *time,
                         const int *iteration, const double *value, const double *value2, int *pass) {
  Verify verify(path);
  verify.verbose = false;
  for (int i = 0; i < n; i++) pass[i] = verify.regression(keys[i], time[i] != 0, iteration[i], value[i], value2[i]);
}

// n draws of drand48 after srand48(seed), the sequence every generator uses.
void ref_drand48(long seed, int n, double *out) {
  srand48(seed);
  for (int i = 0; i < n; i++) out[i] = drand48();
}

}  // extern "C"
