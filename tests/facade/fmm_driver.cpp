// A driver written against include/exafmm_b200.hpp in the shape of
// examples/fmm.cxx (its objects, call sequence and accuracy check), used by
// tests/test_gpu_facade.py.  Arguments: output file, numBodies, distribution,
// P, theta, ncrit, nspawn, images, IneJ (0/1).  Writes, in binary: N, then per
// body in the order the facade leaves them X[3], SRC, IBODY, TRG[4]; the cell
// count and each cell's IPARENT ICHILD NCHILD IBODY NBODY; then the relative
// errors against the direct sum on 100 sampled targets.  Also writes the list
// file and the time file (the solve timed as "Total FMM") in the working
// directory.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "exafmm_b200.hpp"
using namespace exafmm_laplace;

int main(int argc, char **argv) {
  if (argc < 10) return 2;
  const char *out = argv[1];
  const int numBodies = std::atoi(argv[2]);
  const char *distribution = argv[3];
  const int P = std::atoi(argv[4]), ncrit = std::atoi(argv[6]), nspawn = std::atoi(argv[7]);
  const int images = std::atoi(argv[8]), IneJ = std::atoi(argv[9]);
  const double theta = std::atof(argv[5]);
  const vec3 cycle = 2 * M_PI;
  const real_t eps2 = 0.0;
  const complex_t wavek = complex_t(10., 1.) / real_t(2 * M_PI);
  Bodies bodies, bodies2, jbodies, buffer;
  BoundBox boundBox;
  Bounds bounds;
  BuildTree buildTree(ncrit);
  Cells cells, jcells;
  Dataset data;
  Kernel kernel(P, eps2, wavek);
  Traversal traversal(kernel, theta, nspawn, images, "./");
  UpDownPass upDownPass(kernel);
  Verify verify;
  try {
    bodies = data.initBodies(numBodies, distribution, 0);
    if (IneJ) {
      for (B_iter B = bodies.begin(); B != bodies.end(); B++) {
        B->X[0] += M_PI;
        B->X[0] *= 0.5;
      }
      jbodies = data.initBodies(numBodies, distribution, 1);
      for (B_iter B = jbodies.begin(); B != jbodies.end(); B++) {
        B->X[0] -= M_PI;
        B->X[0] *= 0.5;
      }
    }
    logger::startTimer("Total FMM");
    bounds = boundBox.getBounds(bodies);
    if (IneJ) bounds = boundBox.getBounds(jbodies, bounds);
    cells = buildTree.buildTree(bodies, buffer, bounds);
    upDownPass.upwardPass(cells);
    traversal.initListCount(cells);
    traversal.initWeight(cells);
    if (IneJ) {
      jcells = buildTree.buildTree(jbodies, buffer, bounds);
      upDownPass.upwardPass(jcells);
      traversal.traverse(cells, jcells, cycle, true);
    } else {
      traversal.traverse(cells, cells, cycle, true);
      jbodies = bodies;
    }
    upDownPass.downwardPass(cells);
    logger::stopTimer("Total FMM");
    logger::writeTime(0);
    traversal.writeList(cells, 0);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  FILE *f = std::fopen(out, "wb");
  if (!f) return 3;
  const long long n = (long long)bodies.size(), nc = (long long)cells.size();
  std::fwrite(&n, sizeof(n), 1, f);
  for (const Body &B : bodies) {
    const double v[9] = {B.X[0], B.X[1], B.X[2], B.SRC, (double)B.IBODY, B.TRG[0], B.TRG[1], B.TRG[2], B.TRG[3]};
    std::fwrite(v, sizeof(double), 9, f);
  }
  std::fwrite(&nc, sizeof(nc), 1, f);
  for (const Cell &C : cells) {
    const int v[5] = {C.IPARENT, C.ICHILD, C.NCHILD, C.IBODY, C.NBODY};
    std::fwrite(v, sizeof(int), 5, f);
  }
  // examples/fmm.cxx:107-124: 100 sampled targets against the direct sum
  buffer = bodies;
  data.sampleBodies(bodies, 100);
  bodies2 = bodies;
  data.initTarget(bodies);
  traversal.direct(bodies, jbodies, cycle);
  const double err[2] = {std::sqrt(verify.getDifScalar(bodies, bodies2) / verify.getNrmScalar(bodies)),
                         std::sqrt(verify.getDifVector(bodies, bodies2) / verify.getNrmVector(bodies))};
  std::fwrite(err, sizeof(double), 2, f);
  std::fclose(f);
  std::printf("facade driver: N=%lld cells=%lld pot %.3e acc %.3e\n", n, nc, err[0], err[1]);
  return 0;
}
