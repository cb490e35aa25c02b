// Writes Dataset::initBodies of include/exafmm_b200.hpp (no GPU involved) as
// binary n x 4 (x, y, z, SRC) for tests/test_facade.py.  Arguments: output
// file, numBodies, distribution, mpirank, mpisize, numSplit.
#include <cstdio>
#include <cstdlib>

#include "exafmm_b200.hpp"
using namespace exafmm_laplace;

int main(int argc, char **argv) {
  if (argc < 7) return 2;
  Dataset data;
  Bodies bodies = data.initBodies(std::atoi(argv[2]), argv[3], std::atoi(argv[4]), std::atoi(argv[5]),
                                  std::atoi(argv[6]));
  FILE *f = std::fopen(argv[1], "wb");
  if (!f) return 3;
  for (const Body &B : bodies) {
    const double v[4] = {B.X[0], B.X[1], B.X[2], B.SRC};
    std::fwrite(v, sizeof(double), 4, f);
  }
  std::fclose(f);
  return 0;
}
