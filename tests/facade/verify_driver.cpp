// Verify::regression of include/exafmm_b200.hpp over a sequence of calls on one
// Verify object, for tests/test_facade.py.  Arguments: path, then five tokens a
// call (key, time 0/1, iteration, value, value2).  Prints each call's result.
#include <cstdio>
#include <cstdlib>

#include "exafmm_b200.hpp"
using namespace exafmm_laplace;

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  Verify verify(argv[1]);
  for (int a = 2; a + 4 < argc; a += 5) {
    const bool pass = verify.regression(std::strtoull(argv[a], nullptr, 10), std::atoi(argv[a + 1]) != 0,
                                        std::atoi(argv[a + 2]), std::atof(argv[a + 3]), std::atof(argv[a + 4]));
    std::printf("%d\n", pass ? 1 : 0);
  }
  return 0;
}
