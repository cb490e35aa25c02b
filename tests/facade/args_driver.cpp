// Args of include/exafmm_b200.hpp, for tests/test_facade.py: parses its own
// command line and prints the parsed fields and getKey as name / value pairs.
#include "exafmm_b200.hpp"
using namespace EXAFMM_NAMESPACE;

int main(int argc, char **argv) {
  Args args(argc, argv);
  num_threads(args.threads);
  std::cout << "ncrit " << args.ncrit << " P " << args.P << " theta " << args.theta << " numBodies " << args.numBodies
            << " distribution " << args.distribution << " images " << args.images << " nspawn " << args.nspawn
            << " threads " << args.threads << " repeat " << args.repeat << " dual " << args.dual << " IneJ "
            << args.IneJ << " path " << args.path << " verbose " << args.verbose << " key " << args.getKey()
            << std::endl;
  return 0;
}
