// The examples/kernel.cxx chain through include/exafmm_b200.hpp's Kernel:
// P2M at a source leaf, M2M to its parent, M2L to the target's parent, L2L to
// the target leaf, L2P at the target, and P2P for the direct value, on cells
// laid out as the reference's (ICHILD and IPARENT relative to the first cell).
// Arguments: output file, P.  Writes Mj, MJ, LI, Li (complex, NTERM each),
// then the target's TRG from L2P and from P2P (4 doubles each).
#include <cstdio>
#include <cstdlib>

#include "exafmm_b200.hpp"
using namespace exafmm_laplace;

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  const int P = std::atoi(argv[2]);
  Kernel kernel(P, 0.0, complex_t(10., 1.) / real_t(2 * M_PI));
  Bodies jbodies(1), bodies(1), bodies2(1);
  for (int d = 0; d < 3; d++) {
    jbodies[0].X[d] = 2;
    bodies[0].X[d] = 2;
  }
  bodies[0].X[0] = -2;
  jbodies[0].SRC = bodies[0].SRC = 1;
  bodies[0].TRG = 0;
  bodies2 = bodies;
  Cells cells(4);
  const double X[4][3] = {{3, 1, 1}, {4, 0, 0}, {-4, 0, 0}, {-3, 1, 1}};  // Cj, CJ, CI, Ci
  for (int c = 0; c < 4; c++) {
    for (int d = 0; d < 3; d++) cells[c].X[d] = X[c][d];
    cells[c].R = 1;
    cells[c].NBODY = 0;
    cells[c].NCHILD = 0;
  }
  C_iter C0 = cells.begin(), Cj = C0, CJ = C0 + 1, CI = C0 + 2, Ci = C0 + 3;
  Cj->BODY = jbodies.begin();
  Cj->NBODY = 1;
  CJ->ICHILD = 0;
  CJ->NCHILD = 1;
  Ci->IPARENT = 2;
  Ci->BODY = bodies.begin();
  Ci->NBODY = 1;
  try {
    kernel.P2M(Cj);
    kernel.M2M(CJ, C0);
    kernel.M2L(CI, CJ);
    kernel.L2L(Ci, C0);
    kernel.L2P(Ci);
    Cells c2(1);
    c2[0] = *Ci;
    c2[0].BODY = bodies2.begin();
    kernel.P2P(c2.begin(), Cj);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  FILE *f = std::fopen(argv[1], "wb");
  if (!f) return 3;
  for (C_iter C : {Cj, CJ}) std::fwrite(C->M.data(), sizeof(complex_t), C->M.size(), f);
  for (C_iter C : {CI, Ci}) std::fwrite(C->L.data(), sizeof(complex_t), C->L.size(), f);
  for (const Bodies *b : {&bodies, &bodies2}) {
    const double v[4] = {(*b)[0].TRG[0], (*b)[0].TRG[1], (*b)[0].TRG[2], (*b)[0].TRG[3]};
    std::fwrite(v, sizeof(double), 4, f);
  }
  std::fclose(f);
  return 0;
}
