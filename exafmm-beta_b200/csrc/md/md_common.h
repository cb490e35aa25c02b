// Host helpers shared by the MD-code ABIs (libexafmm_md_gromacs.so,
// libexafmm_md_distributed.so): periodic wrap / unwrap, the one-rank
// octsection, and the error convention (a failing call leaves its outputs
// untouched, prints the reason and keeps it for FMM_Error()).
#ifndef EXAFMM_MD_COMMON_H
#define EXAFMM_MD_COMMON_H
#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../../include/exafmm_b200.h"

namespace exafmm_md {

// vec.h:217-235 wrap / unwrap, one period per dimension: a coordinate below
// -w/2 or above w/2 moves by one period and its dimension is flagged.
inline int wrap3(double v[3], const double w[3]) {
  int iw = 0;
  for (int i = 0; i < 3; i++) {
    if (v[i] < -w[i] / 2) {
      v[i] += w[i];
      iw |= 1 << i;
    }
    if (v[i] > w[i] / 2) {
      v[i] -= w[i];
      iw |= 1 << i;
    }
  }
  return iw;
}
inline void unwrap3(double v[3], const double w[3], int iw) {
  for (int i = 0; i < 3; i++)
    if ((iw >> i) & 1) v[i] += (v[i] > 0 ? -w[i] : w[i]);
}

// Partition::octsection with one rank (include/partition.h:185-207): Xmin
// stays, Xmax becomes Xmin + 1 * ((Xmax - Xmin) / 1), which can differ from
// Xmax in its last bit.
inline void octsection_one_rank(const double g[6], double local[6]) {
  for (int d = 0; d < 3; d++) {
    const double part = (g[3 + d] - g[d]) / 1;
    local[d] = g[d] + 0 * part;
    local[3 + d] = g[d] + (0 + 1) * part;
  }
}

// Throws with the context's error text when an engine call fails.
inline void check(exafmm_ctx *ctx, int rc, const char *what) {
  if (rc == 0) return;
  std::string m = what;
  if (ctx) m += std::string(": ") + exafmm_last_error(ctx);
  throw std::runtime_error(m);
}

template <typename F>
void guarded(std::string &err, const char *name, F &&f) {
  try {
    err.clear();
    f();
  } catch (const std::exception &e) {
    err = std::string(name) + ": " + e.what();
    std::fprintf(stderr, "exafmm %s\n", err.c_str());
  }
}

}  // namespace exafmm_md
#endif
