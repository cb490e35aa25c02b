// Records of a solve in the reference's file formats (host code):
//  * Traversal::writeList (include/traversal.h:412-421): one line per cell, in
//    cell order, "<ICELL left-aligned in 20> <P2P list size> <M2L list size>",
//    into path + "list%06d.dat"; ICELL is BuildTree::getKey of the cell center
//    (include/build_tree.h:111-120, 132);
//  * logger::writeTime (include/logger.h:116-127): one line per timer event in
//    name order, "<name left-aligned in 20> <seconds>" with the stream's default
//    six significant digits, into path + "time%06d.dat".
#include <cstdio>
#include <stdexcept>
#include <string>

#include "records.h"

namespace exafmm_b200 {

// getKey evaluated as the compiled reference evaluates it: its shifts are of
// 32-bit ints, so shift counts of 32 and more wrap modulo 32 (x86 shl), the
// level offset (2^(3 level) - 1) / 7 wraps with them, and a bit landing in
// position 31 sign-extends into the 64-bit key.  Below level 11 this is the
// plain Morton key with its level offset.
unsigned long long morton_key(const double X[3], const double Xmin[3], double diameter, int level) {
  int iX[3];
  for (int d = 0; d < 3; d++) iX[d] = (int)((X[d] - Xmin[d]) / diameter);
  const int base = (int)((1u << ((3 * level) & 31)) - 1u);
  unsigned long long index = (unsigned long long)(long long)(base / 7);
  for (int l = 0; l < level; l++) {
    for (int d = 0; d < 3; d++) {
      const int bit = (int)((unsigned)(iX[d] & 1) << ((3 * l + d) & 31));
      index += (unsigned long long)(long long)bit;
    }
    for (int d = 0; d < 3; d++) iX[d] >>= 1;
  }
  return index;
}

static std::string record_name(const char *path, const char *stem, int rank) {
  char num[32];
  std::snprintf(num, sizeof(num), "%06d", rank);
  return std::string(path ? path : "./") + stem + num + ".dat";
}

void write_list_file(const char *path, int rank, long long ncells, const unsigned long long *icell,
                     const int *p2p_off, const int *m2l_off) {
  const std::string name = record_name(path, "list", rank);
  FILE *f = std::fopen(name.c_str(), "w");
  if (!f) throw std::runtime_error("cannot open " + name);
  for (long long c = 0; c < ncells; c++)
    std::fprintf(f, "%-20llu %d %d\n", icell[c], p2p_off[c + 1] - p2p_off[c], m2l_off[c + 1] - m2l_off[c]);
  if (std::fclose(f) != 0) throw std::runtime_error("cannot write " + name);
}

void write_time_file(const char *path, int rank, const std::map<std::string, double> &timer) {
  const std::string name = record_name(path, "time", rank);
  FILE *f = std::fopen(name.c_str(), "w");
  if (!f) throw std::runtime_error("cannot open " + name);
  for (const auto &e : timer) std::fprintf(f, "%-20s %g\n", e.first.c_str(), e.second);
  if (std::fclose(f) != 0) throw std::runtime_error("cannot write " + name);
}

}  // namespace exafmm_b200

using namespace exafmm_b200;

extern "C" {

unsigned long long exafmm_morton_key(const double *X, const double *Xmin, double diameter, int level) {
  return morton_key(X, Xmin, diameter, level);
}

int exafmm_write_time_events(const char *path, int rank, int count, const char *const *names,
                             const double *seconds) {
  try {
    if (count < 0 || (count > 0 && (!names || !seconds))) throw std::runtime_error("bad event arrays");
    std::map<std::string, double> timer;
    for (int i = 0; i < count; i++) timer[names[i]] += seconds[i];
    write_time_file(path, rank, timer);
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

}  // extern "C"
