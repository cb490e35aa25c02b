// Solve records in the reference's file formats (records.cu).
#pragma once
#include <map>
#include <string>

namespace exafmm_b200 {

// BuildTree::getKey (include/build_tree.h:111-120) as the compiled reference evaluates it.
unsigned long long morton_key(const double X[3], const double Xmin[3], double diameter, int level);

// Traversal::writeList: path + "list%06d.dat", one line per cell; offsets are ncells + 1 CSR offsets.
void write_list_file(const char *path, int rank, long long ncells, const unsigned long long *icell,
                     const int *p2p_off, const int *m2l_off);

// logger::writeTime: path + "time%06d.dat", one line per event in name order (seconds).
void write_time_file(const char *path, int rank, const std::map<std::string, double> &timer);

}  // namespace exafmm_b200
