// Per-order expansion tables, built once per (device, P) and kept resident.
// The reference keeps its tables inside Kernel (kernels/laplace.h:116-148) and
// scales A_n^m by 1/EPS; the scaling cancels in every product it enters, so
// the tables here are the unscaled values.
#include <math.h>

#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "harmonics.cuh"

namespace exafmm_b200 {

namespace {
std::mutex g_mutex;
std::map<std::pair<int, int>, DevTables> g_tables;
std::vector<void *> g_allocs;

double factorial(int k) {
  double f = 1.0;
  for (int i = 2; i <= k; i++) f *= i;
  return f;
}
}  // namespace

const DevTables &device_tables(int P) {
  int dev = 0;
  EXA_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_mutex);
  auto key = std::make_pair(dev, P);
  auto it = g_tables.find(key);
  if (it != g_tables.end()) return it->second;
  const int Q = 2 * P + 2;
  const int T = tri(Q) + 1;
  std::vector<double> anm(T, 0.0), ainv(T, 0.0), ra(T, 0.0), rb(T, 0.0), rd(Q + 1, 1.0);
  for (int n = 0; n < Q; n++) {
    for (int m = 0; m <= n; m++) {
      const int o = tri(n) + m;
      anm[o] = ((n & 1) ? -1.0 : 1.0) / sqrt(factorial(n - m) * factorial(n + m));
      ainv[o] = 1.0 / anm[o];
      const double den = double(n + 1) * double(n + 1) - double(m) * double(m);
      ra[o] = (2.0 * n + 1.0) / sqrt(den);
      rb[o] = sqrt((double(n) * n - double(m) * m) / den);
    }
  }
  for (int m = 1; m <= Q; m++) rd[m] = sqrt((2.0 * m - 1.0) / (2.0 * m));
  auto upload = [&](const std::vector<double> &v) {
    void *p = nullptr;
    EXA_CUDA(cudaMalloc(&p, v.size() * sizeof(double)));
    EXA_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
    g_allocs.push_back(p);
    return (const double *)p;
  };
  DevTables t;
  t.P = P;
  t.nterm = tri(P);
  t.anm = upload(anm);
  t.ainv = upload(ainv);
  t.ra = upload(ra);
  t.rb = upload(rb);
  t.rd = upload(rd);
  auto res = g_tables.emplace(key, t);
  return res.first->second;
}

}  // namespace exafmm_b200
