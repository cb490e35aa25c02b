// Per-order expansion tables, built once per (device, P) and kept resident.
// The reference keeps its tables inside Kernel (kernels/laplace.h:116-148) and
// scales A_n^m by 1/EPS; the scaling cancels in every product it enters, so
// the tables here are the unscaled values.
#include <math.h>

#include <algorithm>
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
  // M2M and L2L term lists, in the order the terms are summed (n, then m)
  auto aidx = [&](int n, int m) { return tri(n) + (m < 0 ? -m : m); };
  std::vector<TransOp> m2m, l2l;
  std::vector<int> m2m_start, l2l_start;
  for (int j = 0; j < P; j++) {
    for (int k = 0; k <= j; k++) {
      m2m_start.push_back((int)m2m.size());
      const double ajk = anm[tri(j) + k];
      for (int n = 0; n <= j; n++) {
        for (int m = -n; m <= n; m++) {
          const int km = k - m;
          if (km > j - n || -km > j - n) continue;
          const double w = anm[aidx(n, m)] * anm[aidx(j - n, km)] / ajk;
          TransOp op;
          op.b = aidx(n, m) | ((m < 0 ? 1 : 0) << 16);
          if (m < k) {
            const double ph = (m < 0 && (m & 1)) ? -1.0 : 1.0;
            op.a = tri(j - n) + km;
            op.w = ph * ((n & 1) ? -1.0 : 1.0) * w;
          } else {
            op.a = (tri(j - n) - km) | (1 << 16);
            op.w = (((k + n + m) & 1) ? -1.0 : 1.0) * w;
          }
          m2m.push_back(op);
        }
      }
      l2l_start.push_back((int)l2l.size());
      for (int n = j; n < P; n++) {
        for (int m = -n; m <= n; m++) {
          const int mk = m - k;
          if (mk > n - j || -mk > n - j) continue;
          const double w = anm[aidx(n - j, mk)] * ajk / anm[aidx(n, m)];
          TransOp op;
          op.b = aidx(n - j, mk) | ((mk < 0 ? 1 : 0) << 16);
          if (m < 0) {
            op.a = (tri(n) - m) | (1 << 16);
            op.w = ((k & 1) ? -1.0 : 1.0) * w;
          } else {
            const double ph = (mk < 0 && (mk & 1)) ? -1.0 : 1.0;
            op.a = tri(n) + m;
            op.w = ph * w;
          }
          l2l.push_back(op);
        }
      }
    }
  }
  m2m_start.push_back((int)m2m.size());
  l2l_start.push_back((int)l2l.size());
  std::vector<double> gz(tri(P) + 1, 0.0), s1(tri(P) + 1, 0.0), s2(tri(P) + 1, 0.0);
  for (int n = 0; n + 1 < P; n++) {
    for (int m = 0; m <= n; m++) {
      const int o = tri(n) + m;
      const double wm = (m == 0) ? 1.0 : 2.0;
      gz[o] = wm * sqrt((double)((n + 1) * (n + 1) - m * m));
      s1[o] = sqrt(0.5 * (double)((n + m + 2) * (n + m + 1)));
      if (m == 1) s2[o] = -sqrt(0.5 * (double)((n + 1) * n));
      else if (m >= 2) s2[o] = -sqrt(0.5 * (double)((n + 2 - m) * (n + 1 - m)));
    }
  }
  auto upload_raw = [&](const void *src, size_t bytes) {
    void *p = nullptr;
    EXA_CUDA(cudaMalloc(&p, bytes ? bytes : 1));
    if (bytes) EXA_CUDA(cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice));
    g_allocs.push_back(p);
    return p;
  };
  DevTables t;
  t.P = P;
  t.nterm = tri(P);
  t.m2m_ops = (const TransOp *)upload_raw(m2m.data(), m2m.size() * sizeof(TransOp));
  t.m2m_start = (const int *)upload_raw(m2m_start.data(), m2m_start.size() * sizeof(int));
  t.l2l_ops = (const TransOp *)upload_raw(l2l.data(), l2l.size() * sizeof(TransOp));
  t.l2l_start = (const int *)upload_raw(l2l_start.data(), l2l_start.size() * sizeof(int));
  // Balanced lane assignment of the output coefficients (see DevTables).
  auto balance = [&](const std::vector<int> &start) {
    const int NT = tri(P), MO = (NT + 31) / 32;
    std::vector<int> order(NT);
    for (int o = 0; o < NT; o++) order[o] = o;
    auto cost = [&](int o) { return start[o + 1] - start[o]; };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    std::vector<long long> load(32, 0);
    std::vector<int> used(32, 0);
    std::vector<short> out((size_t)32 * MO, (short)-1);
    for (int o : order) {
      int best = -1;
      for (int l = 0; l < 32; l++)
        if (used[l] < MO && (best < 0 || load[l] < load[best])) best = l;
      out[(size_t)best * MO + used[best]] = (short)o;
      used[best]++;
      load[best] += cost(o) + 1;
    }
    return out;
  };
  const std::vector<short> m2m_lane = balance(m2m_start), l2l_lane = balance(l2l_start);
  t.m2m_lane = (const short *)upload_raw(m2m_lane.data(), m2m_lane.size() * sizeof(short));
  t.l2l_lane = (const short *)upload_raw(l2l_lane.data(), l2l_lane.size() * sizeof(short));
  t.l2p_gz = upload(gz);
  t.l2p_s1 = upload(s1);
  t.l2p_s2 = upload(s2);
  t.anm = upload(anm);
  t.ainv = upload(ainv);
  t.ra = upload(ra);
  t.rb = upload(rb);
  t.rd = upload(rd);
  auto res = g_tables.emplace(key, t);
  return res.first->second;
}

}  // namespace exafmm_b200
