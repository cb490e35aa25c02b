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
  // Pieces of the translation terms and their lanes (see DevTables).
  struct Split {
    std::vector<int4> piece;
    std::vector<int> piece_start;
    std::vector<short> slot;
    int slots = 0;
  };
  auto split = [&](const std::vector<int> &start) {
    const int NT = tri(P);
    const int total = start[NT] - start[0];
    const int cap = std::max(1, (total + 31) / 32);  // about the lanes' average share
    Split s;
    for (int o = 0; o < NT; o++) {
      s.piece_start.push_back((int)s.piece.size());
      const int b = start[o], n = start[o + 1] - start[o];
      const int k = std::max(1, (n + cap - 1) / cap);
      for (int q = 0; q < k; q++) s.piece.push_back(make_int4(o, b + n * q / k, b + n * (q + 1) / k, 0));
    }
    s.piece_start.push_back((int)s.piece.size());
    const int np = (int)s.piece.size();
    s.slots = (np + 31) / 32;
    std::vector<int> order(np);
    for (int q = 0; q < np; q++) order[q] = q;
    auto len = [&](int q) { return s.piece[q].z - s.piece[q].y; };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return len(a) > len(b); });
    std::vector<long long> load(32, 0);
    std::vector<int> used(32, 0);
    s.slot.assign((size_t)32 * s.slots, (short)-1);
    for (int q : order) {
      int best = -1;
      for (int l = 0; l < 32; l++)
        if (used[l] < s.slots && (best < 0 || load[l] < load[best])) best = l;
      s.slot[(size_t)best * s.slots + used[best]] = (short)q;
      used[best]++;
      load[best] += len(q) + 1;
    }
    return s;
  };
  // M2M's lanes: whole output coefficients, longest first to the least loaded
  // lane (cutting them into pieces measured slower at P = 10).
  {
    const int NT = tri(P), MO = (NT + 31) / 32;
    std::vector<int> order(NT);
    for (int o = 0; o < NT; o++) order[o] = o;
    auto cost = [&](int o) { return m2m_start[o + 1] - m2m_start[o]; };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    std::vector<long long> load(32, 0);
    std::vector<int> used(32, 0);
    std::vector<short> lane_out((size_t)32 * MO, (short)-1);
    for (int o : order) {
      int best = -1;
      for (int l = 0; l < 32; l++)
        if (used[l] < MO && (best < 0 || load[l] < load[best])) best = l;
      lane_out[(size_t)best * MO + used[best]] = (short)o;
      used[best]++;
      load[best] += cost(o) + 1;
    }
    t.m2m_lane = (const short *)upload_raw(lane_out.data(), lane_out.size() * sizeof(short));
  }
  const Split sl = split(l2l_start);
  t.l2l_piece = (const int4 *)upload_raw(sl.piece.data(), sl.piece.size() * sizeof(int4));
  t.l2l_piece_start = (const int *)upload_raw(sl.piece_start.data(), sl.piece_start.size() * sizeof(int));
  t.l2l_slot = (const short *)upload_raw(sl.slot.data(), sl.slot.size() * sizeof(short));
  t.l2l_slots = sl.slots;
  t.l2l_pieces = (int)sl.piece.size();
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
