// Host runtime over the solve contexts: a batch solver for many independent
// systems and a request server with HBM-budget admission.
//
// Both keep a pool of workers; each worker is a host thread that owns one
// solve context (its own CUDA stream and buffers), so independent systems run
// concurrently on the GPU while each one's launches stay ordered.  A system's
// result depends only on its own bodies and parameters: every kernel of a
// solve reduces in a fixed order, so a system gives the same bits alone, in a
// batch, or beside other requests.
//
// The reference has no counterpart: it solves one system per process
// (examples/fmm.cxx:163-179) and leaves concurrency to the caller.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/exafmm_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// ---------------------------------------------------------------- ncrit autotuner
// Per size class (floor(log2 n)) the candidates are tried in turn on the first
// systems of that class; the one with the lowest device time per body is kept.
class NcritTuner {
 public:
  explicit NcritTuner(std::vector<int> cand) : cand_(std::move(cand)) {}

  // New candidates start the tuning over (the table found so far is kept
  // until a class has tried them all).
  void set_candidates(std::vector<int> cand) {
    std::lock_guard<std::mutex> lk(mu_);
    cand_ = std::move(cand);
    cls_.clear();
  }

  int pick(long long n, int fallback) { return pick_class(size_class(n), fallback); }

  void report(long long n, int ncrit, double ms) {
    if (n > 0) report_class(size_class(n), ncrit, ms / (double)n);
  }

  // The same keyed by a class directly (a forest bucket is keyed by the
  // lowest size class it holds), with the cost already per body.
  int pick_class(int cls, int fallback) {
    std::lock_guard<std::mutex> lk(mu_);
    if (!enabled_) {
      auto it = best_.find(cls);
      return it == best_.end() ? fallback : it->second;
    }
    Class &c = cls_[cls];
    if (c.trials.size() < cand_.size()) return cand_[c.trials.size()];
    return best_of(c);
  }

  void report_class(int cls, int ncrit, double ms_per_body) {
    std::lock_guard<std::mutex> lk(mu_);
    if (!enabled_) return;
    Class &c = cls_[cls];
    if (c.trials.size() < cand_.size() && ncrit == cand_[c.trials.size()]) c.trials.push_back(ms_per_body);
    if (c.trials.size() == cand_.size()) best_[cls] = best_of(c);
  }

  static int size_class(long long n) { return n <= 1 ? 0 : (int)std::floor(std::log2((double)n)); }

  void enable(bool on) {
    std::lock_guard<std::mutex> lk(mu_);
    enabled_ = on;
  }

  void load(const int *pairs, int k) {
    std::lock_guard<std::mutex> lk(mu_);
    enabled_ = false;
    best_.clear();
    for (int i = 0; i < k; i++) best_[pairs[2 * i]] = pairs[2 * i + 1];
  }

  // class -> chosen ncrit, as pairs
  std::vector<int> table() {
    std::lock_guard<std::mutex> lk(mu_);
    std::vector<int> out;
    for (auto &kv : best_) {
      out.push_back(kv.first);
      out.push_back(kv.second);
    }
    return out;
  }

 private:
  struct Class {
    std::vector<double> trials;  // ms per body, in candidate order
  };
  int best_of(const Class &c) const {
    size_t b = 0;
    for (size_t i = 1; i < c.trials.size(); i++)
      if (c.trials[i] < c.trials[b]) b = i;
    return cand_[b];
  }
  std::vector<int> cand_;
  std::mutex mu_;
  bool enabled_ = false;
  std::map<int, Class> cls_;
  std::map<int, int> best_;
};

struct SolveParams {
  int P = 10;
  double theta = 0.4;
  int ncrit = 64;
  int nspawn = 5000;
  int images = 0;
  double cycle = 6.283185307179586;
  int precision = EXAFMM_FP64;
  int p2p_tpl = 0;  // exafmm_set_p2p_targets_per_lane
};

// A tuned configuration packed in one int: ncrit and the P2P targets per lane.
inline int pack_config(int ncrit, int tpl) { return ncrit * 4 + (tpl == 2 ? 1 : tpl == 3 ? 2 : 0); }
inline int config_ncrit(int cfg) { return cfg / 4; }
inline int config_tpl(int cfg) { return cfg % 4 == 1 ? 2 : cfg % 4 == 2 ? 3 : 0; }

// exafmm_set_mixed_policy's arguments, applied to every context a batch uses.
struct MixedPolicy {
  bool set = false;
  int m2l_fp32 = 1, p2p_fp32 = 1, min_level = 2, max_dl = 3;
};

// One worker's context, created on first use and re-parameterized per system.
struct Slot {
  exafmm_ctx *ctx = nullptr;
  SolveParams cur;
  ~Slot() { release(); }
  void release() {
    if (ctx) exafmm_destroy(ctx);
    ctx = nullptr;
  }
  long long bytes() const {
    long long b = 0;
    if (ctx) exafmm_device_bytes(ctx, &b);
    return b;
  }
  // Solve one system; returns the device time of the solve (ms).
  double solve(int device, const SolveParams &p, const double *xyzq, long long n, double *trg,
               const MixedPolicy *pol = nullptr) {
    prepare(device, p, pol);
    check(exafmm_set_bodies(ctx, xyzq, n));
    check(exafmm_solve(ctx));
    check(exafmm_get_results(ctx, trg));
    double ms[8];
    check(exafmm_phase_times(ctx, ms));
    return ms[7];
  }

  // Solve count systems as one forest (exafmm_set_systems_list): the
  // context's stream first waits for `start`, and `done` is recorded on it
  // after the results are copied out.  Returns the forest's solve time (ms).
  double solve_forest(int device, const SolveParams &p, const MixedPolicy *pol, int count, const long long *n,
                      const double *const *xyzq, double *const *trg, cudaEvent_t start, cudaEvent_t done) {
    prepare(device, p, pol);
    cudaStream_t st = (cudaStream_t)exafmm_stream(ctx);
    if (start && cudaStreamWaitEvent(st, start, 0) != cudaSuccess) throw std::runtime_error("cudaStreamWaitEvent");
    check(exafmm_set_systems_list(ctx, count, n, xyzq));
    check(exafmm_solve(ctx));
    check(exafmm_get_results_list(ctx, trg));
    if (done && cudaEventRecord(done, st) != cudaSuccess) throw std::runtime_error("cudaEventRecord");
    double ms[8];
    check(exafmm_phase_times(ctx, ms));
    return ms[7];
  }

  void prepare(int device, const SolveParams &p, const MixedPolicy *pol) {
    if (!ctx || p.precision != cur.precision) {
      release();
      if (exafmm_create(&ctx, p.P, p.theta, p.ncrit, p.nspawn, p.images, p.cycle, p.precision, device) != 0) {
        ctx = nullptr;
        throw std::runtime_error(exafmm_create_error());
      }
      cur = p;
      ctx_tpl = 0;
    } else if (p.P != cur.P || p.theta != cur.theta || p.ncrit != cur.ncrit || p.nspawn != cur.nspawn ||
               p.images != cur.images || p.cycle != cur.cycle) {
      check(exafmm_set_params(ctx, p.P, p.theta, p.ncrit, p.nspawn, p.images, p.cycle));
      cur = p;
    }
    if (pol && pol->set && p.precision == EXAFMM_MIXED)
      check(exafmm_set_mixed_policy(ctx, pol->m2l_fp32, pol->p2p_fp32, pol->min_level, pol->max_dl));
    if (p.p2p_tpl != ctx_tpl) {
      check(exafmm_set_p2p_targets_per_lane(ctx, p.p2p_tpl));
      ctx_tpl = p.p2p_tpl;
    }
  }
  int ctx_tpl = 0;  // the context's P2P targets per lane
  void check(int rc) {
    if (rc != 0) throw std::runtime_error(exafmm_last_error(ctx));
  }
};

}  // namespace

// ================================================================ batch
struct exafmm_batch {
  int device = 0;
  int workers = 1;
  SolveParams prm;
  MixedPolicy policy;
  int forest_buckets = 0;       // 0: one context per system; k > 0: up to k forests by size
  std::vector<Slot> slots;
  // the autotuner's candidates: every ncrit with every P2P targets-per-lane
  // setting, packed (pack_config); the table maps a size class to one of them
  std::vector<int> ncrit_cands{32, 64, 128}, tpl_cands{0};
  NcritTuner tuner{{pack_config(32, 0), pack_config(64, 0), pack_config(128, 0)}};
  void retune() {
    std::vector<int> c;
    for (int t : tpl_cands)
      for (int n : ncrit_cands) c.push_back(pack_config(n, t));
    tuner.set_candidates(c);
  }
  std::vector<double> last_ms;  // per system of the last call, device ms
  double last_elapsed_ms = 0;   // the last forest call, first copy in to last copy out, on the device
  std::vector<int> last_bucket; // bucket of each system in the last forest call
  std::vector<int> last_bucket_ncrit, last_bucket_tpl;
  cudaStream_t timing = nullptr;
  cudaEvent_t ev_start = nullptr, ev_end = nullptr;
  std::vector<cudaEvent_t> ev_done;
  std::string error;
  ~exafmm_batch() {
    slots.clear();
    for (auto e : ev_done) cudaEventDestroy(e);
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_end) cudaEventDestroy(ev_end);
    if (timing) cudaStreamDestroy(timing);
  }
};

namespace {

// Forest buckets: the non-empty systems' size classes (floor(log2 n)) in
// increasing order, cut into at most `buckets` runs of whole classes with
// about equal bodies each (bucket b's share ends at (b + 1) / buckets of all
// bodies); empty systems join the first bucket.  Returns the
// number of buckets and fills bucket_of[count] and, if given, the lowest class
// of each bucket (its tuner key).
int forest_buckets(int count, const long long *n, int buckets, int *bucket_of, std::vector<int> *key) {
  std::map<int, long long> per_class;
  long long total = 0;
  for (int i = 0; i < count; i++)
    if (n[i] > 0) {
      per_class[NcritTuner::size_class(n[i])] += n[i];
      total += n[i];
    }
  std::map<int, int> class_bucket;
  std::vector<int> lowest;
  int b = 0;
  long long acc = 0;
  for (auto &kv : per_class) {
    // start the next bucket before this class when taking it would overshoot
    // the current bucket's share by more than stopping here falls short of it
    const double target = (double)total * (b + 1) / buckets;
    if ((int)lowest.size() == b + 1 && b < buckets - 1 &&
        (double)(acc + kv.second) - target > target - (double)acc)
      b++;
    if ((int)lowest.size() == b) lowest.push_back(kv.first);
    class_bucket[kv.first] = b;
    acc += kv.second;
  }
  if (lowest.empty()) lowest.push_back(0);
  const int nb = (int)lowest.size();
  for (int i = 0; i < count; i++) bucket_of[i] = n[i] > 0 ? class_bucket[NcritTuner::size_class(n[i])] : 0;
  if (key) *key = lowest;
  return nb;
}

}  // namespace

// ================================================================ server
namespace {

// A repeat chain kept on the device: one context holds the chain's bodies,
// tree and expansions between steps; each step after the first moves the
// bodies in place on the device (or takes new positions from device memory)
// and solves again, so no step uploads bodies from the host.
struct Session {
  long long id = 0;
  SolveParams prm;
  const double *xyzq0 = nullptr;  // the first step's bodies (host)
  long long n = 0;
  exafmm_ctx *ctx = nullptr;
  long long held = 0;             // the context's device bytes while no step runs
  bool busy = false;              // a step is queued or running
  int steps = 0;                  // steps completed
  ~Session() {
    if (ctx) exafmm_destroy(ctx);
  }
};

struct Request {
  long long id = 0;
  SolveParams prm;
  const double *xyzq = nullptr;
  long long n = 0;
  double *trg = nullptr;
  Session *sess = nullptr;        // a chain step (prm and n are the session's)
  double sigma = 0;
  unsigned long long seed = 0;
  const double *d_xyzq = nullptr; // a chain step's new positions in device memory (or null)
  long long est_bytes = 0;   // estimate at submission, then the bytes charged while in flight
  Clock::time_point t_submit, t_start, t_end;
  double device_ms = 0;
  bool done = false;
  int status = 0;
  std::string err;
};

thread_local std::string g_server_error;

}  // namespace

struct exafmm_server {
  int device = 0;
  int workers = 1;
  double budget = 0;
  MixedPolicy policy;              // for the mixed-precision requests
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request *> queue;
  std::unordered_map<long long, std::unique_ptr<Request>> reqs;
  std::vector<Slot> slots;
  std::vector<long long> held;     // device bytes held by each worker's idle context
  std::unordered_map<long long, std::unique_ptr<Session>> sessions;
  long long session_held = 0;      // device bytes held by sessions between steps
  long long next_session = 1;
  long long in_flight = 0;         // bytes charged to the requests being solved
  int running = 0;                 // requests being solved
  long long peak_admitted = 0;
  long long next_id = 1, completed = 0;
  // continuous batching: queued requests of at most group_max_n bodies with
  // the same parameters are solved together as one forest, up to group_max
  // requests and group_bodies bodies (group_max <= 1: one request per solve)
  int group_max = 64;
  long long group_max_n = 262144;
  long long group_bodies = 4LL << 20;
  long long grouped = 0;           // requests solved inside a group of two or more
  bool stop = false;
  std::vector<std::thread> threads;

  // Upper estimate of a solve's device bytes: per body the bodies, keys,
  // permutation, results and two-float copies, the cells' expansions and the
  // interaction lists at their initial capacities; plus a fixed part.  A
  // worker's context keeps its buffers, so a request is charged the larger of
  // this and what that context already holds.
  static long long estimate(long long n, int P) {
    const long long nt = (long long)P * (P + 1) / 2;
    return n * (1400 + 24 * nt) + (64LL << 20);
  }

  long long held_total(int except) const {
    long long s = session_held;
    for (int w = 0; w < (int)held.size(); w++)
      if (w != except) s += held[w];
    return s;
  }

  // What a request brings onto the device: a chain step its session's context
  // (which it then no longer holds idle), any other request the estimate or
  // the worker context it will use.
  long long charge_of(const Request *r, int w) const {
    return r->sess ? std::max(r->est_bytes, r->sess->held) : std::max(r->est_bytes, held[w]);
  }

  // Head-of-line admission: the request fits beside what the other workers
  // and the idle sessions hold and what is in flight; with nothing in flight
  // it is always admitted, so a request larger than the budget still runs
  // (alone).
  bool admissible(const Request *r, int w) const {
    if (running == 0) return true;
    const long long others = held_total(w) - (r->sess ? r->sess->held : 0) + (r->sess ? held[w] : 0);
    return (double)(others + in_flight + charge_of(r, w)) <= budget;
  }

  // One chain step on the session's own context.
  double run_step(Request *r) {
    Session *q = r->sess;
    auto check = [&](int rc) {
      if (rc != 0) throw std::runtime_error(exafmm_last_error(q->ctx));
    };
    if (!q->ctx) {
      if (exafmm_create(&q->ctx, q->prm.P, q->prm.theta, q->prm.ncrit, q->prm.nspawn, q->prm.images, q->prm.cycle,
                        q->prm.precision, device) != 0) {
        q->ctx = nullptr;
        throw std::runtime_error(exafmm_create_error());
      }
      if (policy.set && q->prm.precision == EXAFMM_MIXED)
        check(exafmm_set_mixed_policy(q->ctx, policy.m2l_fp32, policy.p2p_fp32, policy.min_level, policy.max_dl));
    }
    if (q->steps == 0) check(exafmm_set_bodies(q->ctx, q->xyzq0, q->n));
    else if (r->d_xyzq) check(exafmm_set_bodies_device(q->ctx, r->d_xyzq, q->n));
    else check(exafmm_displace_bodies(q->ctx, r->sigma, r->seed));
    check(exafmm_solve(q->ctx));
    check(exafmm_get_results(q->ctx, r->trg));
    double ms[8];
    check(exafmm_phase_times(q->ctx, ms));
    return ms[7];
  }

  void worker(int w) {
    cudaSetDevice(device);
    std::vector<Request *> grp;
    for (;;) {
      Request *r = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return (stop && queue.empty()) || (!queue.empty() && admissible(queue.front(), w)); });
        if (queue.empty()) return;
        r = queue.front();
        queue.pop_front();
        grp.assign(1, r);
        long long charge = charge_of(r, w);
        if (!r->sess && group_max > 1 && r->n <= group_max_n) {
          // the queued requests that can share this solve, in queue order,
          // each joining only if the group still fits the budget (the head
          // request alone is admitted as before)
          long long bodies = r->n, est = r->est_bytes;
          for (auto it = queue.begin(); it != queue.end() && (int)grp.size() < group_max;) {
            Request *q = *it;
            const long long est2 = est + q->est_bytes;
            const long long charge2 = std::max(est2, held[w]);
            if (!q->sess && q->n <= group_max_n && bodies + q->n <= group_bodies && same_params(q->prm, r->prm) &&
                (double)(held_total(w) + in_flight + charge2) <= budget) {
              grp.push_back(q);
              bodies += q->n;
              est = est2;
              charge = charge2;
              it = queue.erase(it);
            } else {
              ++it;
            }
          }
        }
        in_flight += charge;
        running++;
        if (r->sess) {
          session_held -= r->sess->held;
          r->sess->held = 0;
        } else {
          held[w] = 0;
        }
        peak_admitted = std::max(peak_admitted, in_flight + held_total(w) + held[w]);
        r->est_bytes = charge;  // what is charged while the solve runs (the group's, on its first request)
        const auto t = Clock::now();
        for (Request *q : grp) q->t_start = t;
        if (grp.size() > 1) grouped += (long long)grp.size();
      }
      int status = 0;
      std::string err;
      double dev_ms = 0;
      try {
        if (r->sess) {
          dev_ms = run_step(r);
        } else if (grp.size() == 1) {
          dev_ms = slots[w].solve(device, r->prm, r->xyzq, r->n, r->trg, &policy);
        } else {
          std::vector<long long> nn(grp.size());
          std::vector<const double *> in(grp.size());
          std::vector<double *> out(grp.size());
          for (size_t j = 0; j < grp.size(); j++) {
            nn[j] = grp[j]->n;
            in[j] = grp[j]->xyzq;
            out[j] = grp[j]->trg;
          }
          dev_ms = slots[w].solve_forest(device, r->prm, &policy, (int)grp.size(), nn.data(), in.data(), out.data(),
                                         nullptr, nullptr);
        }
      } catch (const std::exception &e) {
        status = 1;
        err = e.what();
        if (r->sess) {
          if (r->sess->ctx) exafmm_destroy(r->sess->ctx);
          r->sess->ctx = nullptr;
        } else {
          slots[w].release();
        }
      }
      long long sess_bytes = 0;
      if (r->sess && r->sess->ctx) exafmm_device_bytes(r->sess->ctx, &sess_bytes);
      const long long now_held = r->sess ? 0 : slots[w].bytes();
      bool release = false;
      {
        std::lock_guard<std::mutex> lk(mu);
        in_flight -= r->est_bytes;
        running--;
        if (r->sess) {
          r->sess->held = sess_bytes;
          session_held += sess_bytes;
          if (status == 0) r->sess->steps++;
          r->sess->busy = false;
        } else {
          // keep the context for reuse unless idle contexts crowd the budget
          release = (double)(held_total(w) + now_held) > 0.5 * budget;
          held[w] = release ? 0 : now_held;
        }
      }
      if (release) slots[w].release();
      {
        std::lock_guard<std::mutex> lk(mu);
        const auto t = Clock::now();
        long long bodies = 0;
        for (Request *q : grp) bodies += q->n;
        for (Request *q : grp) {
          q->t_end = t;
          // a group's device time is shared in proportion to the bodies
          q->device_ms = grp.size() == 1 ? dev_ms : (bodies > 0 ? dev_ms * (double)q->n / (double)bodies : 0.0);
          q->status = status;
          q->err = err;
          q->done = true;
          completed++;
        }
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }

  static bool same_params(const SolveParams &a, const SolveParams &b) {
    return a.P == b.P && a.theta == b.theta && a.ncrit == b.ncrit && a.nspawn == b.nspawn && a.images == b.images &&
           a.cycle == b.cycle && a.precision == b.precision;
  }
};

extern "C" {

// ---------------------------------------------------------------- batch entry points
int exafmm_batch_create(exafmm_batch **out, int P, double theta, int ncrit, int nspawn, int precision, int device,
                        int workers) {
  if (!out) return 2;
  *out = nullptr;
  if (workers < 1 || workers > 256 || P < 2 || ncrit < 1 || !(theta > 0)) return 2;
  if (precision != EXAFMM_FP64 && precision != EXAFMM_MIXED) return 2;
  int dev = device;
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return 1;
  auto *b = new exafmm_batch;
  b->device = dev;
  b->workers = workers;
  b->prm.P = P;
  b->prm.theta = theta;
  b->prm.ncrit = ncrit;
  b->prm.nspawn = nspawn;
  b->prm.precision = precision;
  b->slots.resize(workers);
  *out = b;
  return 0;
}

int exafmm_batch_destroy(exafmm_batch *b) {
  delete b;
  return 0;
}

const char *exafmm_batch_error(const exafmm_batch *b) { return b ? b->error.c_str() : "null batch"; }

int exafmm_batch_autotune(exafmm_batch *b, int enable) {
  if (!b) return 2;
  b->tuner.enable(enable != 0);
  return 0;
}

int exafmm_batch_ncrit_table(exafmm_batch *b, int *pairs, int cap) {
  if (!b) return -1;
  std::vector<int> t = b->tuner.table();
  const int k = (int)t.size() / 2;
  for (int i = 0; i < k && i < cap; i++) {
    pairs[2 * i] = t[2 * i];
    pairs[2 * i + 1] = config_ncrit(t[2 * i + 1]);
  }
  return k;
}

int exafmm_batch_set_ncrit_table(exafmm_batch *b, const int *pairs, int k) {
  if (!b || k < 0 || (k > 0 && !pairs)) return 2;
  std::vector<int> packed(2 * (size_t)k);
  for (int i = 0; i < k; i++) {
    if (pairs[2 * i + 1] < 1 || pairs[2 * i + 1] > 1024) return 2;
    packed[2 * i] = pairs[2 * i];
    packed[2 * i + 1] = pack_config(pairs[2 * i + 1], 0);
  }
  b->tuner.load(packed.data(), k);
  return 0;
}

int exafmm_batch_config_table(exafmm_batch *b, int *triples, int cap) {
  if (!b) return -1;
  std::vector<int> t = b->tuner.table();
  const int k = (int)t.size() / 2;
  for (int i = 0; i < k && i < cap; i++) {
    triples[3 * i] = t[2 * i];
    triples[3 * i + 1] = config_ncrit(t[2 * i + 1]);
    triples[3 * i + 2] = config_tpl(t[2 * i + 1]);
  }
  return k;
}

int exafmm_batch_set_config_table(exafmm_batch *b, const int *triples, int k) {
  if (!b || k < 0 || (k > 0 && !triples)) return 2;
  std::vector<int> packed(2 * (size_t)k);
  for (int i = 0; i < k; i++) {
    const int nc = triples[3 * i + 1], tpl = triples[3 * i + 2];
    if (nc < 1 || nc > 1024 || (tpl != 0 && tpl != 2 && tpl != 3)) return 2;
    packed[2 * i] = triples[3 * i];
    packed[2 * i + 1] = pack_config(nc, tpl);
  }
  b->tuner.load(packed.data(), k);
  return 0;
}

int exafmm_batch_set_p2p_candidates(exafmm_batch *b, const int *tpl, int k) {
  if (!b || k < 1 || k > 3 || !tpl) return 2;
  for (int i = 0; i < k; i++)
    if (tpl[i] != 0 && tpl[i] != 2 && tpl[i] != 3) return 2;
  b->tpl_cands.assign(tpl, tpl + k);
  b->retune();
  return 0;
}

namespace {

// Forest mode: every bucket's systems are one forest on one worker context;
// buckets run concurrently, largest first.  The device time of the whole call
// spans from an event that every context stream waits on to the last bucket's
// copy out.
int batch_solve_forest(exafmm_batch *b, int count, const long long *n, const double *const *xyzq,
                       double *const *trg) {
  cudaSetDevice(b->device);
  std::vector<int> bucket(count);
  std::vector<int> key;
  const int nb = forest_buckets(count, n, b->forest_buckets, bucket.data(), &key);
  std::vector<std::vector<int>> members(nb);
  std::vector<long long> bodies(nb, 0);
  for (int i = 0; i < count; i++) {
    members[bucket[i]].push_back(i);
    bodies[bucket[i]] += n[i];
  }
  std::vector<int> order(nb);
  for (int i = 0; i < nb; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return bodies[x] > bodies[y]; });
  const int nw = std::min(b->workers, nb);
  if (!b->timing) {
    if (cudaStreamCreateWithFlags(&b->timing, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev_start) != cudaSuccess || cudaEventCreate(&b->ev_end) != cudaSuccess) {
      b->error = "timing stream or events";
      return 1;
    }
  }
  while ((int)b->ev_done.size() < nw) {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      b->error = "cudaEventCreate";
      return 1;
    }
    b->ev_done.push_back(e);
  }
  b->last_bucket = bucket;
  b->last_bucket_ncrit.assign(nb, b->prm.ncrit);
  b->last_bucket_tpl.assign(nb, 0);
  if (cudaEventRecord(b->ev_start, b->timing) != cudaSuccess) {
    b->error = "cudaEventRecord";
    return 1;
  }
  std::atomic<int> next{0};
  std::atomic<bool> failed{false};
  std::mutex emu;
  std::vector<char> used(nw, 0);
  auto run = [&](int w) {
    cudaSetDevice(b->device);
    for (;;) {
      const int i = next.fetch_add(1);
      if (i >= nb || failed.load()) return;
      const int k = order[i];
      const std::vector<int> &mem = members[k];
      std::vector<long long> nn(mem.size());
      std::vector<const double *> in(mem.size());
      std::vector<double *> out(mem.size());
      for (size_t j = 0; j < mem.size(); j++) {
        nn[j] = n[mem[j]];
        in[j] = xyzq[mem[j]];
        out[j] = trg[mem[j]];
      }
      SolveParams p = b->prm;
      const int cfg = b->tuner.pick_class(key[k], pack_config(b->prm.ncrit, 0));
      p.ncrit = config_ncrit(cfg);
      p.p2p_tpl = config_tpl(cfg);
      b->last_bucket_ncrit[k] = p.ncrit;
      b->last_bucket_tpl[k] = p.p2p_tpl;
      try {
        const double ms = b->slots[w].solve_forest(b->device, p, &b->policy, (int)mem.size(), nn.data(), in.data(),
                                                   out.data(), b->ev_start, b->ev_done[w]);
        used[w] = 1;
        for (size_t j = 0; j < mem.size(); j++)
          b->last_ms[mem[j]] = bodies[k] > 0 ? ms * (double)nn[j] / (double)bodies[k] : 0.0;
        if (bodies[k] > 0) b->tuner.report_class(key[k], cfg, ms / (double)bodies[k]);
      } catch (const std::exception &e) {
        std::lock_guard<std::mutex> lk(emu);
        if (!failed.exchange(true)) b->error = std::string("forest bucket ") + std::to_string(k) + ": " + e.what();
        b->slots[w].release();
        return;
      }
    }
  };
  std::vector<std::thread> th;
  for (int w = 1; w < nw; w++) th.emplace_back(run, w);
  run(0);
  for (auto &t : th) t.join();
  if (failed.load()) return 1;
  for (int w = 0; w < nw; w++)
    if (used[w] && cudaStreamWaitEvent(b->timing, b->ev_done[w], 0) != cudaSuccess) {
      b->error = "cudaStreamWaitEvent";
      return 1;
    }
  float ms = 0.f;
  if (cudaEventRecord(b->ev_end, b->timing) != cudaSuccess || cudaEventSynchronize(b->ev_end) != cudaSuccess ||
      cudaEventElapsedTime(&ms, b->ev_start, b->ev_end) != cudaSuccess) {
    b->error = "timing events";
    return 1;
  }
  b->last_elapsed_ms = ms;
  return 0;
}

}  // namespace

int exafmm_batch_solve(exafmm_batch *b, int count, const long long *n, const double *const *xyzq, double *const *trg) {
  if (!b) return 2;
  if (count < 0 || (count > 0 && (!n || !xyzq || !trg))) return 2;
  for (int i = 0; i < count; i++)
    if (n[i] < 0) return 2;
  b->error.clear();
  b->last_ms.assign(count, 0.0);
  if (b->forest_buckets > 0 && count > 0) return batch_solve_forest(b, count, n, xyzq, trg);
  std::vector<int> order(count);
  for (int i = 0; i < count; i++) order[i] = i;
  // largest first: the long solves start early and the short ones fill in
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return n[x] > n[y]; });
  std::atomic<int> next{0};
  std::atomic<bool> failed{false};
  std::mutex emu;
  auto run = [&](int w) {
    cudaSetDevice(b->device);
    for (;;) {
      const int i = next.fetch_add(1);
      if (i >= count || failed.load()) return;
      const int k = order[i];
      SolveParams p = b->prm;
      const int cfg = b->tuner.pick(n[k], pack_config(b->prm.ncrit, 0));
      p.ncrit = config_ncrit(cfg);
      p.p2p_tpl = config_tpl(cfg);
      try {
        const double ms = b->slots[w].solve(b->device, p, xyzq[k], n[k], trg[k], &b->policy);
        b->last_ms[k] = ms;
        b->tuner.report(n[k], cfg, ms);
      } catch (const std::exception &e) {
        std::lock_guard<std::mutex> lk(emu);
        if (!failed.exchange(true)) b->error = std::string("system ") + std::to_string(k) + ": " + e.what();
        b->slots[w].release();
        return;
      }
    }
  };
  const int nw = std::min(b->workers, std::max(count, 1));
  std::vector<std::thread> th;
  for (int w = 1; w < nw; w++) th.emplace_back(run, w);
  run(0);
  for (auto &t : th) t.join();
  return failed.load() ? 1 : 0;
}

int exafmm_batch_times(exafmm_batch *b, double *ms) {
  if (!b || !ms) return 2;
  std::copy(b->last_ms.begin(), b->last_ms.end(), ms);
  return 0;
}

int exafmm_batch_set_forest(exafmm_batch *b, int buckets) {
  if (!b || buckets < 0 || buckets > 64) return 2;
  b->forest_buckets = buckets;
  return 0;
}

int exafmm_batch_set_mixed_policy(exafmm_batch *b, int m2l_fp32, int p2p_fp32, int min_level, int max_dl) {
  if (!b || m2l_fp32 < 0 || m2l_fp32 > 5 || min_level < 0 || max_dl < 0) return 2;
  b->policy.set = true;
  b->policy.m2l_fp32 = m2l_fp32;
  b->policy.p2p_fp32 = p2p_fp32;
  b->policy.min_level = min_level;
  b->policy.max_dl = max_dl;
  return 0;
}

int exafmm_batch_set_ncrit_candidates(exafmm_batch *b, const int *ncrit, int k) {
  if (!b || k < 1 || k > 16 || !ncrit) return 2;
  for (int i = 0; i < k; i++)
    if (ncrit[i] < 1 || ncrit[i] > 1024) return 2;
  b->ncrit_cands.assign(ncrit, ncrit + k);
  b->retune();
  return 0;
}

int exafmm_batch_elapsed(exafmm_batch *b, double *ms) {
  if (!b || !ms) return 2;
  *ms = b->last_elapsed_ms;
  return 0;
}

int exafmm_batch_buckets(exafmm_batch *b, int *bucket_of, int *bucket_ncrit, int cap) {
  if (!b) return -1;
  const int nb = (int)b->last_bucket_ncrit.size();
  if (bucket_of) std::copy(b->last_bucket.begin(), b->last_bucket.end(), bucket_of);
  if (bucket_ncrit)
    for (int i = 0; i < nb && i < cap; i++) bucket_ncrit[i] = b->last_bucket_ncrit[i];
  return nb;
}

int exafmm_batch_bucket_p2p(exafmm_batch *b, int *bucket_tpl, int cap) {
  if (!b) return -1;
  const int nb = (int)b->last_bucket_tpl.size();
  if (bucket_tpl)
    for (int i = 0; i < nb && i < cap; i++) bucket_tpl[i] = b->last_bucket_tpl[i];
  return nb;
}

int exafmm_forest_buckets(int count, const long long *n, int buckets, int *bucket_of) {
  if (count < 0 || buckets < 1 || (count > 0 && (!n || !bucket_of))) return -1;
  for (int i = 0; i < count; i++)
    if (n[i] < 0) return -1;
  return forest_buckets(count, n, buckets, bucket_of, nullptr);
}

// ---------------------------------------------------------------- server entry points
int exafmm_server_create(exafmm_server **out, int device, int workers, double hbm_budget_bytes) {
  if (!out) return 2;
  *out = nullptr;
  if (workers < 1 || workers > 256 || !(hbm_budget_bytes > 0)) return 2;
  int dev = device;
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return 1;
  auto *s = new exafmm_server;
  s->device = dev;
  s->workers = workers;
  s->budget = hbm_budget_bytes;
  s->slots.resize(workers);
  s->held.assign(workers, 0);
  for (int w = 0; w < workers; w++) s->threads.emplace_back(&exafmm_server::worker, s, w);
  *out = s;
  return 0;
}

int exafmm_server_destroy(exafmm_server *s) {
  if (!s) return 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto &t : s->threads) t.join();
  cudaSetDevice(s->device);  // the sessions' contexts are released with it
  delete s;
  return 0;
}

int exafmm_server_submit(exafmm_server *s, const double *xyzq, long long n, double *trg, int P, double theta,
                         int ncrit, int nspawn, int precision, long long *ticket) {
  if (!s || !ticket || n < 0 || (n > 0 && (!xyzq || !trg))) return 2;
  if (P < 2 || P > 20 || ncrit < 1 || !(theta > 0)) return 2;
  if (precision != EXAFMM_FP64 && precision != EXAFMM_MIXED) return 2;
  auto r = std::make_unique<Request>();
  r->prm.P = P;
  r->prm.theta = theta;
  r->prm.ncrit = ncrit;
  r->prm.nspawn = nspawn;
  r->prm.precision = precision;
  r->xyzq = xyzq;
  r->n = n;
  r->trg = trg;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return 1;
    r->id = s->next_id++;
    r->est_bytes = s->estimate(n, P);
    *ticket = r->id;
    s->queue.push_back(r.get());
    s->reqs.emplace(r->id, std::move(r));
  }
  s->cv_work.notify_all();
  return 0;
}

int exafmm_server_open_session(exafmm_server *s, const double *xyzq, long long n, int P, double theta, int ncrit,
                               int nspawn, int precision, long long *session) {
  if (!s || !session || n < 0 || (n > 0 && !xyzq)) return 2;
  if (P < 2 || P > 20 || ncrit < 1 || !(theta > 0)) return 2;
  if (precision != EXAFMM_FP64 && precision != EXAFMM_MIXED) return 2;
  auto q = std::make_unique<Session>();
  q->prm.P = P;
  q->prm.theta = theta;
  q->prm.ncrit = ncrit;
  q->prm.nspawn = nspawn;
  q->prm.precision = precision;
  q->xyzq0 = xyzq;
  q->n = n;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return 1;
  q->id = s->next_session++;
  *session = q->id;
  s->sessions.emplace(q->id, std::move(q));
  return 0;
}

int exafmm_server_submit_step(exafmm_server *s, long long session, double sigma, unsigned long long seed,
                              const double *d_xyzq, double *trg, long long *ticket) {
  if (!s || !ticket || !(sigma >= 0) || !std::isfinite(sigma)) return 2;
  auto r = std::make_unique<Request>();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return 1;
    auto it = s->sessions.find(session);
    if (it == s->sessions.end()) {
      g_server_error = "unknown session";
      return 2;
    }
    Session *q = it->second.get();
    if (q->busy) {
      g_server_error = "the session's previous step has not completed";
      return 2;
    }
    if (q->n > 0 && !trg) return 2;
    q->busy = true;
    r->sess = q;
    r->prm = q->prm;
    r->n = q->n;
    r->trg = trg;
    r->sigma = sigma;
    r->seed = seed;
    r->d_xyzq = d_xyzq;
    r->t_submit = Clock::now();
    r->id = s->next_id++;
    r->est_bytes = s->estimate(q->n, q->prm.P);
    *ticket = r->id;
    s->queue.push_back(r.get());
    s->reqs.emplace(r->id, std::move(r));
  }
  s->cv_work.notify_all();
  return 0;
}

int exafmm_server_session_bodies(exafmm_server *s, long long session, double *xyzq) {
  if (!s || !xyzq) return 2;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->sessions.find(session);
  if (it == s->sessions.end() || it->second->busy || !it->second->ctx) {
    g_server_error = "no such idle session with a completed step";
    return 2;
  }
  cudaSetDevice(s->device);
  if (exafmm_get_bodies(it->second->ctx, xyzq) != 0) {
    g_server_error = exafmm_last_error(it->second->ctx);
    return 1;
  }
  return 0;
}

int exafmm_server_close_session(exafmm_server *s, long long session) {
  if (!s) return 2;
  std::unique_ptr<Session> q;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->sessions.find(session);
    if (it == s->sessions.end()) {
      g_server_error = "unknown session";
      return 2;
    }
    if (it->second->busy) {
      g_server_error = "the session has a step in flight";
      return 2;
    }
    s->session_held -= it->second->held;
    q = std::move(it->second);
    s->sessions.erase(it);
  }
  cudaSetDevice(s->device);
  q.reset();
  s->cv_work.notify_all();  // its bytes are free for queued requests
  return 0;
}

int exafmm_server_poll(exafmm_server *s, long long ticket, int *done) {
  if (!s || !done) return 2;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return 2;
  *done = it->second->done ? 1 : 0;
  return 0;
}

// times4: queue wait, host time from start to results, total from submit (ms), device solve time (ms).
int exafmm_server_wait(exafmm_server *s, long long ticket, double *times4) {
  if (!s) return 2;
  std::unique_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) {
      g_server_error = "unknown ticket";
      return 2;
    }
    Request *q = it->second.get();
    s->cv_done.wait(lk, [&] { return q->done; });
    r = std::move(it->second);
    s->reqs.erase(it);
  }
  if (times4) {
    times4[0] = ms_between(r->t_submit, r->t_start);
    times4[1] = ms_between(r->t_start, r->t_end);
    times4[2] = ms_between(r->t_submit, r->t_end);
    times4[3] = r->device_ms;
  }
  if (r->status != 0) g_server_error = r->err;
  return r->status;
}

// stats6: bytes in flight, bytes held by idle contexts, peak admitted bytes,
// completed requests, queued requests, budget.
int exafmm_server_stats(exafmm_server *s, double *stats6) {
  if (!s || !stats6) return 2;
  std::lock_guard<std::mutex> lk(s->mu);
  stats6[0] = (double)s->in_flight;
  stats6[1] = (double)s->held_total(-1);
  stats6[2] = (double)s->peak_admitted;
  stats6[3] = (double)s->completed;
  stats6[4] = (double)s->queue.size();
  stats6[5] = s->budget;
  return 0;
}

int exafmm_server_set_grouping(exafmm_server *s, int max_requests, long long max_request_bodies,
                               long long max_group_bodies) {
  if (!s || max_requests < 1 || max_requests > 4096 || max_request_bodies < 0 || max_group_bodies < 1) return 2;
  std::lock_guard<std::mutex> lk(s->mu);
  s->group_max = max_requests;
  s->group_max_n = max_request_bodies;
  s->group_bodies = max_group_bodies;
  return 0;
}

int exafmm_server_set_mixed_policy(exafmm_server *s, int m2l_fp32, int p2p_fp32, int min_level, int max_dl) {
  if (!s || m2l_fp32 < 0 || m2l_fp32 > 5 || min_level < 0 || max_dl < 0) return 2;
  std::lock_guard<std::mutex> lk(s->mu);
  s->policy.set = true;
  s->policy.m2l_fp32 = m2l_fp32;
  s->policy.p2p_fp32 = p2p_fp32;
  s->policy.min_level = min_level;
  s->policy.max_dl = max_dl;
  return 0;
}

int exafmm_server_grouped(exafmm_server *s, long long *requests) {
  if (!s || !requests) return 2;
  std::lock_guard<std::mutex> lk(s->mu);
  *requests = s->grouped;
  return 0;
}

const char *exafmm_server_error(void) { return g_server_error.c_str(); }

}  // extern "C"
