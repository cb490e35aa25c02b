"""Workload drivers for the batched and served configurations.

Batched: many independent systems solved per call (Batch).  Served: a request
trace with Poisson arrivals, replayed against a Server; repeat systems are
chains of solves of one system whose bodies move a little between steps (an MD
trajectory), each step submitted when the previous one returns.

The trace logic is plain Python over a small server interface (submit / done /
wait), so it runs the same against the real Server and against a stand-in.
"""
from __future__ import annotations

import heapq
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import datasets


# ---------------------------------------------------------------- batched systems
def batch_systems(count: int = 512, lo: int = 2000, hi: int = 200_000, seed0: int = 1000):
    """count systems, N log-uniform in [lo, hi]; even ones uniform in [-1, 1]^3,
    odd ones on the unit sphere; charges U[-1, 1]; seed seed0 + index."""
    out = []
    for i in range(count):
        rng = np.random.default_rng(seed0 + i)
        n = int(math.exp(rng.uniform(math.log(lo), math.log(hi))))
        out.append(datasets.cube(n, seed=seed0 + i) if i % 2 == 0 else datasets.sphere(n, seed=seed0 + i))
    return out


# ---------------------------------------------------------------- request traces
@dataclass
class Job:
    """One trace entry: a single solve, or a chain of `steps` solves of one system."""
    arrival: float                 # seconds from the start of the replay
    n: int
    P: int
    kind: str                      # "cube" or "plummer"
    seed: int
    steps: int = 1
    sigma: float = 0.0             # per-step Gaussian displacement of a chain


@dataclass
class Trace:
    jobs: list
    rate: float
    theta: float = 0.4

    @property
    def solves(self) -> int:
        return sum(j.steps for j in self.jobs)


def make_trace(count: int, rate: float, lo: int = 1000, hi: int = 1_000_000, orders=(6, 8, 10),
               repeat_frac: float = 0.2, repeat_steps: int = 50, seed: int = 4000, theta: float = 0.4) -> Trace:
    """Poisson arrivals at `rate` jobs/s; N log-uniform in [lo, hi]; P uniform over
    `orders`; cube or Plummer with equal odds; a fraction `repeat_frac` of the
    jobs are chains of `repeat_steps` solves with displacement sigma = 1e-3 times
    the mean spacing (V / N)^(1/3)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        n = int(math.exp(rng.uniform(math.log(lo), math.log(hi))))
        kind = "cube" if rng.uniform() < 0.5 else "plummer"
        P = int(orders[rng.integers(len(orders))])
        chain = rng.uniform() < repeat_frac
        volume = 8.0 if kind == "cube" else 4.0 / 3.0 * math.pi  # [-1,1]^3, or the Plummer core
        sigma = 1e-3 * (volume / n) ** (1.0 / 3.0) if chain else 0.0
        jobs.append(Job(arrival=t, n=n, P=P, kind=kind, seed=seed + 1 + i, steps=repeat_steps if chain else 1,
                        sigma=sigma))
    return Trace(jobs=jobs, rate=rate, theta=theta)


def job_bodies(job: Job) -> np.ndarray:
    return datasets.cube(job.n, seed=job.seed) if job.kind == "cube" else datasets.plummer(job.n, seed=job.seed)


def displace(x: np.ndarray, sigma: float, rng) -> np.ndarray:
    y = x.copy()
    y[:, :3] += rng.normal(scale=sigma, size=(len(x), 3))
    return y


@dataclass
class Completion:
    job: int
    step: int
    n: int
    P: int
    latency_ms: float             # scheduled arrival (or previous step's return) to results on the host
    times: np.ndarray = field(default_factory=lambda: np.zeros(4))
    end_s: float = 0.0            # completion, seconds from the start of the replay
    steps: int = 1                # steps of its job (1: a single solve)


def chain_seed(job: Job, step: int) -> int:
    """Seed of a chain step's device-side displacement (the same in every replay)."""
    return job.seed * 1_000_003 + step


def replay(server, trace: Trace, precision: int, ncrit: int = 64, nspawn: int = 5000, poll_s: float = 2e-4,
           clock=time.perf_counter, sleep=time.sleep, deadline_s: float | None = None,
           device_chains: bool | None = None, samples: dict | None = None, sample_size: int = 256,
           host_alloc=None):
    """Replays the trace against `server` (submit(x, P=, theta=, ncrit=, nspawn=, precision=) -> ticket,
    done(ticket) -> bool, wait(ticket) -> (results, times)).  Returns the completions and the wall time.
    With deadline_s, a replay that runs longer raises instead of waiting on.

    Chains run device-resident when the server has sessions (open_session / submit_step /
    session_bodies / close_session; device_chains=None means whenever it does): the first step
    uploads the bodies, every later step moves them on the device by a Gaussian step of the
    job's sigma (seed chain_seed(job, step)) and solves again.  Otherwise each step is displaced
    on the host and submitted as a new request.

    samples (a dict) receives, per job, the final step's results on `sample_size` strided
    targets: {job: (target indices, results there, final bodies or None when they are the
    job's initial bodies)}.

    host_alloc(shape) -> float64 array, if given, allocates the requests' host
    buffers (pinned memory, for instance); they are filled before the clock starts."""
    if device_chains is None:
        device_chains = hasattr(server, "open_session")
    # the requests' inputs exist before the replay starts (generating them is
    # not the server's work): every job's bodies, and a result buffer whose
    # pages are already touched
    alloc = host_alloc or (lambda shape: np.empty(shape))
    inputs, outputs = {}, {}
    for k, j in enumerate(trace.jobs):
        x = alloc((j.n, 4))
        x[:] = job_bodies(j)
        o = alloc((j.n, 4))
        o.fill(0.0)
        inputs[k], outputs[k] = x, o
    events = [(j.arrival, k, 0) for k, j in enumerate(trace.jobs)]  # (due time, job, step)
    heapq.heapify(events)
    pending = {}           # ticket -> (job, step, due)
    bodies = {}            # job -> current bodies (chains displaced on the host)
    sessions = {}          # job -> session (device-resident chains)
    rngs = {}
    done = []
    t0 = clock()
    while events or pending:
        now = clock() - t0
        if deadline_s is not None and now > deadline_s:
            raise TimeoutError(f"trace replay exceeded {deadline_s} s with {len(pending)} requests pending")
        while events and events[0][0] <= now:
            due, k, step = heapq.heappop(events)
            job = trace.jobs[k]
            if job.steps > 1 and device_chains:
                if step == 0:
                    sessions[k] = server.open_session(inputs[k], P=job.P, theta=trace.theta, ncrit=ncrit,
                                                      nspawn=nspawn, precision=precision)
                    tk = server.submit_step(sessions[k], out=outputs[k])
                else:
                    tk = server.submit_step(sessions[k], sigma=job.sigma, seed=chain_seed(job, step), out=outputs[k])
            else:
                if step == 0:
                    x = inputs[k]
                    rngs[k] = np.random.default_rng(job.seed + 7)
                else:
                    x = displace(bodies[k], job.sigma, rngs[k])
                bodies[k] = x
                tk = server.submit(x, P=job.P, theta=trace.theta, ncrit=ncrit, nspawn=nspawn, precision=precision,
                                   out=outputs[k])
            pending[tk] = (k, step, due)
        finished = [tk for tk in pending if server.done(tk)]
        for tk in finished:
            k, step, due = pending.pop(tk)
            res, times = server.wait(tk)
            end = clock() - t0
            job = trace.jobs[k]
            done.append(Completion(job=k, step=step, n=job.n, P=job.P, latency_ms=1e3 * (end - due), times=times,
                                   end_s=end, steps=job.steps))
            if step + 1 < job.steps:
                heapq.heappush(events, (end, k, step + 1))
            else:
                if samples is not None:
                    idx = datasets.strided_sample(job.n, sample_size)
                    final = None
                    if job.steps > 1:
                        final = server.session_bodies(sessions[k]) if k in sessions else bodies[k]
                    samples[k] = (idx, np.array(res[idx]), final)
                if k in sessions:
                    server.close_session(sessions.pop(k))
                bodies.pop(k, None)
                rngs.pop(k, None)
                inputs.pop(k, None)
                outputs.pop(k, None)
        if not finished:
            if events and not pending:
                sleep(max(0.0, min(events[0][0] - (clock() - t0), 0.01)))
            else:
                sleep(poll_s)
    return done, clock() - t0


def latency_summary(done, wall_s: float) -> dict:
    lat = np.array([c.latency_ms for c in done]) if done else np.zeros(1)
    bodies = sum(c.n for c in done)
    out = {"requests": len(done), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
           "mean_ms": float(lat.mean()), "bodies_per_s": bodies / wall_s if wall_s > 0 else 0.0,
           "wall_s": wall_s}
    out["device_ms_sum"] = float(sum(float(c.times[3]) for c in done))
    chain = [c.latency_ms for c in done if c.steps > 1 and c.step > 0]
    if chain:
        out["chain_step_p50_ms"] = float(np.percentile(chain, 50))
        out["chain_step_p99_ms"] = float(np.percentile(chain, 99))
    return out


def saturated_throughput(done) -> dict:
    """Bodies/s while a saturated replay still has single solves to run: every
    completion up to the last single solve's, over that time.  After it only the
    repeat chains' remaining steps are left, one step at a time each, which
    measures their sequential latency rather than the server's throughput."""
    singles = [c.end_s for c in done if c.steps == 1]
    if not singles:
        return {"bodies_per_s": 0.0, "window_s": 0.0, "requests": 0}
    t = max(singles)
    inside = [c for c in done if c.end_s <= t]
    return {"bodies_per_s": sum(c.n for c in inside) / t if t > 0 else 0.0, "window_s": t,
            "requests": len(inside), "bodies": sum(c.n for c in inside)}
