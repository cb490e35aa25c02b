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


def replay(server, trace: Trace, precision: int, ncrit: int = 64, nspawn: int = 5000, poll_s: float = 2e-4,
           clock=time.perf_counter, sleep=time.sleep, deadline_s: float | None = None):
    """Replays the trace against `server` (submit(x, P=, theta=, ncrit=, nspawn=, precision=) -> ticket,
    done(ticket) -> bool, wait(ticket) -> (results, times)).  Returns the completions and the wall time.
    With deadline_s, a replay that runs longer raises instead of waiting on."""
    events = [(j.arrival, k, 0) for k, j in enumerate(trace.jobs)]  # (due time, job, step)
    heapq.heapify(events)
    pending = {}           # ticket -> (job, step, due)
    bodies = {}            # job -> current bodies (chains)
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
            if step == 0:
                x = job_bodies(job)
                rngs[k] = np.random.default_rng(job.seed + 7)
            else:
                x = displace(bodies[k], job.sigma, rngs[k])
            bodies[k] = x
            tk = server.submit(x, P=job.P, theta=trace.theta, ncrit=ncrit, nspawn=nspawn, precision=precision)
            pending[tk] = (k, step, due)
        finished = [tk for tk in pending if server.done(tk)]
        for tk in finished:
            k, step, due = pending.pop(tk)
            _, times = server.wait(tk)
            end = clock() - t0
            job = trace.jobs[k]
            done.append(Completion(job=k, step=step, n=job.n, P=job.P, latency_ms=1e3 * (end - due), times=times))
            if step + 1 < job.steps:
                heapq.heappush(events, (end, k, step + 1))
            else:
                bodies.pop(k, None)
                rngs.pop(k, None)
        if not finished:
            if events and not pending:
                sleep(max(0.0, min(events[0][0] - (clock() - t0), 0.01)))
            else:
                sleep(poll_s)
    return done, clock() - t0


def latency_summary(done, wall_s: float) -> dict:
    lat = np.array([c.latency_ms for c in done]) if done else np.zeros(1)
    bodies = sum(c.n for c in done)
    return {"requests": len(done), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "bodies_per_s": bodies / wall_s if wall_s > 0 else 0.0,
            "wall_s": wall_s}
