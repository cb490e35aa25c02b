"""Host logic of the batched and served workloads (no GPU): system and trace
generation, and the trace replay against a stand-in server on a simulated clock."""
import numpy as np
import pytest

from conftest import load_package


@pytest.fixture(scope="module")
def wl():
    load_package()
    import exafmm_b200.workloads as w
    return w


def test_batch_systems_are_seeded_and_in_range(wl):
    a = wl.batch_systems(count=6, lo=2000, hi=20000, seed0=1000)
    b = wl.batch_systems(count=6, lo=2000, hi=20000, seed0=1000)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert all(2000 <= len(x) <= 20000 for x in a)
    assert np.allclose(np.linalg.norm(a[1][:, :3], axis=1), 1.0)      # odd: sphere surface
    assert np.abs(a[0][:, :3]).max() <= 1.0                            # even: cube


def test_trace_statistics(wl):
    tr = wl.make_trace(count=4000, rate=50.0, lo=1000, hi=1_000_000, seed=9)
    gaps = np.diff([0.0] + [j.arrival for j in tr.jobs])
    assert abs(gaps.mean() - 1 / 50.0) < 0.1 / 50.0
    chains = [j for j in tr.jobs if j.steps > 1]
    assert abs(len(chains) / len(tr.jobs) - 0.2) < 0.03
    assert all(j.steps == 50 and j.sigma > 0 for j in chains)
    assert all(1000 <= j.n <= 1_000_000 and j.P in (6, 8, 10) for j in tr.jobs)
    assert tr.solves == len(tr.jobs) + 49 * len(chains)


class _Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, s):
        self.t += max(s, 1e-5)


class _FakeServer:
    """Completes a request 1 ms + 10 ns per body after its submission."""

    def __init__(self, clock):
        self.clock, self.next, self.live, self.log = clock, 1, {}, []

    def submit(self, x, P, theta, ncrit, nspawn, precision):
        t = self.next
        self.next += 1
        self.live[t] = (self.clock(), len(x), x)
        self.log.append((t, self.clock(), len(x)))
        return t

    def done(self, t):
        t0, n, _ = self.live[t]
        return self.clock() - t0 >= 1e-3 + 1e-8 * n

    def wait(self, t):
        _, n, x = self.live.pop(t)
        return np.zeros((n, 4)), np.zeros(4)


def test_replay_runs_every_step_in_order(wl):
    tr = wl.make_trace(count=30, rate=200.0, lo=1000, hi=20000, repeat_frac=0.3, repeat_steps=5, seed=3)
    clk = _Clock()
    srv = _FakeServer(clk)
    done, wall = wl.replay(srv, tr, precision=1, clock=clk, sleep=clk.sleep)
    assert len(done) == tr.solves and not srv.live
    for k, j in enumerate(tr.jobs):
        steps = [c for c in done if c.job == k]
        assert [c.step for c in steps] == list(range(j.steps))
        # service time bounds the latency from below
        assert all(c.latency_ms >= 1e3 * (1e-3 + 1e-8 * j.n) - 1e-6 for c in steps)
    s = wl.latency_summary(done, wall)
    assert s["requests"] == tr.solves and s["p99_ms"] >= s["p50_ms"] > 0


def test_chain_steps_move_the_bodies(wl):
    rng = np.random.default_rng(0)
    x = np.zeros((100, 4))
    y = wl.displace(x, 1e-3, rng)
    assert np.allclose(y[:, 3], 0) and 0 < np.abs(y[:, :3]).max() < 1e-2
