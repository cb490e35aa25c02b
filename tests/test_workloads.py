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

    def submit(self, x, P, theta, ncrit, nspawn, precision, out=None):
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


class _FakeSessionServer(_FakeServer):
    """The stand-in with device-resident chains: a session keeps its bodies and
    moves them by a seeded Gaussian step per later step."""

    def __init__(self, clock):
        super().__init__(clock)
        self.sessions, self.opened, self.closed, self.steps = {}, 0, 0, []

    def open_session(self, x, P, theta, ncrit, nspawn, precision):
        self.opened += 1
        sid = 1000 + self.opened
        self.sessions[sid] = [x.copy(), False]
        return sid

    def submit_step(self, sid, sigma=0.0, seed=0, out=None):
        s = self.sessions[sid]
        assert not s[1], "a session runs one step at a time"
        if sigma:
            s[0] = s[0].copy()
            s[0][:, :3] += np.random.default_rng(seed).normal(scale=sigma, size=(len(s[0]), 3))
        s[1] = True
        self.steps.append((sid, sigma, seed))
        t = self.submit(s[0], None, None, None, None, None)
        self.live[t] = self.live[t][:2] + (sid,)
        return t

    def wait(self, t):
        _, n, tag = self.live.pop(t)
        if isinstance(tag, int) and tag in self.sessions:
            self.sessions[tag][1] = False
        return np.zeros((n, 4)), np.zeros(4)

    def session_bodies(self, sid):
        return self.sessions[sid][0].copy()

    def close_session(self, sid):
        assert not self.sessions[sid][1]
        del self.sessions[sid]
        self.closed += 1


def test_replay_keeps_chains_on_the_device_when_the_server_can(wl):
    tr = wl.make_trace(count=20, rate=300.0, lo=1000, hi=5000, repeat_frac=0.4, repeat_steps=4, seed=5)
    clk = _Clock()
    srv = _FakeSessionServer(clk)
    samples = {}
    done, wall = wl.replay(srv, tr, precision=1, clock=clk, sleep=clk.sleep, samples=samples, sample_size=16)
    chains = [k for k, j in enumerate(tr.jobs) if j.steps > 1]
    assert chains and srv.opened == srv.closed == len(chains) and not srv.sessions
    assert len(done) == tr.solves and not srv.live
    # chain steps after the first carry the job's sigma and a per-step seed; only
    # the single solves were submitted with host bodies
    moved = [s for s in srv.steps if s[1] > 0]
    assert len(moved) == sum(tr.jobs[k].steps - 1 for k in chains)
    assert len({s[2] for s in moved}) == len(moved)
    assert len(srv.log) == tr.solves
    assert set(samples) == set(range(len(tr.jobs)))
    for k, (idx, res, final) in samples.items():
        j = tr.jobs[k]
        assert len(idx) == min(16, j.n) and res.shape == (len(idx), 4)
        assert (final is None) == (j.steps == 1)
        if final is not None:
            assert final.shape == (j.n, 4) and not np.array_equal(final, wl.job_bodies(j))


def test_saturated_throughput_stops_at_the_last_single_solve(wl):
    C = wl.Completion
    done = [C(job=0, step=0, n=100, P=6, latency_ms=1, end_s=1.0),
            C(job=1, step=0, n=50, P=6, latency_ms=1, end_s=1.5, steps=3),
            C(job=2, step=0, n=300, P=6, latency_ms=1, end_s=2.0),
            C(job=1, step=1, n=50, P=6, latency_ms=1, end_s=3.0, steps=3),
            C(job=1, step=2, n=50, P=6, latency_ms=1, end_s=4.0, steps=3)]
    t = wl.saturated_throughput(done)
    assert t["window_s"] == 2.0 and t["requests"] == 3 and t["bodies_per_s"] == 450 / 2.0
    s = wl.latency_summary(done, 4.0)
    assert s["chain_step_p50_ms"] == 1 and s["requests"] == 5
