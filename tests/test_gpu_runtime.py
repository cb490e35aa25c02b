"""The batch solver and the request server (host runtime over pools of solve
contexts).  A system's result must not depend on what runs beside it: the
same bits alone, in a batch, or among other requests."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _systems(datasets, k, lo, hi, seed):
    sizes = datasets.log_uniform_sizes(k, lo, hi, seed)
    return [datasets.cube(int(n), seed=seed + i) if i % 2 == 0 else datasets.sphere(int(n), seed=seed + i)
            for i, n in enumerate(sizes)]


def _alone(ex, x, **kw):
    f = ex.Fmm(**kw)
    f.set_bodies(x)
    f.solve()
    r = f.results()
    f.close()
    return r


def test_batch_matches_single_solves(ex, datasets):
    xs = _systems(datasets, 12, 500, 40000, 100)
    b = ex.Batch(P=6, theta=0.4, ncrit=32, workers=4)
    outs = b.solve(xs)
    for x, o in zip(xs, outs):
        assert np.array_equal(o, _alone(ex, x, P=6, theta=0.4, ncrit=32))
    again = b.solve(xs)
    assert all(np.array_equal(a, c) for a, c in zip(outs, again))
    assert (b.times(len(xs)) > 0).all()
    b.close()


def test_batch_mixed_precision_and_empty(ex, datasets):
    xs = _systems(datasets, 6, 1000, 20000, 300) + [np.zeros((0, 4)), datasets.cube(1, seed=9)]
    b = ex.Batch(P=8, theta=0.4, ncrit=64, precision=ex.MIXED, workers=3)
    outs = b.solve(xs)
    for x, o in zip(xs, outs):
        assert np.array_equal(o, _alone(ex, x, P=8, theta=0.4, ncrit=64, precision=ex.MIXED))
    b.close()


def test_batch_autotune_then_frozen(ex, datasets):
    xs = _systems(datasets, 12, 3000, 5000, 200)
    b = ex.Batch(P=4, theta=0.4, ncrit=64, workers=3)
    b.autotune(True)
    b.solve(xs)
    b.autotune(False)
    table = b.ncrit_table()
    assert table and all(v in (32, 64, 128) for v in table.values())
    o1 = b.solve(xs)
    o2 = b.solve(xs)
    assert all(np.array_equal(a, c) for a, c in zip(o1, o2))
    for x, o in zip(xs, o1):  # each system ran with its class's tuned ncrit
        nc = table.get(int(np.floor(np.log2(len(x)))), 64)
        assert np.array_equal(o, _alone(ex, x, P=4, theta=0.4, ncrit=nc))
    b2 = ex.Batch(P=4, theta=0.4, ncrit=64, workers=2)  # a loaded table reproduces the same trees
    b2.set_ncrit_table(table)
    assert b2.ncrit_table() == table
    assert all(np.array_equal(a, c) for a, c in zip(o1, b2.solve(xs)))
    b2.close()
    b.close()


def test_server_result_same_alone_and_in_mix(ex, datasets):
    s = ex.Server(workers=4, hbm_budget_bytes=40e9)
    x = datasets.plummer(30000, seed=5)
    kw = dict(P=8, theta=0.4, ncrit=64, precision=ex.MIXED)
    alone, t_alone = s.wait(s.submit(x, **kw))
    mix = []
    for i, n in enumerate([50000, 2000, 120000, 8000]):
        mix.append(s.submit(datasets.cube(n, seed=40 + i), P=(6, 8, 10)[i % 3], theta=0.4, ncrit=64,
                            precision=(ex.FP64, ex.MIXED)[i % 2]))
    tk = s.submit(x, **kw)
    for i, n in enumerate([30000, 70000, 1000]):
        mix.append(s.submit(datasets.sphere(n, seed=60 + i), P=10, theta=0.4, ncrit=32))
    in_mix, times = s.wait(tk)
    for t in mix:
        s.wait(t)
    assert np.array_equal(alone, in_mix)
    assert np.array_equal(alone, _alone(ex, x, **kw))
    assert times[2] >= times[1] >= 0 and times[3] > 0
    st = s.stats()
    assert st["completed"] == 2 + len(mix) and st["queued"] == 0
    s.close()


def test_server_admission_serializes_under_tiny_budget(ex, datasets):
    s = ex.Server(workers=4, hbm_budget_bytes=1.0)  # no two requests fit together
    xs = _systems(datasets, 6, 2000, 30000, 500)
    tickets = [s.submit(x, P=6, theta=0.4, ncrit=32) for x in xs]
    outs = [s.wait(t)[0] for t in tickets]
    for x, o in zip(xs, outs):
        assert np.array_equal(o, _alone(ex, x, P=6, theta=0.4, ncrit=32))
    st = s.stats()
    assert st["completed"] == len(xs) and st["held"] == 0 and st["in_flight"] == 0
    s.close()


def test_forest_batch_matches_single_solves(ex, datasets):
    """Forest mode: the systems of a call are grouped by size into forests, one
    context each; every system still gets the bits of its solo solve at its
    group's ncrit, through host or device pointers, and again on a second call."""
    import torch
    xs = _systems(datasets, 14, 500, 60000, 700) + [np.zeros((0, 4)), datasets.cube(1, seed=11)]
    kw = dict(P=8, theta=0.4, precision=ex.MIXED)
    b = ex.Batch(ncrit=64, workers=3, forest=3, **kw)
    b.set_mixed_policy(m2l_fp32=1, min_level=2)
    outs = b.solve(xs)
    group, ncrit = b.buckets(len(xs))
    assert len(ncrit) == group.max() + 1 <= 3
    assert b.elapsed_ms() > 0
    for x, o, gi in zip(xs, outs, group):
        f = ex.Fmm(ncrit=int(ncrit[gi]), **kw)
        f.set_mixed_policy(m2l_fp32=1, min_level=2)
        f.set_bodies(x)
        f.solve()
        assert np.array_equal(o, f.results())
        f.close()
    dev = [torch.from_numpy(x.copy()).cuda() for x in xs]
    dout = [torch.zeros_like(d) for d in dev]
    b.solve_device([len(x) for x in xs], [d.data_ptr() for d in dev], [d.data_ptr() for d in dout])
    torch.cuda.synchronize()
    assert all(np.array_equal(o, d.cpu().numpy()) for o, d in zip(outs, dout))
    b.close()


def test_forest_batch_autotune_per_group(ex, datasets):
    xs = _systems(datasets, 10, 1000, 40000, 800)
    b = ex.Batch(P=6, theta=0.4, ncrit=64, workers=2, forest=2)
    b.autotune(True)
    for _ in range(3):                 # one candidate per call
        b.solve(xs)
    b.autotune(False)
    table = b.ncrit_table()
    group, ncrit = b.buckets(len(xs))
    assert len(table) == group.max() + 1 and all(v in (32, 64, 128) for v in table.values())
    o1 = b.solve(xs)
    group, ncrit = b.buckets(len(xs))
    assert sorted(ncrit.tolist()) == sorted(table.values())
    for x, o, gi in zip(xs, o1, group):
        assert np.array_equal(o, _alone(ex, x, P=6, theta=0.4, ncrit=int(ncrit[gi])))
    b2 = ex.Batch(P=6, theta=0.4, ncrit=64, workers=2, forest=2)   # a loaded table gives the same trees
    b2.set_ncrit_table(table)
    assert all(np.array_equal(a, c) for a, c in zip(o1, b2.solve(xs)))
    b2.close()
    b.close()


def test_server_chain_steps_stay_on_the_device(ex, datasets):
    """A session's step k (bodies moved on the device, tree rebuilt there) gives
    the bits of a fresh solve of the same positions, alone or beside other
    requests; the first step solves the opened bodies."""
    s = ex.Server(workers=3, hbm_budget_bytes=40e9)
    x = datasets.plummer(20000, seed=21)
    kw = dict(P=8, theta=0.4, ncrit=64, precision=ex.MIXED)
    sid = s.open_session(x, **kw)
    r0, _ = s.wait(s.submit_step(sid))
    assert np.array_equal(r0, _alone(ex, x, **kw))
    assert np.array_equal(s.session_bodies(sid), x)
    sigma = 1e-3 * (4 / 3 * np.pi / len(x)) ** (1 / 3)
    prev = x
    for k in range(1, 4):
        other = s.submit(datasets.cube(30000, seed=k), P=6, theta=0.4, ncrit=32)
        rk, _ = s.wait(s.submit_step(sid, sigma=sigma, seed=1000 + k))
        s.wait(other)
        xk = s.session_bodies(sid)
        moved = xk[:, :3] - prev[:, :3]
        assert np.array_equal(xk[:, 3], x[:, 3]) and 0 < np.abs(moved).max() < 20 * sigma
        assert abs(np.std(moved) / sigma - 1) < 0.05
        assert np.array_equal(rk, _alone(ex, xk, **kw))
        prev = xk
    # the displacement depends only on (seed, sigma, body index)
    f = ex.Fmm(**kw)
    f.set_bodies(x)
    f.displace_bodies(sigma, 1001)
    sid2 = s.open_session(x, **kw)
    s.wait(s.submit_step(sid2))
    s.wait(s.submit_step(sid2, sigma=sigma, seed=1001))
    assert np.array_equal(f.bodies(), s.session_bodies(sid2))
    f.close()
    with pytest.raises(ex.FmmError):        # one step at a time per session
        t = s.submit_step(sid, sigma=sigma, seed=7)
        s.submit_step(sid, sigma=sigma, seed=8)
    s.wait(t)
    s.close_session(sid)
    s.close_session(sid2)
    st = s.stats()
    assert st["queued"] == 0 and st["in_flight"] == 0
    s.close()


def test_server_groups_small_queued_requests_into_one_forest(ex, datasets):
    """Continuous batching: small requests with equal parameters that queue behind
    a running one are solved together as a forest; each still gets its solo bits,
    and requests with other parameters are not mixed in."""
    s = ex.Server(workers=1, hbm_budget_bytes=40e9)
    big = s.submit(datasets.plummer(400000, seed=3), P=8, theta=0.4, ncrit=64, precision=ex.MIXED)
    kw = dict(P=8, theta=0.4, ncrit=64, precision=ex.MIXED)
    xs = _systems(datasets, 12, 1000, 30000, 900)
    tickets = [s.submit(x, **kw) for x in xs]
    odd = datasets.cube(5000, seed=5)
    t_odd = s.submit(odd, P=6, theta=0.4, ncrit=64, precision=ex.MIXED)
    s.wait(big)
    outs = [s.wait(t)[0] for t in tickets]
    r_odd, _ = s.wait(t_odd)
    assert s.stats()["grouped"] >= 2
    for x, o in zip(xs, outs):
        assert np.array_equal(o, _alone(ex, x, **kw))
    assert np.array_equal(r_odd, _alone(ex, odd, P=6, theta=0.4, ncrit=64, precision=ex.MIXED))
    s.set_grouping(max_requests=1)     # off: one request per solve
    g0 = s.stats()["grouped"]
    big = s.submit(datasets.plummer(400000, seed=3), **kw)
    tickets = [s.submit(x, **kw) for x in xs[:4]]
    s.wait(big)
    assert all(np.array_equal(s.wait(t)[0], o) for t, o in zip(tickets, outs[:4]))
    assert s.stats()["grouped"] == g0
    s.close()


def test_forest_batch_tunes_ncrit_and_targets_per_lane(ex, datasets):
    """The autotuner tries every ncrit with every P2P targets-per-lane setting,
    one pair per call, and keeps the fastest per group; each system then has the
    bits of its solo solve with its group's pair, and a loaded table reproduces
    them."""
    xs = _systems(datasets, 10, 2000, 40000, 900)
    kw = dict(P=8, theta=0.4, precision=ex.MIXED)
    b = ex.Batch(ncrit=64, workers=2, forest=2, **kw)
    b.set_ncrit_candidates([32, 64])
    b.set_p2p_candidates([0, 2, 3])
    b.autotune(True)
    for _ in range(6):
        b.solve(xs)
    b.autotune(False)
    table = b.config_table()
    group, ncrit = b.buckets(len(xs))
    assert len(table) == group.max() + 1
    assert all(nc in (32, 64) and tp in (0, 2, 3) for nc, tp in table.values())
    outs = b.solve(xs)
    group, ncrit = b.buckets(len(xs))
    tpl = b.bucket_p2p()
    for x, o, gi in zip(xs, outs, group):
        f = ex.Fmm(ncrit=int(ncrit[gi]), **kw)
        f.set_p2p_targets_per_lane(int(tpl[gi]))
        f.set_bodies(x)
        f.solve()
        assert np.array_equal(o, f.results())
        f.close()
    b2 = ex.Batch(ncrit=64, workers=2, forest=2, **kw)
    b2.set_config_table(table)
    assert b2.config_table() == table
    assert all(np.array_equal(a, c) for a, c in zip(outs, b2.solve(xs)))
    b2.close()
    b.close()
