"""A forest of independent systems solved together (exafmm_set_systems).

Every system must come out exactly as its solo solve does: the same bounds,
the same cell table (shifted by the system's first cell), the same body
order, the same interaction lists in the same order, and -- in FP64 and in
the pair-by-pair mixed form -- the same bits.  The solo path itself is pinned
to the reference (test_gpu_parity.py); two systems are also checked against
the CPU restatement directly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mixed_systems(datasets):
    return [datasets.cube(3000, seed=31), datasets.cube(1, seed=32), np.zeros((0, 4)),
            datasets.sphere(2500, seed=33), datasets.plummer(6000, seed=34), datasets.cube(40, seed=35),
            datasets.cube(20000, seed=36), datasets.sphere(700, seed=37), datasets.plummer(1, seed=38)]


def _solo(ex, x, policy=None, **kw):
    f = ex.Fmm(**kw)
    if policy is not None:
        f.set_mixed_policy(m2l_fp32=policy)
    f.set_bodies(x)
    f.solve()
    out = {"trg": f.results(), "bounds": f.get_bounds() if len(x) else np.zeros(6)}
    if len(x):
        out["cells"] = f.cells()
        out["perm"] = f.perm()
        out["lists"] = f.lists()
    f.close()
    return out


def _system_view(cells, perm, lists, lay, s):
    """System s's cells, order and lists in its own (solo) numbering."""
    cb, bo = lay["cell_base"], lay["body_off"]
    c0, c1, b0, b1 = cb[s], cb[s + 1], bo[s], bo[s + 1]
    ints, reals = cells[0][c0:c1].copy(), cells[1][c0:c1].copy()
    ints[:, 0] -= c0                             # IPARENT
    ints[:, 1] -= np.where(ints[:, 2] > 0, c0, 0)  # ICHILD (0 for leaves, as in the solo layout)
    ints[:, 3] -= b0                             # IBODY
    sel = []
    for lst in lists:
        m = (lst[:, 0] >= c0) & (lst[:, 0] < c1)
        part = lst[m].copy()
        part[:, :2] -= c0
        sel.append(part)
    return (ints, reals), perm[b0:b1] - b0, sel


@pytest.mark.parametrize("P,ncrit", [(6, 16), (10, 64)])
def test_forest_fp64_equals_solo_solves(ex, datasets, P, ncrit):
    xs = _mixed_systems(datasets)
    kw = dict(P=P, theta=0.4, ncrit=ncrit)
    f = ex.Fmm(**kw)
    f.set_systems(xs)
    f.solve()
    res = f.system_results()
    lay = f.systems()
    cells, perm, lists = f.cells(), f.perm(), f.lists()
    assert lay["cell_base"][-1] == f.info()["ncells"]
    for s, x in enumerate(xs):
        solo = _solo(ex, x, **kw)
        assert np.array_equal(lay["bounds"][s], solo["bounds"]), s
        assert np.array_equal(res[s], solo["trg"]), s
        if not len(x):
            assert lay["cell_base"][s + 1] == lay["cell_base"][s]
            continue
        c, p, (m2l, p2p) = _system_view(cells, perm, lists, lay, s)
        assert np.array_equal(c[0], solo["cells"][0]) and np.array_equal(c[1], solo["cells"][1]), s
        assert np.array_equal(p, solo["perm"]), s
        assert np.array_equal(m2l, solo["lists"][0]) and np.array_equal(p2p, solo["lists"][1]), s
    f.close()


def test_forest_systems_match_the_cpu_restatement(ex, datasets, oracle):
    xs = [datasets.plummer(3000, seed=41), datasets.cube(2000, seed=42)]
    f = ex.Fmm(P=8, theta=0.35, ncrit=32)
    f.set_systems(xs)
    f.solve()
    res, lay = f.system_results(), f.systems()
    cells, perm, lists = f.cells(), f.perm(), f.lists()
    for s, x in enumerate(xs):
        ref = oracle.solve(x, P=8, theta=0.35, ncrit=32)
        c, p, (m2l, p2p) = _system_view(cells, perm, lists, lay, s)
        assert np.array_equal(lay["bounds"][s], ref.bounds)
        assert np.array_equal(p, ref.perm)
        assert np.array_equal(c[0], ref.cells_int) and np.array_equal(c[1], ref.cells_real)
        as_set = lambda q: set(map(tuple, np.asarray(q)[:, :2].tolist()))
        assert as_set(m2l) == as_set(ref.m2l) and as_set(p2p) == as_set(ref.p2p)
        assert datasets.rel_l2(res[s], ref.trg) < 1e-11
    f.close()


def test_forest_mixed_pair_by_pair_equals_solo_bits(ex, datasets):
    xs = _mixed_systems(datasets)
    kw = dict(P=8, theta=0.4, ncrit=32, precision=ex.MIXED)
    f = ex.Fmm(**kw)
    f.set_mixed_policy(m2l_fp32=2)  # FP32 M2L pair by pair: no size-dependent choice of engine
    f.set_systems(xs)
    f.solve()
    res = f.system_results()
    for s, x in enumerate(xs):
        assert np.array_equal(res[s], _solo(ex, x, policy=2, **kw)["trg"]), s
    f.close()


def test_forest_mixed_tensor_cores_within_precision_bar(ex, datasets):
    # enough systems that the per-class tensor-core products run; each system's
    # mixed result against its own plain FP64 result (the same trees)
    xs = [datasets.cube(int(n), seed=500 + i) if i % 2 == 0 else datasets.sphere(int(n), seed=500 + i)
          for i, n in enumerate(datasets.log_uniform_sizes(48, 2000, 40000, 7))]
    outs = {}
    for prec, policy in ((ex.FP64, None), (ex.MIXED, 3), (ex.MIXED, 5)):
        f = ex.Fmm(P=10, theta=0.4, ncrit=64, precision=prec)
        if policy is not None:
            f.set_mixed_policy(m2l_fp32=policy)
        f.set_systems(xs)
        f.solve()
        outs[policy] = [r.copy() for r in f.system_results()]
        f.solve()  # a second solve of the same forest gives the same bits
        assert all(np.array_equal(a, b) for a, b in zip(outs[policy], f.system_results()))
        f.close()
    for policy in (3, 5):
        for s in range(len(xs)):
            plain, mixed = outs[None][s], outs[policy][s]
            assert datasets.rel_l2(mixed[:, 0], plain[:, 0]) < 1e-6, (policy, s)
            assert datasets.rel_l2(mixed[:, 1:], plain[:, 1:]) < 1e-6, (policy, s)


def test_forest_relayout_and_back_to_one_system(ex, datasets):
    xs = [datasets.cube(5000, seed=61), datasets.sphere(3000, seed=62)]
    f = ex.Fmm(P=6, theta=0.4, ncrit=32)
    f.set_systems(xs)
    f.solve()
    a = [r.copy() for r in f.system_results()]
    ys = [x.copy() for x in xs]
    ys[0][:, :3] *= 0.5                      # same layout, new positions
    f.set_systems(ys)
    f.solve()
    assert np.array_equal(f.system_results()[0], _solo(ex, ys[0], P=6, theta=0.4, ncrit=32)["trg"])
    f.set_systems(xs[::-1])                  # another layout
    f.solve()
    b = f.system_results()
    assert np.array_equal(b[0], a[1]) and np.array_equal(b[1], a[0])
    f.set_bodies(xs[0])                      # one system again
    f.solve()
    assert np.array_equal(f.results(), a[0])
    with pytest.raises(ex.FmmError):
        f.set_systems(xs)
        f.build_tree(np.array([-1.0, -1, -1, 1, 1, 1]))  # a forest takes no caller bounds
    f.close()
