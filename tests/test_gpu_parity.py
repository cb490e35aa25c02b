"""Parity of the CUDA path (through the C ABI) with the reference: golden fixtures
made by the reference headers, and the CPU restatement on fresh seeded inputs.

Tree, bounds and interaction lists must match bit for bit; FP64 values within
rel-L2 1e-11 of the reference (the bar for the plain method is 1e-10)."""
import os

import numpy as np
import pytest

from conftest import golden_cases, load_golden, pair_set, rel_l2, GOLDEN

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _sorted(p):
    p = np.asarray(p)[:, :2]
    return p[np.lexsort((p[:, 1], p[:, 0]))] if len(p) else p.reshape(0, 2)


def _solve(ex, x, **kw):
    f = ex.Fmm(**kw)
    f.set_bodies(x)
    bounds = f.get_bounds()
    f.solve()
    return f, bounds, f.results()


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
def test_gpu_matches_golden(ex, path):
    g = load_golden(path)
    P, theta, ncrit, nspawn = g["params"]
    f, bounds, trg = _solve(ex, g["xyzq"], P=int(P), theta=float(theta), ncrit=int(ncrit), nspawn=int(nspawn))
    assert np.array_equal(bounds, g["bounds"])
    assert np.array_equal(f.perm(), g["perm"])
    ci, cr = f.cells()
    assert np.array_equal(ci, g["cells_int"])
    assert np.array_equal(cr, g["cells_real"])
    m2l, p2p = f.lists()
    assert np.array_equal(_sorted(m2l), g["m2l"])
    assert np.array_equal(_sorted(p2p), g["p2p"])
    assert rel_l2(trg[:, 0], g["trg"][:, 0]) < TOL
    assert rel_l2(trg[:, 1:], g["trg"][:, 1:]) < TOL
    if "M" in g:
        M, L = f.expansions()
        assert np.abs(M - g["M"]).max() <= 1e-12 * np.abs(g["M"]).max()
        assert np.abs(L - g["L"]).max() <= 1e-12 * max(np.abs(g["L"]).max(), 1e-300)
    f.close()


def test_gpu_kernel_chain_matches_golden(ex):
    """examples/kernel.cxx known-answer chain through the per-operator entry points."""
    g = load_golden(os.path.join(GOLDEN, "kernel_kat.npz"))
    src = np.array([[2.0, 2.0, 2.0, 1.0]])
    tgt = np.array([[-2.0, 2.0, 2.0, 1.0]])
    Xj, XJ, XI, Xi = [3.0, 1.0, 1.0], [4.0, 0.0, 0.0], [-4.0, 0.0, 0.0], [-3.0, 1.0, 1.0]
    for P in (4, 8, 10, 14):
        Mj = ex.p2m(P, Xj, src)
        MJ = ex.m2m(P, XJ, np.array([Xj]), Mj[None, :])
        LI = ex.m2l(P, XI, XJ, MJ)
        Li = ex.l2l(P, Xi, XI, LI)
        trg = ex.l2p(P, Xi, Li, tgt)
        for name, v in (("Mj", Mj), ("MJ", MJ), ("LI", LI), ("Li", Li)):
            ref = g[f"P{P}_{name}"]
            assert np.abs(v - ref).max() <= 1e-13 * np.abs(ref).max(), (P, name)
        assert rel_l2(trg, g[f"P{P}_trg"]) < 1e-13
        assert rel_l2(ex.p2p(tgt, src), g[f"P{P}_direct"]) < 1e-15


@pytest.mark.parametrize("P", [3, 6, 12, 17, 20])
def test_gpu_operators_match_oracle_all_orders(ex, oracle, P):
    # High orders sum terms with factorially large weights, so two FP64 evaluation
    # orders drift apart by ~1e-11 of the largest coefficient at P = 20.
    tol = 1e-12 if P <= 12 else 1e-10
    rng = np.random.default_rng(P)
    xs = np.c_[rng.uniform(-0.5, 0.5, (37, 3)), rng.uniform(-1, 1, 37)]
    X = np.array([0.1, -0.2, 0.05])
    M = oracle.p2m(P, X, xs)
    assert np.abs(ex.p2m(P, X, xs) - M).max() <= tol * np.abs(M).max()
    Xc = X + rng.uniform(-0.6, 0.6, (3, 3))
    Mc = np.stack([oracle.p2m(P, c, xs) for c in Xc])
    Mp = oracle.m2m(P, X, Xc, Mc)
    assert np.abs(ex.m2m(P, X, Xc, Mc) - Mp).max() <= tol * np.abs(Mp).max()
    Xi = np.array([4.0, 1.0, -2.0])
    L = oracle.m2l(P, Xi, X, Mp)
    assert np.abs(ex.m2l(P, Xi, X, Mp) - L).max() <= tol * np.abs(L).max()
    Xch = Xi + np.array([-0.3, 0.2, 0.25])
    Lc = oracle.l2l(P, Xch, Xi, L)
    assert np.abs(ex.l2l(P, Xch, Xi, L) - Lc).max() <= tol * np.abs(Lc).max()
    tb = np.c_[Xch + rng.uniform(-0.2, 0.2, (45, 3)), np.ones(45)]
    assert rel_l2(ex.l2p(P, Xch, Lc, tb), oracle.l2p(P, Xch, Lc, tb)) < tol


def test_gpu_p2p_and_direct_match_oracle(ex, oracle, datasets):
    xi, xj = datasets.cube(300, seed=1), datasets.cube(257, seed=2)
    assert rel_l2(ex.p2p(xi, xj), oracle.p2p(xi, xj)) < 1e-14
    shift = np.array([2.0, -2.0, 0.0])
    assert rel_l2(ex.p2p(xi, xj, Xper=shift), oracle.p2p(xi, xj, Xper=shift)) < 1e-14
    assert rel_l2(ex.direct(xi, xj), oracle.direct(xi, xj)) < 1e-14
    assert rel_l2(ex.direct(xi, xj, images=1), oracle.direct(xi, xj, images=1)) < 1e-14
    # self-interaction (r = 0) pairs are skipped, as in the reference
    assert rel_l2(ex.p2p(xi, xi), oracle.p2p(xi, xi)) < 1e-14


@pytest.mark.parametrize("dist,n,P,theta,ncrit,nspawn", [
    ("cube", 100000, 10, 0.4, 64, 5000),     # the plain-method workload (N=1e5, P=10)
    ("plummer", 60000, 8, 0.35, 32, 5000),   # strongly adaptive
    ("sphere", 30000, 10, 0.4, 64, 5000),
    ("cube", 20000, 6, 0.5, 16, 1),          # nspawn = 1: every internal pair splits both
    ("plummer", 20000, 4, 0.6, 128, 5000),
])
def test_gpu_matches_oracle(ex, oracle, datasets, dist, n, P, theta, ncrit, nspawn):
    x = getattr(datasets, dist)(n, seed=202)
    a = oracle.solve(x, P=P, theta=theta, ncrit=ncrit, nspawn=nspawn)
    f, bounds, trg = _solve(ex, x, P=P, theta=theta, ncrit=ncrit, nspawn=nspawn)
    assert np.array_equal(bounds, a.bounds)
    assert np.array_equal(f.perm(), a.perm)
    ci, cr = f.cells()
    assert np.array_equal(ci, a.cells_int) and np.array_equal(cr, a.cells_real)
    m2l, p2p = f.lists()
    assert len(m2l) == len(a.m2l) and pair_set(m2l) == pair_set(a.m2l)
    assert len(p2p) == len(a.p2p) and pair_set(p2p) == pair_set(a.p2p)
    assert rel_l2(trg[:, 0], a.trg[:, 0]) < TOL
    assert rel_l2(trg[:, 1:], a.trg[:, 1:]) < TOL
    f.close()


@pytest.mark.parametrize("n,ncrit", [(1, 64), (2, 1), (64, 64), (65, 64), (7, 1)])
def test_gpu_small_and_root_leaf_cases(ex, oracle, datasets, n, ncrit):
    x = datasets.cube(n, seed=n)
    a = oracle.solve(x, P=6, ncrit=ncrit)
    f, bounds, trg = _solve(ex, x, P=6, ncrit=ncrit)
    assert np.array_equal(bounds, a.bounds)
    assert np.array_equal(f.perm(), a.perm)
    assert np.array_equal(f.cells()[0], a.cells_int)
    assert rel_l2(trg, a.trg) < TOL if n > 1 else np.allclose(trg, 0)


def test_gpu_empty_input(ex):
    f = ex.Fmm(P=6)
    f.set_bodies(np.zeros((0, 4)))
    assert np.array_equal(f.get_bounds(), np.zeros(6))
    f.solve()
    assert f.results().shape == (0, 4)
    assert f.info()["ncells"] == 0


def test_gpu_coincident_bodies_within_ncrit(ex, oracle):
    """Bodies at identical positions: r = 0 pairs are skipped and the tree still splits."""
    rng = np.random.default_rng(9)
    base = np.c_[rng.uniform(-1, 1, (500, 3)), rng.uniform(-1, 1, 500)]
    x = np.vstack([base, base[:20], base[:20]])  # triplicated bodies, fewer than ncrit per spot
    a = oracle.solve(x, P=6, ncrit=16)
    f, bounds, trg = _solve(ex, x, P=6, ncrit=16)
    assert np.array_equal(f.perm(), a.perm)
    assert rel_l2(trg, a.trg) < TOL


def test_gpu_too_deep_tree_is_an_error(ex):
    """More than ncrit coincident bodies make the reference recurse without end;
    the engine reports an error instead (no GPU fault: the kernels only set a flag)."""
    x = np.zeros((40, 4))
    x[:, 3] = 1.0
    x[:20, :3] = 0.25
    x[20:, :3] = np.random.default_rng(1).uniform(-1, 1, (20, 3))
    f = ex.Fmm(P=4, ncrit=8)
    f.set_bodies(x)
    with pytest.raises(ex.FmmError, match="deeper"):
        f.solve()
    # the context stays usable
    f.set_bodies(np.c_[np.random.default_rng(2).uniform(-1, 1, (100, 3)), np.ones(100)])
    f.solve()
    assert np.isfinite(f.results()).all()


def test_gpu_bad_parameters_are_errors(ex):
    with pytest.raises(ex.FmmError):
        ex.Fmm(P=1)
    with pytest.raises(ex.FmmError):
        ex.Fmm(P=21)
    with pytest.raises(ex.FmmError):
        ex.Fmm(P=6, ncrit=0)
    f = ex.Fmm(P=6)
    with pytest.raises(ex.FmmError):
        f.upward()  # before any tree


def test_gpu_device_pointer_api_and_determinism(ex, datasets):
    import torch
    x = datasets.cube(50000, seed=4)
    f, _, trg = _solve(ex, x, P=8, ncrit=32)
    dx = torch.from_numpy(x).cuda()
    dout = torch.zeros_like(dx)
    g = ex.Fmm(P=8, ncrit=32)
    torch.cuda.synchronize()
    g.set_bodies_device(dx.data_ptr(), len(x))
    g.solve()
    g.results_device(dout.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(dout.cpu().numpy(), trg)  # same engine, same order: bitwise
    g.solve()
    assert np.array_equal(g.results(), trg)


def test_gpu_results_follow_input_order(ex, datasets):
    """With the same bounds, permuting the caller's bodies permutes the results:
    the tree is the same, only the order inside leaves (and so the summation
    order) changes.  (getBounds itself depends on input order through its drift.)"""
    x = datasets.plummer(20000, seed=8)
    p = np.random.default_rng(0).permutation(len(x))
    outs = []
    for xx in (x, x[p]):
        f = ex.Fmm(P=8, ncrit=32)
        f.set_bodies(xx)
        f.build_tree(bounds=[-21.0, -21.0, -21.0, 21.0, 21.0, 21.0])
        f.upward()
        f.traverse()
        f.downward()
        outs.append(f.results())
    assert rel_l2(outs[1], outs[0][p]) < 1e-12


def test_gpu_context_reuse_with_growing_systems(ex, datasets):
    """One context solving ever larger systems (its buffers grow between solves)
    gives the same bits as fresh contexts, in both precision modes."""
    for prec in (ex.FP64, ex.MIXED):
        f = ex.Fmm(P=6, theta=0.4, ncrit=32, precision=prec)
        for n, gen in ((700, "cube"), (40000, "plummer"), (3000, "sphere"), (250000, "plummer")):
            x = getattr(datasets, gen)(n, seed=n)
            f.set_bodies(x)
            f.solve()
            reused = f.results()
            g = ex.Fmm(P=6, theta=0.4, ncrit=32, precision=prec)
            g.set_bodies(x)
            g.solve()
            assert np.array_equal(reused, g.results())
            g.close()
        f.close()


def test_p2p_interaction_count_matches_the_lists(ex, datasets):
    """exafmm_list_work: the sum over P2P list entries of NBODY(target) * NBODY(source),
    recomputed here from the cell table and the lists (free space, periodic, forest)."""
    for kw, systems in ((dict(P=6, theta=0.4, ncrit=32), None), (dict(P=6, theta=0.4, ncrit=32, images=1), None),
                        (dict(P=6, theta=0.4, ncrit=16), [datasets.cube(3000, seed=8), datasets.plummer(2000, seed=9)])):
        f = ex.Fmm(**kw)
        if systems is None:
            f.set_bodies(datasets.plummer(20000, seed=7) if not kw.get("images") else datasets.cube(5000, seed=7))
        else:
            f.set_systems(systems)
        f.solve()
        ints, _ = f.cells()
        _, p2p = f.lists()
        nb = ints[:, 4].astype(np.int64)
        expect = int(np.sum(nb[p2p[:, 0]] * nb[p2p[:, 1]]))
        assert f.p2p_interactions() == expect
        f.close()
