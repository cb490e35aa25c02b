"""Pins the CPU restatement (oracle/) to the reference: golden fixtures made by the
reference's own headers (tests/golden/make_golden.py) and, where it was built,
the compiled reference itself on fresh seeded inputs.  CPU only."""
import os

import numpy as np
import pytest

from conftest import golden_cases, load_golden, pair_set, periodic_golden_cases, rel_l2, GOLDEN


def _sorted(p):
    p = np.asarray(p)[:, :2]
    return p[np.lexsort((p[:, 1], p[:, 0]))] if len(p) else p.reshape(0, 2)


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_matches_golden(oracle, path):
    g = load_golden(path)
    P, theta, ncrit, nspawn = g["params"]
    run = oracle.solve(g["xyzq"], P=int(P), theta=float(theta), ncrit=int(ncrit), nspawn=int(nspawn),
                       expansions="M" in g)
    assert np.array_equal(run.bounds, g["bounds"])           # bit-exact, including the 1e-5 drift
    assert np.array_equal(run.perm, g["perm"])               # tree order of the bodies
    assert np.array_equal(run.cells_int, g["cells_int"])     # IPARENT, ICHILD, NCHILD, IBODY, NBODY
    assert np.array_equal(run.cells_real, g["cells_real"])   # centers and radii
    assert np.array_equal(_sorted(run.m2l), g["m2l"])
    assert np.array_equal(_sorted(run.p2p), g["p2p"])
    assert rel_l2(run.trg[:, 0], g["trg"][:, 0]) < 1e-12
    assert rel_l2(run.trg[:, 1:], g["trg"][:, 1:]) < 1e-12
    if "M" in g:
        assert np.abs(run.M - g["M"]).max() <= 1e-12 * np.abs(g["M"]).max()
        assert np.abs(run.L - g["L"]).max() <= 1e-12 * max(np.abs(g["L"]).max(), 1e-300)


def test_oracle_kernel_chain_matches_golden(oracle):
    """examples/kernel.cxx: P2M -> M2M -> M2L -> L2L -> L2P against P2P."""
    g = load_golden(os.path.join(GOLDEN, "kernel_kat.npz"))
    src = np.array([[2.0, 2.0, 2.0, 1.0]])
    tgt = np.array([[-2.0, 2.0, 2.0, 1.0]])
    Xj, XJ, XI, Xi = [3.0, 1.0, 1.0], [4.0, 0.0, 0.0], [-4.0, 0.0, 0.0], [-3.0, 1.0, 1.0]
    for P in (4, 8, 10, 14):
        Mj = oracle.p2m(P, Xj, src)
        MJ = oracle.m2m(P, XJ, np.array([Xj]), Mj[None, :])
        LI = oracle.m2l(P, XI, XJ, MJ)
        Li = oracle.l2l(P, Xi, XI, LI)
        trg = oracle.l2p(P, Xi, Li, tgt)
        for name, v in (("Mj", Mj), ("MJ", MJ), ("LI", LI), ("Li", Li)):
            ref = g[f"P{P}_{name}"]
            assert np.abs(v - ref).max() <= 1e-13 * np.abs(ref).max(), (P, name)
        assert rel_l2(trg, g[f"P{P}_trg"]) < 1e-13
        assert rel_l2(oracle.p2p(tgt, src), g[f"P{P}_direct"]) < 1e-15
    # the truncation error of the chain falls with P, as in the reference's kernel.dat
    errs = [rel_l2(g[f"P{P}_trg"][:, 0], g[f"P{P}_direct"][:, 0]) for P in (4, 8, 10, 14)]
    assert errs == sorted(errs, reverse=True) and errs[-1] < 1e-3


@pytest.mark.parametrize("dist,n,P,ncrit,nspawn", [
    ("cube", 6000, 6, 32, 5000),
    ("plummer", 8000, 8, 16, 2000),
    ("sphere", 4000, 10, 64, 5000),
    ("cube", 2000, 5, 4, 1),
])
def test_oracle_matches_live_reference(oracle, reference, datasets, dist, n, P, ncrit, nspawn):
    x = getattr(datasets, dist)(n, seed=101)
    a = oracle.solve(x, P=P, ncrit=ncrit, nspawn=nspawn)
    b = reference.solve(x, P=P, ncrit=ncrit, nspawn=nspawn)
    assert np.array_equal(a.bounds, b.bounds)
    assert np.array_equal(a.perm, b.perm)
    assert np.array_equal(a.cells_int, b.cells_int)
    assert np.array_equal(a.cells_real, b.cells_real)
    assert pair_set(a.m2l) == pair_set(b.m2l) and len(a.m2l) == len(b.m2l)
    assert pair_set(a.p2p) == pair_set(b.p2p) and len(a.p2p) == len(b.p2p)
    assert rel_l2(a.trg, b.trg) < 1e-12


def test_oracle_periodic_matches_live_reference(oracle, reference, datasets):
    x = datasets.cube(600, seed=7)
    x[:, :3] *= np.pi  # the reference's periodic box is [-pi, pi]^3 with cycle 2*pi
    a = oracle.solve(x, P=6, ncrit=16, images=2, cycle=2 * np.pi, dipole_correction=True)
    b = reference.solve(x, P=6, ncrit=16, images=2, cycle=2 * np.pi, dipole_correction=True)
    # 27 near images: the same pair may appear once per image, so compare multisets.
    # The reference log also holds the lattice M2Ls of traversePeriodic, whose
    # sources are temporary cells outside the tree: (images-1) * 124 * 125 of them.
    nc = len(b.cells_int)
    lattice = (b.m2l[:, 1] >= nc) | (b.m2l[:, 1] < 0)
    assert lattice.sum() == (2 - 1) * 124 * 125
    assert np.array_equal(_sorted(a.m2l), _sorted(b.m2l[~lattice]))
    assert np.array_equal(_sorted(a.p2p), _sorted(b.p2p))
    assert rel_l2(a.trg, b.trg) < 1e-11


def test_oracle_direct_matches_live_reference(oracle, reference, datasets):
    xi, xj = datasets.cube(50, seed=1), datasets.cube(300, seed=2)
    assert rel_l2(oracle.direct(xi, xj), reference.direct(xi, xj)) < 1e-14
    assert rel_l2(oracle.direct(xi, xj, images=1), reference.direct(xi, xj, images=1)) < 1e-13


@pytest.mark.parametrize("x,k,up", [(0.7, 100000, 0), (-0.9, 300000, 0), (0.3, 250000, 1), (1e-4, 50000, 0),
                                    (-3.0, 1000000, 1), (5e-6, 7, 0), (0.0, 123456, 1)])
def test_oracle_drift_is_stepwise(oracle, x, k, up):
    v = x
    step = 1e-5
    if k <= 300000:
        for _ in range(k):
            v = v + step if up else v - step
        assert oracle.drift_seq(x, k, up) == v
    else:
        assert abs(oracle.drift_seq(x, k, up) - (x + (k * step if up else -k * step))) < 1e-6


@pytest.mark.parametrize("path", periodic_golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_periodic_matches_golden(oracle, path):
    """The C restatement against the reference's periodic fixtures (near images,
    lattice and dipole correction)."""
    g = load_golden(path)
    P, theta, ncrit, nspawn, images, cycle = g["params"]
    r = oracle.solve(g["xyzq"], P=int(P), theta=float(theta), ncrit=int(ncrit), nspawn=int(nspawn),
                     images=int(images), cycle=float(cycle), dipole_correction=True)
    assert np.array_equal(r.bounds, g["bounds"])
    assert np.array_equal(r.cells_int, g["cells_int"])
    assert np.array_equal(_sorted(r.m2l), g["m2l"])
    assert np.array_equal(_sorted(r.p2p), g["p2p"])
    assert rel_l2(r.trg, g["trg"]) < 1e-11


def test_oracle_ewald_matches_reference(oracle, reference):
    """Ewald (include/ewald.h) restated in C against the reference compiled in
    place, with the cutoff below L/2 minus the leaf size, where the reference's
    per-cell-pair periodic image is every pair's nearest image."""
    rng = np.random.default_rng(1)
    for n, ks in ((400, 8), (900, 11)):
        L = 2 * np.pi
        x = np.empty((n, 4))
        x[:, :3] = rng.uniform(-L / 2, L / 2, (n, 3))
        q = rng.uniform(-1, 1, n)
        x[:, 3] = q - q.mean()
        kw = dict(ksize=ks, alpha=ks / L, sigma=0.25 / np.pi, cutoff=L / 4, cycle=L)
        a = oracle.ewald(x, **kw)
        b = reference.ewald(x, ncrit=16, **kw)
        assert rel_l2(a[:, 0], b[:, 0]) < 1e-12
        assert rel_l2(a[:, 1:], b[:, 1:]) < 1e-12


def test_restatement_matches_the_reference_on_the_large_fixture(oracle):
    """The CPU restatement against the compiled reference's 1,048,576-body
    all-positive Plummer run (sampled targets, whole-run sums and list sizes)."""
    import hashlib
    from conftest import GOLDEN, load_golden, load_package
    load_package()
    import exafmm_b200.datasets as datasets
    g = load_golden(os.path.join(GOLDEN, "large_plummer_n1048576_p8.npz"))
    x = getattr(datasets, str(g["generator"]))(int(g["n"]), int(g["seed"]))
    assert hashlib.sha256(x.tobytes()).hexdigest() == str(g["xyzq_sha256"])
    P, theta, ncrit, nspawn = g["params"]
    a = oracle.solve(x, P=int(P), theta=float(theta), ncrit=int(ncrit), nspawn=int(nspawn))
    assert np.array_equal(a.bounds, g["bounds"])
    assert (len(a.cells_int), len(a.m2l), len(a.p2p)) == (int(g["ncells"]), int(g["n_m2l"]), int(g["n_p2p"]))
    idx = g["idx"]
    assert rel_l2(a.trg[idx], g["trg"]) < 1e-12
    assert abs(a.trg[:, 0].sum() / g["pot_sum"] - 1) < 1e-12
