"""The mixed form pinned to the reference itself, not to this engine's own FP64
path: every M2L engine of the mixed form against the CPU restatement on the
plain-method workload (100,000 bodies in the cube, zero net charge, P = 10,
theta = 0.4, ncrit = 64), and against the compiled reference's results on a
1,048,576-body all-positive Plummer sphere (P = 8, theta = 0.35), the
distribution of the single large adaptive solve, where a bias of the FP32 or
tensor-core sums would accumulate (tests/golden/make_golden.py, case "large").

Bars: mixed vs reference <= 1e-6 rel-L2 on the potential (the precision bar),
the gradient within 1e-6 as well; plain FP64 vs reference <= 1e-10."""
import hashlib
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden, rel_l2

pytestmark = pytest.mark.gpu

PRECISION_TOL = 1e-6
PLAIN_TOL = 1e-10
# m2l_fp32 policies: 1 tensor-core class products where they pay, 2 pair by pair
# only, 3 tensor-core class products at any size, 5 CUDA-core class products
ENGINES = (1, 2, 3, 5)


def _solve(ex, x, precision, policy=None, min_level=2, **kw):
    f = ex.Fmm(precision=precision, **kw)
    if policy is not None:
        f.set_mixed_policy(m2l_fp32=policy, min_level=min_level)
    f.set_bodies(x)
    f.solve()
    out, info, bounds = f.results(), f.info(), f.get_bounds()
    f.close()
    return out, info, bounds


@pytest.fixture(scope="module")
def config1(datasets, oracle):
    x = datasets.cube(100000, seed=404)
    return x, oracle.solve(x, P=10, theta=0.4, ncrit=64, nspawn=5000)


@pytest.mark.parametrize("policy,min_level", [(p, 4) for p in ENGINES] + [(1, 2), (2, 2)])
def test_mixed_engines_match_the_restatement_plain_workload(ex, config1, policy, min_level):
    x, ref = config1
    mixed, _, _ = _solve(ex, x, ex.MIXED, policy, min_level, P=10, theta=0.4, ncrit=64)
    e_pot, e_acc = rel_l2(mixed[:, 0], ref.trg[:, 0]), rel_l2(mixed[:, 1:], ref.trg[:, 1:])
    print(f"policy {policy} min_level {min_level}: pot {e_pot:.2e} acc {e_acc:.2e}")
    assert e_pot < PRECISION_TOL and e_acc < PRECISION_TOL


def test_plain_matches_the_restatement_plain_workload(ex, config1):
    x, ref = config1
    plain, _, bounds = _solve(ex, x, ex.FP64, P=10, theta=0.4, ncrit=64)
    assert np.array_equal(bounds, ref.bounds)
    assert rel_l2(plain[:, 0], ref.trg[:, 0]) < PLAIN_TOL and rel_l2(plain[:, 1:], ref.trg[:, 1:]) < PLAIN_TOL


@pytest.fixture(scope="module")
def large(datasets):
    g = load_golden(os.path.join(GOLDEN, "large_plummer_n1048576_p8.npz"))
    x = getattr(datasets, str(g["generator"]))(int(g["n"]), int(g["seed"]))
    assert hashlib.sha256(x.tobytes()).hexdigest() == str(g["xyzq_sha256"]), "bodies do not regenerate"
    P, theta, ncrit, nspawn = g["params"]
    return x, g, dict(P=int(P), theta=float(theta), ncrit=int(ncrit), nspawn=int(nspawn))


def test_large_plummer_plain_matches_the_reference(ex, large):
    x, g, kw = large
    plain, info, bounds = _solve(ex, x, ex.FP64, **kw)
    assert np.array_equal(bounds, g["bounds"])
    assert (info["ncells"], info["n_m2l"], info["n_p2p"]) == (int(g["ncells"]), int(g["n_m2l"]), int(g["n_p2p"]))
    idx = g["idx"]
    assert rel_l2(plain[idx, 0], g["trg"][:, 0]) < PLAIN_TOL
    assert rel_l2(plain[idx, 1:], g["trg"][:, 1:]) < PLAIN_TOL
    assert abs(plain[:, 0].sum() / g["pot_sum"] - 1) < PLAIN_TOL
    assert abs((plain[:, 1:] ** 2).sum() / g["acc_sq_sum"] - 1) < PLAIN_TOL


@pytest.mark.parametrize("policy", ENGINES)
def test_large_plummer_mixed_matches_the_reference(ex, large, policy):
    """All charges positive: the far field of the whole sphere adds up in every
    target's potential, so a systematic error of the FP32 / bf16x3 sums shows
    here as a shift of the potential's sum, not only as scatter."""
    x, g, kw = large
    mixed, _, _ = _solve(ex, x, ex.MIXED, policy, **kw)
    idx = g["idx"]
    e_pot, e_acc = rel_l2(mixed[idx, 0], g["trg"][:, 0]), rel_l2(mixed[idx, 1:], g["trg"][:, 1:])
    bias = mixed[:, 0].sum() / g["pot_sum"] - 1
    print(f"policy {policy}: pot {e_pot:.2e} acc {e_acc:.2e} sum {bias:.2e}")
    assert e_pot < PRECISION_TOL and e_acc < PRECISION_TOL
    assert abs(bias) < PRECISION_TOL
