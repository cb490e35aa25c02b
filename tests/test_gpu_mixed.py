"""The mixed-precision form: FP32 M2L and P2P with compensated / FP64 accumulation,
FP64 at the root levels.  Three errors are reported for every case:
mixed vs FP64 direct, plain FP64 FMM vs FP64 direct (the truncation floor of
the method at this P and theta) and mixed vs plain (the precision-only part,
held to 1e-6)."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

PRECISION_TOL = 1e-6


def _run(ex, x, precision, **kw):
    f = ex.Fmm(precision=precision, **kw)
    f.set_bodies(x)
    f.solve()
    out = f.results()
    info = f.info()
    f.close()
    return out, info


@pytest.mark.parametrize("dist,n,P,theta,ncrit", [
    ("cube", 100000, 10, 0.4, 64),
    ("plummer", 200000, 8, 0.35, 64),
    ("sphere", 50000, 10, 0.4, 64),
    ("plummer", 50000, 6, 0.4, 32),
    ("cube", 30000, 4, 0.5, 32),
])
def test_mixed_precision_error_split(ex, datasets, dist, n, P, theta, ncrit):
    x = getattr(datasets, dist)(n, seed=31)
    plain, info64 = _run(ex, x, ex.FP64, P=P, theta=theta, ncrit=ncrit)
    mixed, info32 = _run(ex, x, ex.MIXED, P=P, theta=theta, ncrit=ncrit)
    assert info64 == info32  # same tree, same lists
    idx = datasets.strided_sample(n, 512)
    direct = ex.direct(x[idx], x)
    e_mixed_direct = rel_l2(mixed[idx, 0], direct[:, 0])
    e_plain_direct = rel_l2(plain[idx, 0], direct[:, 0])
    e_precision = rel_l2(mixed[:, 0], plain[:, 0])
    e_precision_acc = rel_l2(mixed[:, 1:], plain[:, 1:])
    print(f"{dist} n={n} P={P}: mixed-direct {e_mixed_direct:.2e} plain-direct {e_plain_direct:.2e} "
          f"mixed-plain pot {e_precision:.2e} acc {e_precision_acc:.2e}")
    assert e_precision < PRECISION_TOL
    assert e_precision_acc < 10 * PRECISION_TOL
    # the mixed result is as close to the direct sum as the plain method, up to the precision part
    assert e_mixed_direct < e_plain_direct + 2 * PRECISION_TOL


@pytest.mark.parametrize("P", [4, 6, 8, 10])
def test_tile_m2l_matches_pair_by_pair(ex, datasets, P):
    """The per-class products (tensor cores, bf16x3 pieces; CUDA cores, FP32) and
    the pair-by-pair FP32 M2L evaluate the same operator: each within the
    precision bar of the FP64 plain method on the same tree, and of each other (a
    wrong operator would be off by O(1)).  The tensor-core products keep
    FP32-class accuracy: within ten times the CUDA-core products' distance to
    FP64 (two bf16 pieces instead of three would be about a hundred times off)."""
    for gen, n in (("plummer", 60000), ("cube", 40000), ("sphere", 30000)):
        x = getattr(datasets, gen)(n, seed=P)
        res = []
        for prec, pol in ((ex.FP64, None), (ex.MIXED, 3), (ex.MIXED, 5), (ex.MIXED, 2)):
            f = ex.Fmm(P=P, theta=0.4, ncrit=32, precision=prec)
            if pol is not None:
                f.set_mixed_policy(m2l_fp32=pol)
            f.set_bodies(x)
            f.solve()
            res.append(f.results())
            f.close()
        plain, tc, cc, pair = res
        errs = {}
        for name, a, b in (("tc-plain", tc, plain), ("cc-plain", cc, plain), ("pair-plain", pair, plain),
                           ("tc-pair", tc, pair), ("tc-cc", tc, cc)):
            errs[name] = (rel_l2(a[:, 0], b[:, 0]), rel_l2(a[:, 1:], b[:, 1:]))
            assert errs[name][0] < PRECISION_TOL, (name, errs[name])
            assert errs[name][1] < PRECISION_TOL, (name, errs[name])
        print(f"P={P} {gen}: " + " ".join(f"{k} {v[0]:.2e}/{v[1]:.2e}" for k, v in errs.items()))
        for i in range(2):
            assert errs["tc-plain"][i] < 10 * errs["cc-plain"][i] + 1e-8


@pytest.mark.parametrize("dist,n", [("plummer", 60000), ("cube", 40000)])
def test_p2p_targets_per_lane_settings_agree(ex, datasets, dist, n):
    """The mixed P2P's targets per lane (by leaf size, two, three for every leaf)
    is a tuning parameter: each setting stays within the precision bar of the
    plain method on the same tree, and of the others."""
    x = getattr(datasets, dist)(n, seed=77)
    kw = dict(P=8, theta=0.4, ncrit=64)
    plain, _ = _run(ex, x, ex.FP64, **kw)
    outs = {}
    for tpl in (0, 2, 3):
        f = ex.Fmm(precision=ex.MIXED, **kw)
        f.set_p2p_targets_per_lane(tpl)
        f.set_bodies(x)
        f.solve()
        outs[tpl] = f.results()
        f.close()
        assert rel_l2(outs[tpl][:, 0], plain[:, 0]) < PRECISION_TOL
        assert rel_l2(outs[tpl][:, 1:], plain[:, 1:]) < PRECISION_TOL
    assert rel_l2(outs[2][:, 1:], outs[3][:, 1:]) < PRECISION_TOL
    with pytest.raises(ex.FmmError):
        f = ex.Fmm(precision=ex.MIXED, **kw)
        f.set_p2p_targets_per_lane(4)
