"""Separate source bodies (examples/fmm.cxx -j IneJ) on the GPU against fixtures the
reference wrote (tests/golden/make_golden.py inej): extended bounds, both trees and
the cross-tree interaction lists bit for bit, FP64 results within the plain
method's bar."""
import os

import numpy as np
import pytest

from conftest import inej_golden_cases, load_golden, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _sorted(p):
    p = np.asarray(p)[:, :2]
    return p[np.lexsort((p[:, 1], p[:, 0]))] if len(p) else p.reshape(0, 2)


@pytest.mark.parametrize("path", inej_golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
def test_separate_sources_match_reference(ex, path):
    g = load_golden(path)
    P, theta, ncrit, nspawn = g["params"]
    f = ex.Fmm(P=int(P), theta=float(theta), ncrit=int(ncrit), nspawn=int(nspawn))
    f.set_bodies(g["xyzq"])
    f.set_sources(g["jxyzq"])
    assert np.array_equal(f.get_bounds(), g["bounds"])
    f.solve()
    trg = f.results()
    assert np.array_equal(f.perm(), g["perm"])
    ci, cr = f.cells()
    assert np.array_equal(ci, g["cells_int"])
    assert np.array_equal(cr, g["cells_real"])
    ji, jr, jp = f.source_cells()
    assert np.array_equal(ji, g["jcells_int"])
    assert np.array_equal(jr, g["jcells_real"])
    assert np.array_equal(jp, g["jperm"])
    m2l, p2p = f.lists()
    assert np.array_equal(_sorted(m2l), g["m2l"])
    assert np.array_equal(_sorted(p2p), g["p2p"])
    assert rel_l2(trg[:, 0], g["trg"][:, 0]) < TOL
    assert rel_l2(trg[:, 1:], g["trg"][:, 1:]) < TOL
    f.close()


def test_separate_sources_against_direct_and_reset(ex, datasets):
    x = datasets.cube(3000, seed=8)
    jx = datasets.plummer(4000, seed=9)
    f = ex.Fmm(P=10, theta=0.4, ncrit=64)
    f.set_bodies(x)
    f.set_sources(jx)
    f.solve()
    trg = f.results()
    idx = datasets.strided_sample(len(x), 256)
    direct = ex.direct(x[idx], jx)
    assert rel_l2(trg[idx, 0], direct[:, 0]) < 1e-5
    assert rel_l2(trg[idx, 1:], direct[:, 1:]) < 1e-4
    # sources back to the bodies themselves: the same as a fresh context
    f.set_sources(None)
    f.solve()
    self_trg = f.results()
    g = ex.Fmm(P=10, theta=0.4, ncrit=64)
    g.set_bodies(x)
    g.solve()
    assert np.array_equal(self_trg, g.results())
    f.close()
    g.close()


def test_separate_sources_need_free_space(ex, datasets):
    x = datasets.cube(500, seed=1)
    f = ex.Fmm(P=6, images=1)
    f.set_bodies(x)
    f.set_sources(x[:100])
    with pytest.raises(ex.FmmError, match="free space"):
        f.solve()
    f.close()


@pytest.mark.parametrize("path", inej_golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
def test_separate_sources_mixed_form(ex, datasets, path):
    """The mixed form across two trees (FP32 P2P over the source tree's bodies,
    pair-by-pair FP32 M2L from its multipoles, FP64 at the root levels): the same
    trees and lists as the FP64 solve, results within the precision bar of it and
    of the reference's, on the reference fixtures and on a larger pair of sets."""
    g = load_golden(path)
    P, theta, ncrit, nspawn = g["params"]
    kw = dict(P=int(P), theta=float(theta), ncrit=int(ncrit), nspawn=int(nspawn))
    cases = [(g["xyzq"], g["jxyzq"], g["trg"])]
    x = datasets.cube(40000, seed=12)
    jx = datasets.plummer(50000, seed=13)
    x[:, 0] = (x[:, 0] + np.pi) * 0.5   # examples/fmm.cxx's -j shifts
    jx[:, 0] = (jx[:, 0] - np.pi) * 0.5
    cases.append((x, jx, None))
    for xi, xj, ref in cases:
        out = {}
        for prec in (ex.FP64, ex.MIXED):
            f = ex.Fmm(precision=prec, **kw)
            f.set_bodies(xi)
            f.set_sources(xj)
            f.solve()
            out[prec] = (f.results(), f.lists())
            f.close()
        (plain, (m2l64, p2p64)), (mixed, (m2l32, p2p32)) = out[ex.FP64], out[ex.MIXED]
        assert np.array_equal(m2l64, m2l32) and np.array_equal(p2p64, p2p32)
        for a, b in ((mixed, plain),) + (((mixed, ref),) if ref is not None else ()):
            assert rel_l2(a[:, 0], b[:, 0]) < 1e-6 and rel_l2(a[:, 1:], b[:, 1:]) < 1e-6
