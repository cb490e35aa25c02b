"""Solve records of the GPU engine in the reference's file formats: the list file
(Traversal::writeList under EXAFMM_COUNT_LIST) byte for byte against the one the
reference wrote for the same input, and the time file (logger::writeTime) with
the reference's event names, summed over solves and cleared when written."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rec():
    with np.load(os.path.join(GOLDEN, "records.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("tag", ["deep", "periodic"])
@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_list_file_matches_reference(ex, rec, tmp_path, tag, precision):
    P, theta, ncrit, nspawn, images, cycle = rec[f"{tag}_params"].tolist()
    f = ex.Fmm(P=int(P), theta=theta, ncrit=int(ncrit), nspawn=int(nspawn), images=int(images), cycle=cycle,
               precision=getattr(ex, precision))
    f.set_bodies(rec[f"{tag}_xyzq"])
    f.solve()
    path = f.write_list(str(tmp_path) + "/")
    f.close()
    mine = open(path, "rb").read()
    ref = bytes(rec[f"{tag}_list"])
    assert mine.count(b"\n") == ref.count(b"\n")
    assert mine == ref


def test_time_file_sums_solves_and_clears(ex, datasets, tmp_path):
    x = datasets.plummer(20000, seed=3)
    f = ex.Fmm(P=6, theta=0.4, ncrit=32)
    f.set_bodies(x)
    totals = 0.0
    for _ in range(2):
        f.solve()
        totals += f.phase_times()["total"] * 1e-3
    path = f.write_time(str(tmp_path) + "/")
    lines = open(path).read().splitlines()
    names = [ln[:20].rstrip() for ln in lines]
    vals = [float(ln[21:]) for ln in lines]
    assert names == sorted(["Get bounds", "Grow tree", "Link tree", "Upward pass", "Traverse", "Downward pass"])
    assert all(v > 0 for v in vals)
    assert abs(sum(vals) - totals) <= 1e-3 * totals + 1e-5  # the phases tile each solve
    # written and cleared: nothing until the next solve
    assert open(f.write_time(str(tmp_path) + "/")).read() == ""
    f.solve()
    assert len(open(f.write_time(str(tmp_path) + "/", rank=3)).read().splitlines()) == 6
    assert os.path.exists(os.path.join(str(tmp_path), "time000003.dat"))
    f.close()


def test_time_file_periodic_events(ex, datasets, tmp_path):
    x = datasets.cube(3000, seed=4)
    x[:, :3] *= np.pi
    f = ex.Fmm(P=6, theta=0.4, ncrit=32, images=2, cycle=2 * np.pi)
    f.set_bodies(x)
    f.solve()
    names = [ln[:20].rstrip() for ln in open(f.write_time(str(tmp_path) + "/")).read().splitlines()]
    f.close()
    assert "Traverse periodic" in names and "Traverse" in names
