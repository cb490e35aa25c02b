"""Solve records in the reference's file formats, host side (CPU only): the cell
keys of Traversal::writeList (BuildTree::getKey, include/build_tree.h:111-120)
and logger::writeTime's layout (include/logger.h:116-127), against fixtures the
reference itself wrote (tests/golden/make_golden.py records)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

RECORDS = os.path.join(GOLDEN, "records.npz")


@pytest.fixture(scope="module")
def rec():
    with np.load(RECORDS) as z:
        return {k: z[k] for k in z.files}


def _levels(cells_real):
    return np.rint(np.log2(cells_real[0, 3] / cells_real[:, 3])).astype(int)


@pytest.mark.parametrize("tag", ["deep", "periodic"])
def test_cell_keys_match_reference(ex, rec, tag):
    """Every cell's key equals the reference's ICELL, including the levels >= 11
    where the reference's 32-bit shifts wrap (the deep case reaches level 19)."""
    cr = rec[f"{tag}_cells_real"]
    lev = _levels(cr)
    Xmin = cr[0, :3] - cr[0, 3]
    keys = np.array([ex.morton_key(cr[c, :3], Xmin, 2 * cr[c, 3], lev[c]) for c in range(len(cr))],
                    dtype=np.uint64)
    np.testing.assert_array_equal(keys, rec[f"{tag}_icell"])
    if tag == "deep":
        assert lev.max() >= 16
        assert (keys > np.uint64(2 ** 32)).sum() > 0  # sign-extended wraps are exercised


def test_time_file_matches_reference_writer(ex, rec, tmp_path):
    names = [str(s) for s in rec["time_names"]]
    events = dict(zip(names, rec["time_values"].tolist()))
    path = ex.write_time_events(events, str(tmp_path) + "/")
    assert os.path.basename(path) == "time000000.dat"
    with open(path, "rb") as f:
        assert f.read() == bytes(rec["time_text"])


def test_time_file_rank_and_accumulation(ex, tmp_path):
    """The rank is zero-padded to six digits; events are written in name order."""
    path = ex.write_time_events({"b": 1.0, "a": 2.5e-9}, str(tmp_path) + "/", rank=42)
    assert path.endswith("time000042.dat")
    lines = open(path).read().splitlines()
    assert lines == ["a                    2.5e-09", "b                    1"]


def test_time_file_matches_reference_on_random_events(ex, reference, tmp_path):
    rng = np.random.default_rng(7)
    events = {f"event {i:02d}" + "x" * int(rng.integers(0, 25)): float(10.0 ** rng.uniform(-9, 6))
              for i in range(12)}
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    ex.write_time_events(events, str(a) + "/")
    reference.write_time(events, str(b) + "/")
    assert (a / "time000000.dat").read_bytes() == (b / "time000000.dat").read_bytes()
