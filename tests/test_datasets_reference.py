"""The reference's body generators, Dataset::initBodies (include/dataset.h:29-257),
restated in exafmm_b200.datasets: equal bit for bit to the reference compiled
without fast-math (tests/golden/datasets_reference.npz, made by
tests/golden/make_golden.py datasets from oracle/_ref/libexafmm_ref_dataset.so),
and to that library itself where it is built.  CPU only."""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DATASET = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libexafmm_ref_dataset.so")


@pytest.fixture(scope="module")
def gold():
    with np.load(os.path.join(GOLDEN, "datasets_reference.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def ref_lib():
    if not os.path.exists(REF_DATASET):
        pytest.skip("oracle/_ref was not built here (needs the reference tree)")
    lib = ctypes.CDLL(REF_DATASET)
    lib.ref_dataset_init_bodies.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    lib.ref_drand48.argtypes = [ctypes.c_long, ctypes.c_int, ctypes.c_void_p]
    return lib


def test_drand48_matches_libc_and_reference(datasets, gold):
    libc = ctypes.CDLL(None)
    libc.drand48.restype = ctypes.c_double
    libc.srand48.argtypes = [ctypes.c_long]
    for seed in (0, 1, 12345, -3, 2 ** 33 + 5):
        libc.srand48(seed)
        expect = np.array([libc.drand48() for _ in range(9000)])
        np.testing.assert_array_equal(datasets.drand48(seed, 9000), expect)
    np.testing.assert_array_equal(datasets.drand48(12345, 5000), gold["drand48_12345"])
    assert len(datasets.drand48(4, 0)) == 0


def test_generators_match_golden(datasets, gold):
    for key, ref in gold.items():
        if key.startswith("drand48"):
            continue
        dist, n, rank, size, ns = key.split("_")
        mine = datasets.reference_bodies(int(n), dist, int(rank), int(size), int(ns))
        assert mine.shape == ref.shape, key
        np.testing.assert_array_equal(mine, ref, err_msg=key)


@pytest.mark.parametrize("dist", ["lattice", "cube", "sphere", "octant", "plummer"])
@pytest.mark.parametrize("n,rank,size,ns", [(1, 0, 1, 1), (8, 0, 1, 1), (4101, 3, 1, 3), (50000, 1, 2, 2)])
def test_generators_match_compiled_reference(datasets, ref_lib, dist, n, rank, size, ns):
    buf = np.zeros((n * size + 8, 4))
    m = ref_lib.ref_dataset_init_bodies(n, dist.encode(), rank, size, ns, buf.ctypes.data, len(buf))
    mine = datasets.reference_bodies(n, dist, rank, size, ns)
    assert mine.shape == (m, 4)
    np.testing.assert_array_equal(mine, buf[:m])


def test_charges_have_zero_mean_per_split(datasets):
    x = datasets.reference_bodies(3001, "cube", 0, 1, 3)
    for b, e in ((0, 1001), (1001, 2001), (2001, 3001)):
        assert abs(x[b:e, 3].sum()) < 1e-12
    with pytest.raises(ValueError):
        datasets.reference_bodies(10, "gaussian")


def test_source_target_files_match_reference(datasets, ref_lib, tmp_path, monkeypatch):
    """Dataset::writeSources / writeTargets byte for byte, and successive
    readSources / readTargets going on from the returned file position."""
    monkeypatch.chdir(tmp_path)
    rng = np.random.default_rng(8)
    n = 300
    x = datasets.reference_bodies(2 * n, "plummer", 0)
    x[:5, :3] *= np.array([1e-7, 1e6, -3e-12])
    x[5, 3] = 0.0
    trg = rng.standard_normal((2 * n, 4)) * np.logspace(-9, 9, 2 * n)[:, None]
    lib = ref_lib
    lib.ref_dataset_write.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    lib.ref_dataset_read.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    lib.ref_dataset_write(2 * n, np.ascontiguousarray(x).ctypes.data, np.ascontiguousarray(trg).ctypes.data, 3)
    ref_src = open("source0003.dat", "rb").read()
    ref_trg = open("target0003.dat", "rb").read()
    mine = tmp_path / "mine"
    mine.mkdir()
    datasets.write_sources(x, 3, str(mine) + "/")
    datasets.write_targets(trg, 3, str(mine) + "/")
    assert (mine / "source0003.dat").read_bytes() == ref_src
    assert (mine / "target0003.dat").read_bytes() == ref_trg
    src_out = np.zeros((2 * n, 4))
    trg_out = np.zeros((2 * n, 4))
    lib.ref_dataset_read(n, 3, src_out.ctypes.data, trg_out.ctypes.data)
    a, pos = datasets.read_sources(n, 3)
    b, pos = datasets.read_sources(n, 3, position=pos)
    np.testing.assert_array_equal(np.vstack([a, b]), src_out)
    c, pos = datasets.read_targets(n, 3)
    d, pos = datasets.read_targets(n, 3, position=pos)
    np.testing.assert_array_equal(np.vstack([c, d]), trg_out)
    with pytest.raises(ValueError):
        datasets.read_sources(2 * n + 1, 3)
