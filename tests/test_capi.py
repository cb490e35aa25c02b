"""The C ABI library builds, loads and exports every entry point include/exafmm_b200.h
declares; host-side logic that needs no GPU.  CPU only."""
import ctypes
import subprocess

import numpy as np
import pytest


def test_library_exports_every_declared_symbol(ex):
    L = ctypes.CDLL(ex.LIB_PATH)
    declared = ex.exported_symbols()
    assert len(declared) >= 25
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    # and nm agrees that they are dynamic, defined, C-linkage symbols
    out = subprocess.run(["nm", "-D", "--defined-only", ex.LIB_PATH], capture_output=True, text=True).stdout
    names = {line.split()[-1] for line in out.splitlines() if line.strip()}
    assert set(declared) <= names


@pytest.mark.parametrize("which", ["gromacs", "distributed"])
def test_md_libraries_export_their_abi(ex, which):
    """Each MD-code ABI lives in its own library (their FMM_* names overlap) that
    exports every function its header declares; the engine library exports none."""
    path, header = {"gromacs": (ex.MD_GROMACS_LIB_PATH, ex.MD_HEADER),
                    "distributed": (ex.MD_DISTRIBUTED_LIB_PATH, ex.MDD_HEADER)}[which]
    declared = ex.md_exported_symbols(header)
    assert {"FMM_Init", "FMM_Finalize", "FMM_Partition", "FMM_Error"} <= set(declared)
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    names = {line.split()[-1] for line in out.splitlines() if line.strip()}
    assert set(declared) <= names
    L = ctypes.CDLL(path)
    assert all(hasattr(L, s) for s in declared)
    engine = subprocess.run(["nm", "-D", "--defined-only", ex.LIB_PATH], capture_output=True, text=True).stdout
    assert "FMM_Init" not in engine


@pytest.mark.parametrize("seed", range(6))
def test_closed_form_drift_matches_stepwise_recurrence(ex, oracle, seed):
    """BoundBox::getBounds's running min/max drift (include/bound_box.h:19-20),
    evaluated by the engine in closed form, equals the step-by-step recurrence."""
    rng = np.random.default_rng(seed)
    for _ in range(60):
        x = float(rng.choice([rng.uniform(-1, 1), rng.uniform(-2e-4, 2e-4), rng.uniform(-40, 40),
                              2.0 ** rng.integers(-14, 6), -(2.0 ** rng.integers(-14, 6)), 0.0]))
        k = int(rng.choice([rng.integers(0, 50), rng.integers(0, 20000), rng.integers(0, 400000)]))
        up = int(rng.integers(0, 2))
        assert ex.drift(x, k, up) == oracle.drift_seq(x, k, up), (x, k, up)


def test_closed_form_bounds_equal_sequential_bounds(ex, oracle, datasets):
    """The parallel bounds are min_j g^(N-1-j)(x_j) with g the drift step; evaluated
    on the host with the engine's closed form they equal the oracle's loop."""
    for gen, n in (("cube", 3000), ("plummer", 5000), ("sphere", 2000)):
        x = getattr(datasets, gen)(n, seed=3)
        b = oracle.bounds(x)
        lo = np.full(3, np.inf)
        hi = np.full(3, -np.inf)
        for j in range(n):
            k = n if j == 0 else n - 1 - j
            for d in range(3):
                lo[d] = min(lo[d], ex.drift(x[j, d], k, 0))
                hi[d] = max(hi[d], ex.drift(x[j, d], k, 1))
        assert np.array_equal(np.r_[lo, hi], b), gen


def test_create_without_gpu_fails_loudly(ex):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(ex.FmmError):
        ex.Fmm(P=10)


def test_kernel_entry_points_fail_loudly_without_gpu(ex):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(ex.FmmError):
        ex.p2p(np.zeros((2, 4)), np.ones((3, 4)))


def test_forest_grouping_cuts_whole_size_classes(ex):
    """The batch's forest groups: whole size classes (floor(log2 n)) in increasing
    order, at most the asked number of groups, each near its share of the bodies;
    empty systems go to group 0."""
    rng = np.random.default_rng(7)
    sizes = np.exp(rng.uniform(np.log(2000), np.log(200_000), 512)).astype(np.int64)
    sizes[[3, 40]] = 0
    for k in (1, 2, 3, 4, 8):
        g = ex.forest_buckets(sizes, k)
        assert g.shape == sizes.shape and g.min() == 0 and g.max() < k
        cls = np.floor(np.log2(np.maximum(sizes, 1))).astype(int)
        live = sizes > 0
        for c in np.unique(cls[live]):          # a class is never split
            assert len(np.unique(g[live & (cls == c)])) == 1
        order = np.argsort(sizes[live], kind="stable")   # groups follow size order
        assert np.all(np.diff(g[live][order]) >= 0)
        assert np.all(g[~live] == 0)
    assert list(ex.forest_buckets([2000, 0, 200_000, 5000, 70_000, 3000, 150_000], 3)) == [0, 0, 1, 0, 0, 0, 1]
    assert list(ex.forest_buckets([0, 0], 4)) == [0, 0]
    assert len(ex.forest_buckets([], 2)) == 0
    with pytest.raises(ex.FmmError):
        ex.forest_buckets([5, -1], 2)
    with pytest.raises(ex.FmmError):
        ex.forest_buckets([5], 0)
