"""The MD ABI of include/exafmm_md.h (the reference's GROMACS wrapper shape,
wrappers/gromacs.cxx) through the C symbols of libexafmm_md_gromacs.so, as
wrappers/test_gromacs.cxx calls them: FMM_Init -> FMM_Partition -> FMM_Coulomb, Ewald_Coulomb, Direct_Coulomb.
Pinned to the reference's own solve of the same recipe (tests/golden/md_gromacs.npz)."""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

pytestmark = pytest.mark.gpu

_f = ctypes.POINTER(ctypes.c_float)
_i = ctypes.POINTER(ctypes.c_int)


@pytest.fixture(scope="module")
def md(ex):
    L = ctypes.CDLL(ex.MD_GROMACS_LIB_PATH)
    L.FMM_Init.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_bool, ctypes.c_char_p]
    L.FMM_Finalize.argtypes = []
    L.FMM_Partition.argtypes = [_i, _i, _i, _f, _f, ctypes.c_float]
    L.FMM_Coulomb.argtypes = [ctypes.c_int, _i, _f, _f, _f, _f, ctypes.c_float]
    L.Ewald_Coulomb.argtypes = [ctypes.c_int, _f, _f, _f, _f, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                ctypes.c_float, ctypes.c_float]
    L.Direct_Coulomb.argtypes = [ctypes.c_int, _f, _f, _f, _f, ctypes.c_float]
    L.FMM_Error.restype = ctypes.c_char_p
    for fn in (L.FMM_Init, L.FMM_Finalize, L.FMM_Partition, L.FMM_Coulomb, L.Ewald_Coulomb, L.Direct_Coulomb):
        fn.restype = None
    return L


@pytest.fixture(scope="module")
def gold():
    with np.load(os.path.join(GOLDEN, "md_gromacs.npz")) as z:
        return {k: z[k] for k in z.files}


def _p(a, t):
    return a.ctypes.data_as(t)


def test_partition_coulomb_ewald_match_reference(md, gold, tmp_path):
    n0 = len(gold["q"])
    x = gold["x"].copy()
    q = gold["q"].copy()
    cycle = np.float32(gold["cycle"][0])
    ibody = np.arange(n0, dtype=np.int32)
    icell = ibody.copy()
    md.FMM_Init(3, 16, False, (str(tmp_path) + "/").encode())
    n = ctypes.c_int(n0)
    md.FMM_Partition(ctypes.byref(n), _p(ibody, _i), _p(icell, _i), _p(x, _f), _p(q, _f), cycle)
    assert md.FMM_Error() == b""
    # bodies in the reference tree's order: a permutation of the input, positions restored exactly
    assert n.value == n0
    np.testing.assert_array_equal(ibody, gold["perm"])
    np.testing.assert_array_equal(icell, gold["perm"])
    np.testing.assert_array_equal(x, gold["x"][gold["perm"]])
    np.testing.assert_array_equal(q, gold["q"][gold["perm"]])

    p = np.zeros(n0, np.float32)
    f = np.zeros(3 * n0, np.float32)
    md.FMM_Coulomb(n0, _p(icell, _i), _p(x, _f), _p(q, _f), _p(p, _f), _p(f, _f), cycle)
    assert md.FMM_Error() == b""
    ref = gold["fmm_trg"][ibody]  # the reference's results, in the partitioned order
    assert rel_l2(p, ref[:, 0]) < 1e-6
    assert rel_l2(f.reshape(-1, 3), ref[:, 1:]) < 1e-6

    pe = np.zeros(n0, np.float32)
    fe = np.zeros(3 * n0, np.float32)
    md.Ewald_Coulomb(n0, _p(x, _f), _p(q, _f), _p(pe, _f), _p(fe, _f), 11, np.float32(10 / cycle),
                     np.float32(0.25 / np.pi), np.float32(cycle / 2), cycle)
    assert md.FMM_Error() == b""
    # each pair at its nearest image within the cutoff (the oracle's Ewald)
    enear = gold["ewald_nearest_trg"][ibody]
    assert rel_l2(pe, enear[:, 0]) < 1e-6
    assert rel_l2(fe.reshape(-1, 3), enear[:, 1:]) < 1e-6
    # the reference's tree walk at cutoff L/2 gives some pairs their cells' image
    # instead (include/ewald.h:120-133): a few 1e-6 of difference
    eref = gold["ewald_trg"][ibody]
    assert rel_l2(pe, eref[:, 0]) < 2e-5
    assert rel_l2(fe.reshape(-1, 3), eref[:, 1:]) < 2e-5

    # wrappers/test_gromacs.cxx's check: FMM against Ewald, as close as the reference's own pair
    e_fmm, e_ew = float(np.sum(p * q)), float(np.sum(pe * q))
    e_ref = abs(float(np.sum(gold["fmm_trg"][:, 0] * gold["q"]) - np.sum(gold["ewald_trg"][:, 0] * gold["q"])))
    assert abs(e_fmm - e_ew) <= e_ref * 1.01 + 1e-5 * abs(e_ew)
    assert rel_l2(f.reshape(-1, 3), fe.reshape(-1, 3)) < 2e-3

    # FMM_Coulomb accumulates into p and f
    md.FMM_Coulomb(n0, _p(icell, _i), _p(x, _f), _p(q, _f), _p(p, _f), _p(f, _f), cycle)
    assert rel_l2(p, 2 * ref[:, 0]) < 1e-6
    md.FMM_Finalize()


def _direct_reference(x, q, p, f, cycle, images):
    """wrappers/gromacs.cxx:289-363 restated in numpy: float separations, double sums,
    the dipole correction in float."""
    n = len(q)
    prange = sum(3 ** i for i in range(images))
    xs = x.reshape(-1, 3)
    pp = np.zeros(n)
    fx = np.zeros((n, 3))
    rng = np.arange(-prange, prange + 1, dtype=np.float32)
    for ix in rng:
        for iy in rng:
            for iz in rng:
                per = np.array([ix * cycle, iy * cycle, iz * cycle], np.float32)
                d = ((xs[:, None, :] - xs[None, :, :]) - per).astype(np.float32).astype(np.float64)
                r2 = np.sum(d * d, axis=2)
                with np.errstate(divide="ignore"):
                    inv = np.where(r2 == 0, 0.0, 1 / np.sqrt(r2))
                inv3 = q.astype(np.float64)[None, :] * inv ** 3
                pp += np.sum(q.astype(np.float64)[None, :] * inv, axis=1)
                fx += np.sum(d * inv3[:, :, None], axis=1)
    p = (p.astype(np.float64) + pp).astype(np.float32)
    f = (f.reshape(-1, 3).astype(np.float64) - fx).astype(np.float32)
    dip = np.zeros(3, np.float32)
    for i in range(n):
        dip += xs[i] * q[i]
    norm = float(np.sum((dip * dip).astype(np.float32).astype(np.float64)))
    coef = np.float32(4 * np.pi / (3 * float(cycle) ** 3))
    p = (p.astype(np.float64) - float(coef) * norm / n / q.astype(np.float64)).astype(np.float32)
    f = f - coef * dip[None, :]
    return p, f.reshape(-1)


def test_direct_coulomb_matches_restatement(md, tmp_path):
    rng = np.random.default_rng(5)
    n = 120
    cycle = np.float32(2 * np.pi)
    x = (rng.uniform(size=(n, 3)) * cycle - cycle / 2).astype(np.float32).reshape(-1)
    q = (rng.uniform(size=n) - 0.5).astype(np.float32)
    q -= np.float32(q.mean())
    p = rng.uniform(size=n).astype(np.float32)  # accumulated into
    f = np.zeros(3 * n, np.float32)
    pr, fr = _direct_reference(x, q, p.copy(), f.copy(), cycle, images=1)
    md.FMM_Init(1, 1, False, b"./")
    md.Direct_Coulomb(n, _p(x, _f), _p(q, _f), _p(p, _f), _p(f, _f), cycle)
    assert md.FMM_Error() == b""
    md.FMM_Finalize()
    assert rel_l2(p, pr) < 1e-6
    assert rel_l2(f, fr) < 1e-5


def test_errors_leave_outputs_untouched(md):
    md.FMM_Finalize()
    p = np.ones(4, np.float32)
    f = np.ones(12, np.float32)
    x = np.zeros(12, np.float32)
    q = np.ones(4, np.float32)
    icell = np.arange(4, dtype=np.int32)
    md.FMM_Coulomb(4, _p(icell, _i), _p(x, _f), _p(q, _f), _p(p, _f), _p(f, _f), np.float32(1.0))
    assert b"FMM_Init" in md.FMM_Error()
    md.FMM_Init(2, 1, False, b"./")
    md.FMM_Coulomb(4, _p(icell, _i), _p(x, _f), _p(q, _f), _p(p, _f), _p(f, _f), np.float32(1.0))
    assert b"FMM_Partition" in md.FMM_Error()
    icell[2] = -1
    n = ctypes.c_int(4)
    ibody = np.arange(4, dtype=np.int32)
    md.FMM_Partition(ctypes.byref(n), _p(ibody, _i), _p(icell, _i), _p(x, _f), _p(q, _f), np.float32(1.0))
    assert b"ICELL < 0" in md.FMM_Error()
    assert np.all(p == 1) and np.all(f == 1)
    md.FMM_Finalize()
