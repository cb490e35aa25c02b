"""Host-side logic of the MD-code libraries that needs no GPU: the distributed
wrapper's float dipole correction (wrappers/md_distributed.cxx:383-405) bit for
bit, and the error convention of both wrappers for calls made before FMM_Init
(outputs untouched, the reason kept for FMM_Error).  CPU only."""
import ctypes

import numpy as np
import pytest

_d = ctypes.POINTER(ctypes.c_double)
_f = ctypes.POINTER(ctypes.c_float)
_i = ctypes.POINTER(ctypes.c_int)


def _p(a, t):
    return a.ctypes.data_as(t)


@pytest.fixture(scope="module")
def mdd(ex):
    L = ctypes.CDLL(ex.MD_DISTRIBUTED_LIB_PATH)
    L.Dipole_Correction.argtypes = [ctypes.c_int, _d, _d, _d, _d, _d]
    L.FMM_FMM.argtypes = [ctypes.c_int, _i, _i, _d, _d, _d, _d, _d]
    L.FMM_Ewald.argtypes = [ctypes.c_int, _d, _d, _d, _d, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                            ctypes.c_double, _d]
    L.FMM_Error.restype = ctypes.c_char_p
    for fn in (L.Dipole_Correction, L.FMM_FMM, L.FMM_Ewald):
        fn.restype = None
    return L


@pytest.fixture(scope="module")
def mdg(ex):
    L = ctypes.CDLL(ex.MD_GROMACS_LIB_PATH)
    L.FMM_Coulomb.argtypes = [ctypes.c_int, _i, _f, _f, _f, _f, ctypes.c_float]
    L.FMM_Error.restype = ctypes.c_char_p
    L.FMM_Coulomb.restype = None
    return L


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_dipole_correction_float_arithmetic(mdd, seed):
    rng = np.random.default_rng(seed)
    n = 400
    cycle = np.array([4.0, 5.5, 7.25]) * (1 + seed)
    x = (rng.uniform(size=(n, 3)) - 0.5) * cycle
    q = rng.uniform(size=n) - 0.5
    p = rng.uniform(size=n)
    f = rng.standard_normal(3 * n)
    dip = np.zeros(3, np.float32)
    for i in range(n):
        for d in range(3):
            dip[d] = np.float32(np.float64(dip[d]) + x[i, d] * q[i])
    norm = 0.0
    for d in range(3):
        norm += float(np.float32(dip[d] * dip[d]))
    coef = np.float32(4 * np.pi / (3 * cycle[0] * cycle[1] * cycle[2]))
    pr = p - float(coef) * norm / n / q
    fr = f.reshape(-1, 3) - (coef * dip).astype(np.float64)[None, :]
    mdd.Dipole_Correction(n, _p(np.ascontiguousarray(x.reshape(-1)), _d), _p(q, _d), _p(p, _d), _p(f, _d),
                          _p(cycle, _d))
    assert mdd.FMM_Error() == b""
    np.testing.assert_array_equal(p, pr)
    np.testing.assert_array_equal(f.reshape(-1, 3), fr)


def test_calls_before_init_leave_outputs(mdd, mdg):
    n = 3
    x = np.zeros(3 * n)
    q = np.ones(n)
    p = np.full(n, 7.0)
    f = np.full(3 * n, 7.0)
    res = np.arange(n, dtype=np.int32)
    nj = ctypes.c_int(50)
    cycle = np.full(3, 1.0)
    mdd.FMM_FMM(n, ctypes.byref(nj), _p(res, _i), _p(x, _d), _p(q, _d), _p(p, _d), _p(f, _d), _p(cycle, _d))
    assert b"FMM_Init" in mdd.FMM_Error()
    mdd.FMM_Ewald(n, _p(x, _d), _p(q, _d), _p(p, _d), _p(f, _d), 4, 1.0, 0.1, 0.5, _p(cycle, _d))
    assert b"FMM_Init" in mdd.FMM_Error()
    assert np.all(p == 7) and np.all(f == 7) and nj.value == 50
    xf = np.zeros(3 * n, np.float32)
    qf = np.ones(n, np.float32)
    pf = np.full(n, 7, np.float32)
    ff = np.full(3 * n, 7, np.float32)
    mdg.FMM_Coulomb(n, _p(res, _i), _p(xf, _f), _p(qf, _f), _p(pf, _f), _p(ff, _f), np.float32(1.0))
    assert b"FMM_Init" in mdg.FMM_Error()
    assert np.all(pf == 7) and np.all(ff == 7)
