"""The MD ABI of include/exafmm_md_distributed.h (the reference's distributed MD
wrapper shape, wrappers/md_distributed.cxx) through the C symbols of
libexafmm_md_distributed.so, in the order wrappers/test_md_distributed.cxx calls
them: FMM_Init -> FMM_Partition -> FMM_FMM, FMM_Ewald, FMM_Cutoff, and Set_Index,
Dipole_Correction.  The solve, Set_Index's tree and the Ewald sums are pinned to
the reference's own run of the same recipe (tests/golden/md_distributed.npz); the
ghost bodies, the group labels, the cutoff sum and the float dipole correction are
restated here from the wrapper's source."""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

pytestmark = pytest.mark.gpu

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)
NIMAX = 20000


@pytest.fixture(scope="module")
def md(ex):
    L = ctypes.CDLL(ex.MD_DISTRIBUTED_LIB_PATH)
    L.FMM_Init.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_bool,
                           ctypes.c_char_p]
    L.FMM_Finalize.argtypes = []
    L.Set_Index.argtypes = [_i, ctypes.c_int, _i, _d, _d, _d, _d]
    L.FMM_Partition.argtypes = [_i, ctypes.c_int, _i, _d, _d, _d, _d]
    L.FMM_FMM.argtypes = [ctypes.c_int, _i, _i, _d, _d, _d, _d, _d]
    L.FMM_Ewald.argtypes = [ctypes.c_int, _d, _d, _d, _d, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                            ctypes.c_double, _d]
    L.Dipole_Correction.argtypes = [ctypes.c_int, _d, _d, _d, _d, _d]
    L.FMM_Cutoff.argtypes = [ctypes.c_int, _d, _d, _d, _d, ctypes.c_double, _d]
    L.FMM_Error.restype = ctypes.c_char_p
    for fn in (L.FMM_Init, L.FMM_Finalize, L.Set_Index, L.FMM_Partition, L.FMM_FMM, L.FMM_Ewald,
               L.Dipole_Correction, L.FMM_Cutoff):
        fn.restype = None
    return L


@pytest.fixture(scope="module")
def gold():
    with np.load(os.path.join(GOLDEN, "md_distributed.npz")) as z:
        return {k: z[k] for k in z.files}


def _p(a, t=_d):
    return a.ctypes.data_as(t)


def _wrap(x, w):
    """vec.h:217-229 per dimension; returns the wrapped copy and the wrap codes."""
    X = x.copy()
    iw = np.zeros(len(x), np.int32)
    for d in range(3):
        lo = X[:, d] < -w[d] / 2
        X[lo, d] += w[d]
        hi = X[:, d] > w[d] / 2
        X[hi, d] -= w[d]
        iw |= ((lo | hi).astype(np.int32) << d)
    return X, iw


def _unwrap(X, w, iw):
    X = X.copy()
    for d in range(3):
        m = ((iw >> d) & 1).astype(bool)
        X[m, d] += np.where(X[m, d] > 0, -w[d], w[d])
    return X


def _arrays(n, x, q, v):
    """Caller arrays of NIMAX slots, as the reference's driver allocates them."""
    xa = np.zeros(3 * NIMAX)
    xa[:3 * n] = x.reshape(-1)
    qa = np.zeros(NIMAX)
    qa[:n] = q
    va = np.zeros(3 * NIMAX)
    va[:3 * n] = v.reshape(-1)
    return xa, qa, va


def _ghosts(X, q, res, bounds, cutoff, cycle):
    """md_distributed.cxx:274-298 for one rank: each body (in the given order) at
    each of the 26 neighbouring images strictly inside bounds +- cutoff."""
    gx, gq, gr = [], [], []
    for ix in (-1, 0, 1):
        for iy in (-1, 0, 1):
            for iz in (-1, 0, 1):
                if ix == iy == iz == 0:
                    continue
                Y = X + np.array([ix, iy, iz]) * cycle
                m = np.all((bounds[:3] - cutoff < Y) & (Y < bounds[3:] + cutoff), axis=1)
                gx.append(Y[m])
                gq.append(q[m])
                gr.append(res[m])
    return np.concatenate(gx), np.concatenate(gq), np.concatenate(gr)


def _cutoff_sum(xt, xs, qs, cutoff):
    """test_md_distributed.cxx's check sum: every source closer than the cutoff,
    p = sum q/r, f = -sum dx q/r^3."""
    d = xt[:, None, :] - xs[None, :, :]
    r2 = np.sum(d * d, axis=2)
    m = (r2 < cutoff * cutoff) & (r2 > 0)
    inv = np.zeros_like(r2)
    inv[m] = 1 / np.sqrt(r2[m])
    p = np.sum(qs[None, :] * inv, axis=1)
    f = -np.sum(d * (qs[None, :] * inv ** 3)[:, :, None], axis=1)
    return p, f


def _image_sum(x, q, cycle, cutoff, prange, float_shift):
    """md_distributed.cxx:407-461 restated: for each image -prange..prange per
    direction, dx = (x_i - x_j) - shift with the shift rounded to float there
    (float_shift) or exact; pairs closer than the cutoff."""
    p = np.zeros(len(q))
    f = np.zeros((len(q), 3))
    r = range(-prange, prange + 1)
    for ix in r:
        for iy in r:
            for iz in r:
                sh = np.array([ix * cycle[0], iy * cycle[1], iz * cycle[2]])
                if float_shift:
                    sh = sh.astype(np.float32).astype(np.float64)
                d = (x[:, None, :] - x[None, :, :]) - sh
                r2 = np.sum(d * d, axis=2)
                m = (r2 < cutoff * cutoff) & (r2 > 0)
                inv = np.zeros_like(r2)
                inv[m] = 1 / np.sqrt(r2[m])
                p += np.sum(q[None, :] * inv, axis=1)
                f -= np.sum(d * (q[None, :] * inv ** 3)[:, :, None], axis=1)
    return p, f


def test_partition_fmm_ghosts_ewald_cutoff(md, gold, tmp_path):
    x0, q0 = gold["x"], gold["q"]
    n = len(q0)
    c = float(gold["cycle"][0])
    cycle = np.full(3, c)
    cutoff = c / 2
    perm = gold["perm"]
    rng = np.random.default_rng(9)
    v0 = rng.standard_normal((n, 3))
    xa, qa, va = _arrays(n, x0, q0, v0)
    res = np.zeros(NIMAX, np.int32)
    res[:n] = np.arange(n) + 100
    md.FMM_Init(3, 16, 0.4, cutoff, False, (str(tmp_path) + "/").encode())
    ni = ctypes.c_int(n)
    md.FMM_Partition(ctypes.byref(ni), NIMAX, _p(res, _i), _p(xa), _p(qa), _p(va), _p(cycle))
    assert md.FMM_Error() == b""
    # bodies in the reference tree's order, positions wrapped then unwrapped as there
    assert ni.value == n
    np.testing.assert_array_equal(res[:n], perm + 100)
    Xw, iw = _wrap(x0, cycle)
    np.testing.assert_array_equal(xa[:3 * n].reshape(-1, 3), _unwrap(Xw, cycle, iw)[perm])
    np.testing.assert_array_equal(qa[:n], q0[perm])
    np.testing.assert_array_equal(va[:3 * n].reshape(-1, 3), v0[perm])

    x = xa[:3 * n].reshape(-1, 3).copy()
    q = qa[:n].copy()
    r = res[:n].copy()
    p = np.zeros(n)
    f = np.zeros(3 * n)
    nj = ctypes.c_int(NIMAX)
    md.FMM_FMM(n, ctypes.byref(nj), _p(res, _i), _p(xa), _p(qa), _p(p), _p(f), _p(cycle))
    assert md.FMM_Error() == b""
    ref = gold["fmm_trg"][perm]  # the reference's FP64 results, in the partitioned order
    assert rel_l2(p, ref[:, 0]) < 1e-10
    assert rel_l2(f.reshape(-1, 3), ref[:, 1:]) < 1e-10
    # the ghosts: the 26 images of the wrapped bodies inside the local bounds + cutoff
    Xs, _ = _wrap(x, cycle)
    gx, gq, gr = _ghosts(Xs, q, r, gold["bounds"], cutoff, cycle)
    assert nj.value == n + len(gq)
    np.testing.assert_array_equal(xa[3 * n:3 * nj.value].reshape(-1, 3), gx)
    np.testing.assert_array_equal(qa[n:nj.value], gq)
    np.testing.assert_array_equal(res[n:nj.value], gr)
    np.testing.assert_array_equal(xa[:3 * n].reshape(-1, 3), x)  # the bodies' own slots untouched

    # test_md_distributed.cxx's last check: the cutoff sum over bodies + ghosts
    # against FMM_Cutoff.  The ghosts hold every image a body sees within the
    # cutoff (the exact-shift image sum, to rounding); FMM_Cutoff shifts by
    # float-rounded periods as the reference does, 1e-7 away here.
    pc, fc = _cutoff_sum(Xs, np.concatenate([Xs, gx]), np.concatenate([q, gq]), cutoff)
    pi_, fi_ = _image_sum(Xs, q, cycle, cutoff, 1, float_shift=False)
    assert rel_l2(pc, pi_) < 1e-12 and rel_l2(fc, fi_) < 1e-12
    p2 = np.zeros(n)
    f2 = np.zeros(3 * n)
    xs = np.ascontiguousarray(Xs.reshape(-1))
    md.FMM_Cutoff(n, _p(xs), _p(q), _p(p2), _p(f2), cutoff, _p(cycle))
    assert md.FMM_Error() == b""
    pf, ff = _image_sum(Xs, q, cycle, cutoff, 1, float_shift=True)
    assert rel_l2(p2, pf) < 1e-12
    assert rel_l2(f2.reshape(-1, 3), ff) < 1e-12
    assert rel_l2(p2, pc) < 1e-6
    assert rel_l2(f2.reshape(-1, 3), fc) < 1e-6

    # Ewald in the caller's order
    pe = np.zeros(n)
    fe = np.zeros(3 * n)
    xc = np.ascontiguousarray(x.reshape(-1))
    md.FMM_Ewald(n, _p(xc), _p(q), _p(pe), _p(fe), 11, 10 / c, 0.25 / np.pi, cutoff, _p(cycle))
    assert md.FMM_Error() == b""
    enear = gold["ewald_nearest_trg"][perm]
    assert rel_l2(pe, enear[:, 0]) < 1e-9
    assert rel_l2(fe.reshape(-1, 3), enear[:, 1:]) < 1e-9
    eref = gold["ewald_trg"][perm]  # cell images at cutoff L/2 (include/ewald.h:120-133)
    assert rel_l2(pe, eref[:, 0]) < 2e-5
    assert rel_l2(fe.reshape(-1, 3), eref[:, 1:]) < 2e-5
    # the driver's FMM-vs-Ewald check, as close as the reference's own pair
    e_fmm, e_ew = float(np.sum(p * q)), float(np.sum(pe * q))
    e_ref = abs(float(np.sum(gold["fmm_trg"][:, 0] * q0) - np.sum(gold["ewald_trg"][:, 0] * q0)))
    assert abs(e_fmm - e_ew) <= e_ref * 1.01 + 1e-5 * abs(e_ew)

    # FMM_FMM accumulates into p and f; too small an nj leaves the ghost slots alone
    res[n:] = -7
    nj = ctypes.c_int(n + 5)
    md.FMM_FMM(n, ctypes.byref(nj), _p(res, _i), _p(xa), _p(qa), _p(p), _p(f), _p(cycle))
    assert nj.value == n + len(gq)
    assert np.all(res[n:] == -7)
    assert rel_l2(p, 2 * ref[:, 0]) < 1e-10
    md.FMM_Finalize()


def test_set_index_groups_from_drand48(md, gold, tmp_path):
    libc = ctypes.CDLL(None)
    libc.drand48.restype = ctypes.c_double
    libc.srand48.argtypes = [ctypes.c_long]
    x0, q0 = gold["x"], gold["q"]
    n = len(q0)
    c = float(gold["cycle"][0])
    cycle = np.full(3, c)
    cells = gold["index_cells"]  # IPARENT, ICHILD, NCHILD, IBODY, NBODY of the reference tree
    perm = gold["index_perm"]
    # md_distributed.cxx:113-124 with the same drand48 sequence
    libc.srand48(12345)
    draws = iter([libc.drand48() for _ in range(int(cells[:, 4].sum()))])
    label = np.zeros(n, np.int64)
    nid = 0
    for cb in cells:
        ic = 0
        for k in range(cb[3], cb[3] + cb[4]):
            if (next(draws) > 0.5 and ic > 2) or ic > 5:
                ic = 0
            if ic == 0:
                label[k] = nid
                nid += 1
            else:
                label[k] = -ic
            ic += 1
    v0 = np.random.default_rng(3).standard_normal((n, 3))
    xa, qa, va = _arrays(n, x0, q0, v0)
    res = np.zeros(NIMAX, np.int32)
    md.FMM_Init(3, 16, 0.4, c / 2, False, (str(tmp_path) + "/").encode())
    ni = ctypes.c_int(n)
    libc.srand48(12345)
    md.Set_Index(ctypes.byref(ni), NIMAX, _p(res, _i), _p(xa), _p(qa), _p(va), _p(cycle))
    assert md.FMM_Error() == b""
    assert ni.value == n
    np.testing.assert_array_equal(res[:n], label)
    assert label.min() < 0 and (label >= 0).sum() < n  # groups of several bodies formed
    Xw, iw = _wrap(x0, cycle)
    np.testing.assert_array_equal(xa[:3 * n].reshape(-1, 3), _unwrap(Xw, cycle, iw)[perm])
    np.testing.assert_array_equal(qa[:n], q0[perm])
    np.testing.assert_array_equal(va[:3 * n].reshape(-1, 3), v0[perm])
    # nimax not above ni: nothing written back
    res2 = np.full(n, -9, np.int32)
    x2 = x0.reshape(-1).copy()
    md.Set_Index(ctypes.byref(ni), n, _p(res2, _i), _p(x2), _p(q0.copy()), _p(v0.reshape(-1).copy()), _p(cycle))
    assert np.all(res2 == -9) and np.array_equal(x2, x0.reshape(-1))
    md.FMM_Finalize()


def test_cutoff_sum_matches_restatement(md):
    """md_distributed.cxx:407-461 restated: images out to the cutoff per
    direction, shifts rounded to float, every pair closer than the cutoff."""
    rng = np.random.default_rng(21)
    n = 300
    cycle = np.array([2 * np.pi, 2.2 * np.pi, 1.8 * np.pi])
    x = (rng.uniform(size=(n, 3)) - 0.5) * cycle
    q = rng.uniform(size=n) - 0.5
    cutoff = 6.0
    prange = int(cutoff / cycle.min() * 0.999999) + 1
    assert prange == 2
    p0 = rng.uniform(size=n)
    f0 = rng.standard_normal(3 * n)
    pp, ff = _image_sum(x, q, cycle, cutoff, prange, float_shift=True)
    pr, fr = p0 + pp, f0.reshape(-1, 3) + ff
    p = p0.copy()
    f = f0.copy()
    md.FMM_Cutoff(n, _p(np.ascontiguousarray(x.reshape(-1))), _p(q), _p(p), _p(f), cutoff, _p(cycle))
    assert md.FMM_Error() == b""
    assert rel_l2(p, pr) < 1e-12
    assert rel_l2(f.reshape(-1, 3), fr) < 1e-12


def test_dipole_correction_float_arithmetic(md):
    """md_distributed.cxx:383-405: dipole summed in float, |d|^2 of float squares
    in double, float coefficient; bit for bit."""
    rng = np.random.default_rng(22)
    n = 500
    cycle = np.array([5.0, 6.0, 7.0])
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
    md.Dipole_Correction(n, _p(np.ascontiguousarray(x.reshape(-1))), _p(q), _p(p), _p(f), _p(cycle))
    assert md.FMM_Error() == b""
    np.testing.assert_array_equal(p, pr)
    np.testing.assert_array_equal(f.reshape(-1, 3), fr)


def test_errors_leave_outputs_untouched(md):
    md.FMM_Finalize()
    n = 4
    x = np.zeros(3 * n)
    q = np.ones(n)
    p = np.ones(n)
    f = np.ones(3 * n)
    res = np.arange(n, dtype=np.int32)
    cycle = np.full(3, 1.0)
    nj = ctypes.c_int(100)
    md.FMM_FMM(n, ctypes.byref(nj), _p(res, _i), _p(x), _p(q), _p(p), _p(f), _p(cycle))
    assert b"FMM_Init" in md.FMM_Error()
    md.FMM_Init(1, 1, 0.5, 0.2, False, b"./")
    md.FMM_FMM(n, ctypes.byref(nj), _p(res, _i), _p(x), _p(q), _p(p), _p(f), _p(cycle))
    assert b"FMM_Partition" in md.FMM_Error()
    x = np.random.default_rng(1).uniform(-0.5, 0.5, 3 * n)
    v = np.zeros(3 * n)
    ni = ctypes.c_int(n)
    md.FMM_Partition(ctypes.byref(ni), 100, _p(res, _i), _p(x), _p(q), _p(v), _p(cycle))
    assert md.FMM_Error() == b""
    box = np.array([1.0, 1.0, 2.0])
    md.FMM_FMM(n, ctypes.byref(nj), _p(res, _i), _p(x), _p(q), _p(p), _p(f), _p(box))
    assert b"cubic" in md.FMM_Error()
    assert np.all(p == 1) and np.all(f == 1) and nj.value == 100
    md.FMM_Finalize()
