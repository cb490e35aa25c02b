"""ctypes bindings for the two CPU checkers (test infrastructure only).

* ``Oracle``    -- liboracle.so, the plain-C restatement (oracle/exafmm_oracle.c).
* ``Reference`` -- _ref/libexafmm_ref.so, the exafmm-beta headers compiled in
  place (oracle/ref_harness.cxx); present only where it was built.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
import this module.  The product library never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libexafmm_ref.so")

_c_int, _c_double, _vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p


EXAMPLES_DIR = os.path.join(HERE, "_ref", "examples")


def build(reference_root: str | None = None, examples: bool = True) -> None:
    """Compile liboracle.so and, when reference_root names an exafmm-beta
    source tree that exists, the reference harness compiled in place from it
    and (examples=True, the engine library built first) the reference's own
    example drivers compiled against the facade into _ref/examples/."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if reference_root and os.path.isdir(os.path.join(reference_root, "include")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE_ROOT={reference_root}"], check=True)
        if examples:
            subprocess.run(["make", "-s", "-C", HERE, "examples", f"REFERENCE_ROOT={reference_root}"], check=True)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_vp)


def _as_xyzq(x) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.float64)
    assert a.ndim == 2 and a.shape[1] == 4
    return a


@dataclass
class TreeRun:
    """Outputs of one CPU solve, in the conventions of exafmm_oracle.h."""
    bounds: np.ndarray
    perm: np.ndarray
    cells_int: np.ndarray
    cells_real: np.ndarray
    m2l: np.ndarray | None
    p2p: np.ndarray | None
    trg: np.ndarray | None
    M: np.ndarray | None
    L: np.ndarray | None
    times: np.ndarray | None = None
    icell: np.ndarray | None = None   # Cell::ICELL (the reference only)


class _Lib:
    prefix = ""

    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self._sig()

    def _f(self, name, res, args):
        fn = getattr(self.lib, self.prefix + name)
        fn.restype = res
        fn.argtypes = args
        return fn

    def _sig(self):
        p = self._f
        p("num_cells", _c_int, [_vp])
        p("num_m2l", _c_int, [_vp])
        p("num_p2p", _c_int, [_vp])
        p("get_bounds", None, [_vp, _vp])
        p("get_trg", None, [_vp, _vp])
        p("get_perm", None, [_vp, _vp])
        p("get_lists", None, [_vp, _vp, _vp])
        p("get_expansions", None, [_vp, _vp, _vp])
        p("free", None, [_vp])
        p("p2m", None, [_c_int, _vp, _c_int, _vp, _vp] if self.prefix == "oracle_" else
          [_c_int, _vp, _c_double, _c_int, _vp, _vp])
        p("m2m", None, [_c_int, _vp, _c_int, _vp, _vp, _vp])
        p("m2l", None, [_c_int, _vp, _vp, _vp, _vp, _vp])
        p("l2l", None, [_c_int, _vp, _vp, _vp, _vp])
        p("l2p", None, [_c_int, _vp, _vp, _c_int, _vp, _vp])
        p("p2p", None, [_c_int, _vp, _c_int, _vp, _vp, _vp])
        p("direct", None, [_c_int, _vp, _c_int, _vp, _c_int, _c_double, _c_double, _vp])
        if self.prefix == "oracle_":
            p("ewald", None, [_c_int, _vp, _c_int, _c_double, _c_double, _c_double, _c_double, _vp])
        else:
            p("ewald", None, [_c_int, _vp, _c_int, _c_double, _c_double, _c_double, _c_double, _c_int, _vp])

    def _collect(self, h, n, P, lists=True, trg=True, expansions=False) -> TreeRun:
        g = lambda name: getattr(self.lib, self.prefix + name)
        nc = g("num_cells")(h)
        bounds = np.zeros(6)
        g("get_bounds")(h, _ptr(bounds))
        perm = np.zeros(n, dtype=np.int32)
        g("get_perm")(h, _ptr(perm))
        ci = np.zeros((nc, 5), dtype=np.int32)
        cr = np.zeros((nc, 4))
        self._get_cells(h, ci, cr)
        m2l = p2p = t = M = L = None
        if lists:
            m2l = np.zeros((g("num_m2l")(h), 2), dtype=np.int32)
            p2p = np.zeros((g("num_p2p")(h), 2), dtype=np.int32)
            g("get_lists")(h, _ptr(m2l), _ptr(p2p))
        if trg:
            t = np.zeros((n, 4))
            g("get_trg")(h, _ptr(t))
        if expansions and P:
            nterm = P * (P + 1) // 2
            M = np.zeros((nc, nterm), dtype=np.complex128)
            L = np.zeros((nc, nterm), dtype=np.complex128)
            g("get_expansions")(h, _ptr(M), _ptr(L))
        return TreeRun(bounds, perm, ci, cr, m2l, p2p, t, M, L)

    # ---- per-operator forms: expansions are complex128 arrays of NTERM ----
    def m2m(self, P, Xp, Xc, Mc, Mp=None):
        Xc = np.ascontiguousarray(Xc, dtype=np.float64).reshape(-1, 3)
        Mc = np.ascontiguousarray(Mc, dtype=np.complex128).reshape(len(Xc), -1)
        out = np.zeros(P * (P + 1) // 2, np.complex128) if Mp is None else np.array(Mp, np.complex128)
        getattr(self.lib, self.prefix + "m2m")(P, _ptr(np.asarray(Xp, np.float64)), len(Xc), _ptr(Xc), _ptr(Mc), _ptr(out))
        return out

    def m2l(self, P, Xi, Xj, Mj, Li=None, Xper=None):
        out = np.zeros(P * (P + 1) // 2, np.complex128) if Li is None else np.array(Li, np.complex128)
        Mj = np.ascontiguousarray(Mj, dtype=np.complex128)
        xp = None if Xper is None else np.asarray(Xper, np.float64)
        getattr(self.lib, self.prefix + "m2l")(P, _ptr(np.asarray(Xi, np.float64)), _ptr(np.asarray(Xj, np.float64)),
                                               _ptr(Mj), _ptr(out), _ptr(xp))
        return out

    def l2l(self, P, Xc, Xp, Lp, Lc=None):
        out = np.zeros(P * (P + 1) // 2, np.complex128) if Lc is None else np.array(Lc, np.complex128)
        Lp = np.ascontiguousarray(Lp, dtype=np.complex128)
        getattr(self.lib, self.prefix + "l2l")(P, _ptr(np.asarray(Xc, np.float64)), _ptr(np.asarray(Xp, np.float64)),
                                               _ptr(Lp), _ptr(out))
        return out

    def l2p(self, P, X, L, xyzq, trg=None):
        xyzq = _as_xyzq(xyzq)
        out = np.zeros((len(xyzq), 4)) if trg is None else np.array(trg, np.float64)
        L = np.ascontiguousarray(L, dtype=np.complex128)
        getattr(self.lib, self.prefix + "l2p")(P, _ptr(np.asarray(X, np.float64)), _ptr(L), len(xyzq), _ptr(xyzq), _ptr(out))
        return out

    def p2p(self, xi, xj, Xper=None, trg=None):
        xi, xj = _as_xyzq(xi), _as_xyzq(xj)
        out = np.zeros((len(xi), 4)) if trg is None else np.array(trg, np.float64)
        xp = None if Xper is None else np.asarray(Xper, np.float64)
        getattr(self.lib, self.prefix + "p2p")(len(xi), _ptr(xi), len(xj), _ptr(xj), _ptr(xp), _ptr(out))
        return out

    def ewald(self, xyzq, ksize, alpha, sigma, cutoff, cycle, ncrit=64):
        """Ewald summation (include/ewald.h): (n, 4) potential and gradient, caller order."""
        x = _as_xyzq(xyzq)
        out = np.zeros((len(x), 4))
        if self.prefix == "oracle_":
            self.lib.oracle_ewald(len(x), _ptr(x), ksize, alpha, sigma, cutoff, cycle, _ptr(out))
        else:
            self.lib.ref_ewald(len(x), _ptr(x), ksize, alpha, sigma, cutoff, cycle, ncrit, _ptr(out))
        return out

    def direct(self, xi, xj, images=0, theta=0.4, cycle=2 * np.pi):
        xi, xj = _as_xyzq(xi), _as_xyzq(xj)
        out = np.zeros((len(xi), 4))
        getattr(self.lib, self.prefix + "direct")(len(xi), _ptr(xi), len(xj), _ptr(xj), images, theta, cycle, _ptr(out))
        return out


class Oracle(_Lib):
    prefix = "oracle_"

    def __init__(self, path: str = ORACLE_SO):
        build()  # incremental; keeps the .so in step with exafmm_oracle.c
        super().__init__(path)

    def _sig(self):
        super()._sig()
        self._f("bounds", None, [_c_int, _vp, _vp])
        self._f("solve", _vp, [_c_int, _vp, _c_int, _c_double, _c_int, _c_int, _c_int, _c_double, _vp, _c_int])
        self._f("build_tree", _vp, [_c_int, _vp, _c_int, _vp])
        self._f("get_cells", None, [_vp, _vp, _vp])
        self._f("depth", _c_int, [_vp])
        self._f("drift_seq", _c_double, [_c_double, ctypes.c_longlong, _c_int])

    def _get_cells(self, h, ci, cr):
        self.lib.oracle_get_cells(h, _ptr(ci), _ptr(cr))

    def drift_seq(self, x: float, k: int, up: bool = False) -> float:
        return self.lib.oracle_drift_seq(float(x), int(k), int(up))

    def bounds(self, xyzq) -> np.ndarray:
        xyzq = _as_xyzq(xyzq)
        out = np.zeros(6)
        self.lib.oracle_bounds(len(xyzq), _ptr(xyzq), _ptr(out))
        return out

    def solve(self, xyzq, P=10, theta=0.4, ncrit=64, nspawn=5000, images=0, cycle=2 * np.pi,
              bounds=None, dipole_correction=False, expansions=False) -> TreeRun:
        xyzq = _as_xyzq(xyzq)
        b = None if bounds is None else np.asarray(bounds, np.float64)
        h = self.lib.oracle_solve(len(xyzq), _ptr(xyzq), P, theta, ncrit, nspawn, images, cycle, _ptr(b),
                                  int(dipole_correction))
        try:
            return self._collect(h, len(xyzq), P, expansions=expansions)
        finally:
            self.lib.oracle_free(h)

    def build_tree(self, xyzq, ncrit=64, bounds=None) -> TreeRun:
        xyzq = _as_xyzq(xyzq)
        b = None if bounds is None else np.asarray(bounds, np.float64)
        h = self.lib.oracle_build_tree(len(xyzq), _ptr(xyzq), ncrit, _ptr(b))
        try:
            return self._collect(h, len(xyzq), 0, lists=False, trg=False)
        finally:
            self.lib.oracle_free(h)

    def p2m(self, P, X, xyzq, M=None):
        xyzq = _as_xyzq(xyzq)
        out = np.zeros(P * (P + 1) // 2, np.complex128) if M is None else np.array(M, np.complex128)
        self.lib.oracle_p2m(P, _ptr(np.asarray(X, np.float64)), len(xyzq), _ptr(xyzq), _ptr(out))
        return out


class Reference(_Lib):
    prefix = "ref_"

    def __init__(self, path: str = REF_SO):
        super().__init__(path)

    def _sig(self):
        super()._sig()
        self._f("run", _vp, [_c_int, _vp, _c_int, _c_double, _c_int, _c_int, _c_int, _c_double, _c_int, _c_int,
                             _vp, _c_int])
        self._f("get_cells", None, [_vp, _vp, _vp, _vp])
        self._f("get_times", None, [_vp, _vp])
        self._f("write_list", None, [_vp, ctypes.c_char_p])
        self._f("run_inej", _vp, [_c_int, _vp, _c_int, _vp, _c_int, _c_double, _c_int, _c_int, _c_int])
        self._f("num_jcells", _c_int, [_vp])
        self._f("get_jcells", None, [_vp, _vp, _vp, _vp])
        self._f("write_time", None, [_c_int, _vp, _vp, ctypes.c_char_p])

    def _get_cells(self, h, ci, cr):
        self.lib.ref_get_cells(h, _ptr(ci), _ptr(cr), None)

    def icell(self, h, nc):
        out = np.zeros(nc, dtype=np.uint64)
        ci = np.zeros((nc, 5), dtype=np.int32)
        cr = np.zeros((nc, 4))
        self.lib.ref_get_cells(h, _ptr(ci), _ptr(cr), _ptr(out))
        return out

    def write_time(self, events: dict, path: str) -> None:
        """logger::writeTime of `events` (name -> seconds) into path + 'time000000.dat'."""
        names = (ctypes.c_char_p * len(events))(*[k.encode() for k in events])
        vals = np.array(list(events.values()), dtype=np.float64)
        self.lib.ref_write_time(len(events), names, _ptr(vals), path.encode())

    def solve(self, xyzq, P=10, theta=0.4, ncrit=64, nspawn=5000, images=0, cycle=2 * np.pi,
              bounds=None, threads=1, record_lists=True, dipole_correction=False, expansions=False,
              list_path=None) -> TreeRun:
        """One solve; with list_path, also Traversal::writeList into list_path + 'list000000.dat'."""
        xyzq = _as_xyzq(xyzq)
        b = None if bounds is None else np.asarray(bounds, np.float64)
        h = self.lib.ref_run(len(xyzq), _ptr(xyzq), P, theta, ncrit, nspawn, images, cycle, threads,
                             int(record_lists), _ptr(b), int(dipole_correction))
        try:
            run = self._collect(h, len(xyzq), P, lists=record_lists, expansions=expansions)
            t = np.zeros(8)
            self.lib.ref_get_times(h, _ptr(t))
            run.times = t
            run.icell = self.icell(h, len(run.cells_int))
            if list_path is not None:
                self.lib.ref_write_list(h, list_path.encode())
            return run
        finally:
            self.lib.ref_free(h)

    def solve_inej(self, xyzq, jxyzq, P=10, theta=0.4, ncrit=64, nspawn=5000, record_lists=True):
        """examples/fmm.cxx with -j IneJ: targets xyzq, separate sources jxyzq (free space).
        Returns the target-side TreeRun and (jcells_int, jcells_real, jperm) of the source tree."""
        xyzq, jxyzq = _as_xyzq(xyzq), _as_xyzq(jxyzq)
        h = self.lib.ref_run_inej(len(xyzq), _ptr(xyzq), len(jxyzq), _ptr(jxyzq), P, theta, ncrit, nspawn,
                                  int(record_lists))
        try:
            run = self._collect(h, len(xyzq), P, lists=record_lists)
            nj = self.lib.ref_num_jcells(h)
            ji = np.zeros((nj, 5), dtype=np.int32)
            jr = np.zeros((nj, 4))
            jp = np.zeros(len(jxyzq), dtype=np.int32)
            self.lib.ref_get_jcells(h, _ptr(ji), _ptr(jr), _ptr(jp))
            return run, (ji, jr, jp)
        finally:
            self.lib.ref_free(h)

    def p2m(self, P, X, xyzq, M=None, R=1.0):
        xyzq = _as_xyzq(xyzq)
        out = np.zeros(P * (P + 1) // 2, np.complex128) if M is None else np.array(M, np.complex128)
        self.lib.ref_p2m(P, _ptr(np.asarray(X, np.float64)), R, len(xyzq), _ptr(xyzq), _ptr(out))
        return out


def reference_available() -> bool:
    return os.path.exists(REF_SO)
