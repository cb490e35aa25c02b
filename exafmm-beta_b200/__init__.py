"""Python binding of the B200 Laplace FMM engine (ctypes over include/exafmm_b200.h).

The engine itself is C++/CUDA (libexafmm_b200.so next to this file); this
module only marshals arrays.  There is no CPU fallback: if the shared library
is missing or no CUDA device is usable, the calls raise.

Typical use mirrors examples/fmm.cxx::

    fmm = Fmm(P=10, theta=0.4, ncrit=64)
    fmm.set_bodies(xyzq)          # (n, 4) float64: x, y, z, charge
    fmm.solve()                   # getBounds, buildTree, upward, traverse, downward
    trg = fmm.results()           # (n, 4): potential, grad x, grad y, grad z
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libexafmm_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "exafmm_b200.h")
MD_HEADER = os.path.join(os.path.dirname(HERE), "include", "exafmm_md.h")
MDD_HEADER = os.path.join(os.path.dirname(HERE), "include", "exafmm_md_distributed.h")
# The MD-code ABIs (wrappers/gromacs.cxx and wrappers/md_distributed.cxx shapes):
# separate libraries over libexafmm_b200.so, since their FMM_* names overlap.
MD_GROMACS_LIB_PATH = os.path.join(HERE, "libexafmm_md_gromacs.so")
MD_DISTRIBUTED_LIB_PATH = os.path.join(HERE, "libexafmm_md_distributed.so")

FP64 = 0
MIXED = 1

_c_int, _c_ll, _c_double, _vp = ctypes.c_int, ctypes.c_longlong, ctypes.c_double, ctypes.c_void_p
_lib = None


def build(force: bool = False) -> str:
    """Compile libexafmm_b200.so for sm_100a (nvcc cross-compiles without a GPU).
    make is incremental, so this is cheap when the library is current."""
    args = ["make", "-s", "-j8", "-C", os.path.join(HERE, "csrc")]
    if force:
        subprocess.run(args + ["clean"], check=True)
    subprocess.run(args, check=True)
    return LIB_PATH


def exported_symbols() -> list[str]:
    """Every function declared in include/exafmm_b200.h (libexafmm_b200.so)."""
    import re
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(exafmm_[a-z0-9_]+)\s*\(", text)))


def md_exported_symbols(header: str) -> list[str]:
    """Every function an MD-code ABI header (MD_HEADER or MDD_HEADER) declares."""
    import re
    text = open(header).read()
    return sorted(set(re.findall(r"^\s*(?:void|bool|int|const char \*)\s*([A-Za-z_]\w*)\s*\(", text, re.M)))


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run build() (or __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    sig = {
        "exafmm_create": (_c_int, [ctypes.POINTER(_vp), _c_int, _c_double, _c_int, _c_int, _c_int, _c_double,
                                   _c_int, _c_int]),
        "exafmm_destroy": (_c_int, [_vp]),
        "exafmm_last_error": (ctypes.c_char_p, [_vp]),
        "exafmm_create_error": (ctypes.c_char_p, []),
        "exafmm_kernel_error": (ctypes.c_char_p, []),
        "exafmm_set_bodies": (_c_int, [_vp, _vp, _c_ll]),
        "exafmm_set_bodies_device": (_c_int, [_vp, _vp, _c_ll]),
        "exafmm_get_bounds": (_c_int, [_vp, _vp]),
        "exafmm_build_tree": (_c_int, [_vp, _vp]),
        "exafmm_upward": (_c_int, [_vp]),
        "exafmm_traverse": (_c_int, [_vp]),
        "exafmm_downward": (_c_int, [_vp]),
        "exafmm_solve": (_c_int, [_vp]),
        "exafmm_get_results": (_c_int, [_vp, _vp]),
        "exafmm_get_results_device": (_c_int, [_vp, _vp]),
        "exafmm_tree_info": (_c_int, [_vp, ctypes.POINTER(_c_ll), ctypes.POINTER(_c_int), ctypes.POINTER(_c_ll),
                                      ctypes.POINTER(_c_ll)]),
        "exafmm_get_cells": (_c_int, [_vp, _vp, _vp]),
        "exafmm_get_perm": (_c_int, [_vp, _vp]),
        "exafmm_get_lists": (_c_int, [_vp, _vp, _vp]),
        "exafmm_get_expansions": (_c_int, [_vp, _vp, _vp]),
        "exafmm_stream": (_vp, [_vp]),
        "exafmm_phase_times": (_c_int, [_vp, _vp]),
        "exafmm_direct": (_c_int, [_vp, _c_ll, _vp, _c_ll, _c_int, _c_double, _c_double, _vp]),
        "exafmm_kernel_p2m": (_c_int, [_c_int, _vp, _c_ll, _vp, _vp]),
        "exafmm_kernel_m2m": (_c_int, [_c_int, _vp, _c_int, _vp, _vp, _vp]),
        "exafmm_kernel_m2l": (_c_int, [_c_int, _vp, _vp, _vp, _vp, _vp]),
        "exafmm_kernel_l2l": (_c_int, [_c_int, _vp, _vp, _vp, _vp]),
        "exafmm_kernel_l2p": (_c_int, [_c_int, _vp, _vp, _c_ll, _vp, _vp]),
        "exafmm_kernel_p2p": (_c_int, [_c_ll, _vp, _c_ll, _vp, _vp, _vp]),
        "exafmm_drift": (_c_double, [_c_double, _c_ll, _c_int]),
        "exafmm_launch_count": (_c_ll, []),
        "exafmm_set_params": (_c_int, [_vp, _c_int, _c_double, _c_int, _c_int, _c_int, _c_double]),
        "exafmm_set_mixed_policy": (_c_int, [_vp, _c_int, _c_int, _c_int, _c_int]),
        "exafmm_get_dipole": (_c_int, [_vp, _vp, _vp]),
        "exafmm_device_bytes": (_c_int, [_vp, ctypes.POINTER(_c_ll)]),
        "exafmm_batch_create": (_c_int, [ctypes.POINTER(_vp), _c_int, _c_double, _c_int, _c_int, _c_int, _c_int,
                                         _c_int]),
        "exafmm_batch_destroy": (_c_int, [_vp]),
        "exafmm_batch_error": (ctypes.c_char_p, [_vp]),
        "exafmm_batch_solve": (_c_int, [_vp, _c_int, _vp, _vp, _vp]),
        "exafmm_batch_times": (_c_int, [_vp, _vp]),
        "exafmm_batch_autotune": (_c_int, [_vp, _c_int]),
        "exafmm_batch_ncrit_table": (_c_int, [_vp, _vp, _c_int]),
        "exafmm_batch_set_ncrit_table": (_c_int, [_vp, _vp, _c_int]),
        "exafmm_batch_set_forest": (_c_int, [_vp, _c_int]),
        "exafmm_batch_set_mixed_policy": (_c_int, [_vp, _c_int, _c_int, _c_int, _c_int]),
        "exafmm_batch_elapsed": (_c_int, [_vp, _vp]),
        "exafmm_batch_buckets": (_c_int, [_vp, _vp, _vp, _c_int]),
        "exafmm_forest_buckets": (_c_int, [_c_int, _vp, _c_int, _vp]),
        "exafmm_server_create": (_c_int, [ctypes.POINTER(_vp), _c_int, _c_int, _c_double]),
        "exafmm_server_destroy": (_c_int, [_vp]),
        "exafmm_server_submit": (_c_int, [_vp, _vp, _c_ll, _vp, _c_int, _c_double, _c_int, _c_int, _c_int,
                                          ctypes.POINTER(_c_ll)]),
        "exafmm_server_poll": (_c_int, [_vp, _c_ll, ctypes.POINTER(_c_int)]),
        "exafmm_server_wait": (_c_int, [_vp, _c_ll, _vp]),
        "exafmm_server_stats": (_c_int, [_vp, _vp]),
        "exafmm_server_error": (ctypes.c_char_p, []),
        "exafmm_server_open_session": (_c_int, [_vp, _vp, _c_ll, _c_int, _c_double, _c_int, _c_int, _c_int,
                                                ctypes.POINTER(_c_ll)]),
        "exafmm_server_submit_step": (_c_int, [_vp, _c_ll, _c_double, ctypes.c_ulonglong, _vp, _vp,
                                               ctypes.POINTER(_c_ll)]),
        "exafmm_server_session_bodies": (_c_int, [_vp, _c_ll, _vp]),
        "exafmm_server_close_session": (_c_int, [_vp, _c_ll]),
        "exafmm_server_set_grouping": (_c_int, [_vp, _c_int, _c_ll, _c_ll]),
        "exafmm_list_work": (_c_int, [_vp, ctypes.POINTER(_c_ll)]),
        "exafmm_server_grouped": (_c_int, [_vp, ctypes.POINTER(_c_ll)]),
        "exafmm_server_set_mixed_policy": (_c_int, [_vp, _c_int, _c_int, _c_int, _c_int]),
        "exafmm_batch_set_ncrit_candidates": (_c_int, [_vp, _vp, _c_int]),
        "exafmm_batch_set_p2p_candidates": (_c_int, [_vp, _vp, _c_int]),
        "exafmm_batch_config_table": (_c_int, [_vp, _vp, _c_int]),
        "exafmm_batch_set_config_table": (_c_int, [_vp, _vp, _c_int]),
        "exafmm_batch_bucket_p2p": (_c_int, [_vp, _vp, _c_int]),
        "exafmm_set_p2p_targets_per_lane": (_c_int, [_vp, _c_int]),
        "exafmm_displace_bodies": (_c_int, [_vp, _c_double, ctypes.c_ulonglong]),
        "exafmm_get_bodies": (_c_int, [_vp, _vp]),
        "exafmm_get_bodies_device": (_c_int, [_vp, _vp]),
        "exafmm_ewald": (_c_int, [_vp, _c_ll, _c_int, _c_double, _c_double, _c_double, _c_double, _vp]),
        "exafmm_ewald_error": (ctypes.c_char_p, []),
        "exafmm_dipole_correction": (_c_int, [_vp, _vp, _c_ll]),
        "exafmm_set_sources": (_c_int, [_vp, _vp, _c_ll]),
        "exafmm_get_source_cells": (_c_int, [_vp, ctypes.POINTER(_c_ll), _vp, _vp, _vp]),
        "exafmm_direct_range": (_c_int, [_vp, _c_ll, _vp, _c_ll, _c_int, _c_double, _vp]),
        "exafmm_write_list": (_c_int, [_vp, ctypes.c_char_p, _c_int]),
        "exafmm_write_time": (_c_int, [_vp, ctypes.c_char_p, _c_int]),
        "exafmm_write_time_events": (_c_int, [ctypes.c_char_p, _c_int, _c_int, _vp, _vp]),
        "exafmm_morton_key": (ctypes.c_ulonglong, [_vp, _vp, _c_double, _c_int]),
        "exafmm_set_systems": (_c_int, [_vp, _c_int, _vp, _vp]),
        "exafmm_set_systems_device": (_c_int, [_vp, _c_int, _vp, _vp]),
        "exafmm_get_systems": (_c_int, [_vp, _vp, _vp, _vp]),
        "exafmm_set_systems_list": (_c_int, [_vp, _c_int, _vp, _vp]),
        "exafmm_get_results_list": (_c_int, [_vp, _vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(_vp)


def _f64(a, shape_last=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape_last is not None:
        assert a.shape[-1] == shape_last
    return a


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


class FmmError(RuntimeError):
    pass


class Fmm:
    """One solve context (a CUDA stream plus every device buffer of a solve)."""

    def __init__(self, P=10, theta=0.4, ncrit=64, nspawn=5000, images=0, cycle=2 * np.pi, precision=FP64,
                 device=-1):
        L = lib()
        h = _vp()
        if L.exafmm_create(ctypes.byref(h), P, theta, ncrit, nspawn, images, cycle, precision, device) != 0:
            raise FmmError(L.exafmm_create_error().decode())
        self._h = h
        self.P, self.theta, self.ncrit, self.nspawn, self.images, self.cycle = P, theta, ncrit, nspawn, images, cycle
        self.precision = precision
        self.n = 0
        self.nsys = 0

    def _check(self, rc):
        if rc != 0:
            raise FmmError(lib().exafmm_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            lib().exafmm_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_params(self, P=None, theta=None, ncrit=None, nspawn=None, images=None, cycle=None):
        """Change solve parameters between solves (unchanged ones keep their value)."""
        P = self.P if P is None else P
        theta = self.theta if theta is None else theta
        ncrit = self.ncrit if ncrit is None else ncrit
        nspawn = self.nspawn if nspawn is None else nspawn
        images = self.images if images is None else images
        cycle = self.cycle if cycle is None else cycle
        self._check(lib().exafmm_set_params(self._h, P, theta, ncrit, nspawn, images, cycle))
        self.P, self.theta, self.ncrit, self.nspawn, self.images, self.cycle = P, theta, ncrit, nspawn, images, cycle

    def set_mixed_policy(self, m2l_fp32=1, p2p_fp32=True, min_level=2, max_dl=3):
        """Mixed form: which operators run in FP32 and which M2L pairs may.
        m2l_fp32: 0 FP64; 1 FP32 with per-class products on the tensor cores (bf16x3
        pieces, FP32 accumulation) where they pay; 2 FP32 pair by pair; 3 as 1 with the
        per-class products at any size; 4 and 5 as 1 and 3 with the per-class products in
        FP32 on the CUDA cores."""
        self._check(lib().exafmm_set_mixed_policy(self._h, int(m2l_fp32), int(p2p_fp32), min_level, max_dl))

    def set_p2p_targets_per_lane(self, tpl: int):
        """Mixed P2P: targets per lane, 0 by leaf size (two or three), or 2 / 3 for every leaf."""
        self._check(lib().exafmm_set_p2p_targets_per_lane(self._h, int(tpl)))

    # ---- solve steps (examples/fmm.cxx:163-179) ----
    def set_sources(self, xyzq=None):
        """Separate source bodies (examples/fmm.cxx -j IneJ): later solves evaluate the field
        of these sources at this context's bodies (free space; FP64 or mixed).  None: sources are
        the bodies again."""
        if xyzq is None:
            self._check(lib().exafmm_set_sources(self._h, None, 0))
            return
        xyzq = _f64(xyzq, 4)
        self._check(lib().exafmm_set_sources(self._h, _p(xyzq), len(xyzq)))

    def source_cells(self):
        """The source tree: (cells_int, cells_real, perm) as cells() / perm()."""
        nc = _c_ll()
        self._check(lib().exafmm_get_source_cells(self._h, ctypes.byref(nc), None, None, None))
        ints = np.zeros((nc.value, 5), dtype=np.int32)
        reals = np.zeros((nc.value, 4))
        self._check(lib().exafmm_get_source_cells(self._h, None, _p(ints), _p(reals), None))
        nb = int(ints[0, 4]) if nc.value else 0
        perm = np.zeros(nb, dtype=np.int32)
        self._check(lib().exafmm_get_source_cells(self._h, None, None, None, _p(perm)))
        return ints, reals, perm

    def set_bodies(self, xyzq):
        xyzq = _f64(xyzq, 4)
        self.n = len(xyzq)
        self.nsys = 0
        self._check(lib().exafmm_set_bodies(self._h, _p(xyzq), self.n))

    def set_bodies_device(self, ptr: int, n: int):
        self.n = n
        self.nsys = 0
        self._check(lib().exafmm_set_bodies_device(self._h, _vp(ptr), n))

    # ---- a forest of independent systems, solved together ----
    def set_systems(self, systems):
        """Independent systems (a list of (n_i, 4) arrays) solved as one forest:
        each gets its own bounds, tree, lists and expansions, as a solo solve of
        it would, with every phase launched once for all of them."""
        sizes = np.ascontiguousarray([len(x) for x in systems], dtype=np.int64)
        cat = _f64(np.concatenate([np.asarray(x, dtype=np.float64).reshape(-1, 4) for x in systems])
                   if len(systems) else np.zeros((0, 4)), 4)
        self.n, self.nsys = int(sizes.sum()), len(systems)
        self._sizes = sizes
        self._check(lib().exafmm_set_systems(self._h, self.nsys, _p(sizes), _p(cat)))

    def set_systems_device(self, ptr: int, sizes):
        """The same with the concatenated bodies already on the device."""
        sizes = np.ascontiguousarray(sizes, dtype=np.int64)
        self.n, self.nsys = int(sizes.sum()), len(sizes)
        self._sizes = sizes
        self._check(lib().exafmm_set_systems_device(self._h, self.nsys, _p(sizes), _vp(ptr)))

    def set_systems_list(self, systems):
        """The same forest from one array per system (no concatenation on the host):
        numpy arrays, or (device pointer, n) pairs."""
        sizes, ptrs, keep = [], [], []
        for x in systems:
            if isinstance(x, tuple):
                ptrs.append(int(x[0]))
                sizes.append(int(x[1]))
            else:
                a = _f64(x, 4)
                keep.append(a)
                ptrs.append(a.ctypes.data if len(a) else 0)
                sizes.append(len(a))
        k = len(sizes)
        self._sizes = np.asarray(sizes, dtype=np.int64)
        self.n, self.nsys = int(self._sizes.sum()), k
        n = (_c_ll * max(1, k))(*sizes)
        px = (_vp * max(1, k))(*[p or None for p in ptrs])
        self._check(lib().exafmm_set_systems_list(self._h, k, n, px))

    def system_results_list(self, outs=None) -> list:
        """Per-system results copied straight into `outs` (numpy arrays, or device
        pointers), one copy per system."""
        if outs is None:
            outs = [np.zeros((int(k), 4)) for k in self._sizes]
        ptrs = [o if isinstance(o, int) else (o.ctypes.data if len(o) else 0) for o in outs]
        po = (_vp * max(1, len(ptrs)))(*[p or None for p in ptrs])
        self._check(lib().exafmm_get_results_list(self._h, po))
        return outs

    def systems(self) -> dict:
        """Forest layout after a build: cell_base and body_off (nsys + 1 each), bounds (nsys, 6)."""
        cb = np.zeros(self.nsys + 1, dtype=np.int64)
        bo = np.zeros(self.nsys + 1, dtype=np.int64)
        b = np.zeros((self.nsys, 6))
        self._check(lib().exafmm_get_systems(self._h, _p(cb), _p(bo), _p(b)))
        return {"cell_base": cb, "body_off": bo, "bounds": b}

    def system_results(self, out: np.ndarray | None = None) -> list:
        """Per-system (n_i, 4) views of the concatenated results."""
        r = self.results(out)
        off = np.concatenate([[0], np.cumsum(self._sizes)])
        return [r[off[i]:off[i + 1]] for i in range(self.nsys)]

    def displace_bodies(self, sigma: float, seed: int):
        """Move every body in place on the device by sigma times three standard normals
        (a counter-based stream keyed by seed and body index); the next solve rebuilds."""
        self._check(lib().exafmm_displace_bodies(self._h, float(sigma), int(seed) & (2**64 - 1)))

    def bodies(self) -> np.ndarray:
        """The context's current bodies (caller order)."""
        x = np.zeros((self.n, 4))
        self._check(lib().exafmm_get_bodies(self._h, _p(x)))
        return x

    def get_bounds(self) -> np.ndarray:
        b = np.zeros(6)
        self._check(lib().exafmm_get_bounds(self._h, _p(b)))
        return b

    def build_tree(self, bounds=None):
        b = None if bounds is None else _f64(bounds)
        self._check(lib().exafmm_build_tree(self._h, _p(b)))

    def upward(self):
        self._check(lib().exafmm_upward(self._h))

    def traverse(self):
        self._check(lib().exafmm_traverse(self._h))

    def downward(self):
        self._check(lib().exafmm_downward(self._h))

    def solve(self):
        self._check(lib().exafmm_solve(self._h))

    def results(self, out: np.ndarray | None = None) -> np.ndarray:
        """(n, 4) potential and gradient in input order; out may be a preallocated
        (e.g. pinned) float64 array."""
        if out is None:
            out = np.zeros((self.n, 4))
        assert out.dtype == np.float64 and out.shape == (self.n, 4) and out.flags.c_contiguous
        self._check(lib().exafmm_get_results(self._h, _p(out)))
        return out

    def results_device(self, ptr: int):
        self._check(lib().exafmm_get_results_device(self._h, _vp(ptr)))

    def device_bytes(self) -> int:
        v = _c_ll()
        self._check(lib().exafmm_device_bytes(self._h, ctypes.byref(v)))
        return int(v.value)

    # ---- periodic systems (include/up_down_pass.h:78-99) ----
    def get_dipole(self, X0=None) -> np.ndarray:
        """UpDownPass::getDipole: sum of (x_i - X0) q_i (X0 defaults to the origin)."""
        d = np.zeros(3)
        x0 = None if X0 is None else np.ascontiguousarray(X0, dtype=np.float64)
        self._check(lib().exafmm_get_dipole(self._h, None if x0 is None else _p(x0), _p(d)))
        return d

    def dipole_correction(self, dipole, num_bodies=None):
        """UpDownPass::dipoleCorrection on the results of the last solve."""
        d = np.ascontiguousarray(dipole, dtype=np.float64)
        nb = self.n if num_bodies is None else int(num_bodies)
        self._check(lib().exafmm_dipole_correction(self._h, _p(d), nb))

    # ---- inspection ----
    def info(self) -> dict:
        nc, nm, npp, d = _c_ll(), _c_ll(), _c_ll(), _c_int()
        self._check(lib().exafmm_tree_info(self._h, ctypes.byref(nc), ctypes.byref(d), ctypes.byref(nm),
                                           ctypes.byref(npp)))
        return {"ncells": nc.value, "depth": d.value, "n_m2l": nm.value, "n_p2p": npp.value}

    def p2p_interactions(self) -> int:
        """Sum over the P2P list of NBODY(target) * NBODY(source), counted on the device."""
        v = _c_ll()
        self._check(lib().exafmm_list_work(self._h, ctypes.byref(v)))
        return int(v.value)

    def cells(self):
        nc = self.info()["ncells"]
        ints = np.zeros((nc, 5), dtype=np.int32)
        reals = np.zeros((nc, 4))
        self._check(lib().exafmm_get_cells(self._h, _p(ints), _p(reals)))
        return ints, reals

    def perm(self) -> np.ndarray:
        p = np.zeros(self.n, dtype=np.int32)
        self._check(lib().exafmm_get_perm(self._h, _p(p)))
        return p

    def lists(self):
        i = self.info()
        m2l = np.zeros((max(i["n_m2l"], 0), 3), dtype=np.int32)
        p2p = np.zeros((max(i["n_p2p"], 0), 3), dtype=np.int32)
        self._check(lib().exafmm_get_lists(self._h, _p(m2l), _p(p2p)))
        return m2l, p2p

    def expansions(self):
        nc = self.info()["ncells"]
        nt = self.P * (self.P + 1) // 2
        M = np.zeros((nc, nt), dtype=np.complex128)
        L = np.zeros((nc, nt), dtype=np.complex128)
        self._check(lib().exafmm_get_expansions(self._h, _p(M), _p(L)))
        return M, L

    def stream(self) -> int:
        return lib().exafmm_stream(self._h) or 0

    PHASES = ("bounds", "tree", "upward", "lists", "m2l", "p2p", "downward", "total")

    # ---- records in the reference's file formats ----
    def write_list(self, path: str = "./", rank: int = 0) -> str:
        """Traversal::writeList (EXAFMM_COUNT_LIST): path + 'list%06d.dat' with each cell's
        ICELL and P2P / M2L list sizes from the last traversal.  Returns the file name."""
        self._check(lib().exafmm_write_list(self._h, path.encode(), int(rank)))
        return f"{path}list{int(rank):06d}.dat"

    def write_time(self, path: str = "./", rank: int = 0) -> str:
        """logger::writeTime: path + 'time%06d.dat' with the phase times summed since the last
        call, under the reference's event names; clears them.  Returns the file name."""
        self._check(lib().exafmm_write_time(self._h, path.encode(), int(rank)))
        return f"{path}time{int(rank):06d}.dat"

    def phase_times(self) -> dict:
        """Device milliseconds of each phase of the last solve (CUDA events on its stream)."""
        t = np.zeros(8)
        self._check(lib().exafmm_phase_times(self._h, _p(t)))
        return dict(zip(self.PHASES, t.tolist()))


# ---- free functions: direct sum and per-operator forms ----
def _kcheck(rc):
    if rc != 0:
        raise FmmError(lib().exafmm_kernel_error().decode())


def write_time_events(events: dict, path: str = "./", rank: int = 0) -> str:
    """logger::writeTime of `events` (name -> seconds) into path + 'time%06d.dat'."""
    names = (ctypes.c_char_p * max(len(events), 1))(*[k.encode() for k in events])
    vals = np.array(list(events.values()) or [0.0], dtype=np.float64)
    if lib().exafmm_write_time_events(path.encode(), int(rank), len(events), ctypes.cast(names, _vp), _p(vals)):
        raise FmmError(f"cannot write {path}time{int(rank):06d}.dat")
    return f"{path}time{int(rank):06d}.dat"


def morton_key(X, Xmin, diameter: float, level: int) -> int:
    """BuildTree::getKey (include/build_tree.h:111-120) as the compiled reference evaluates it."""
    X = _f64(X).reshape(3)
    Xmin = _f64(Xmin).reshape(3)
    return int(lib().exafmm_morton_key(_p(X), _p(Xmin), float(diameter), int(level)))


def ewald(xyzq, ksize, alpha, sigma, cutoff, cycle, trg=None) -> np.ndarray:
    """Ewald summation (include/ewald.h) on the GPU in FP64; (n, 4) potential and
    gradient in input order (accumulated into trg when given)."""
    x = _f64(xyzq, 4)
    out = np.zeros((len(x), 4)) if trg is None else trg
    if lib().exafmm_ewald(_p(x), len(x), ksize, alpha, sigma, cutoff, cycle, _p(out)) != 0:
        raise FmmError(lib().exafmm_ewald_error().decode())
    return out


def direct(targets, sources, images=0, theta=0.4, cycle=2 * np.pi, trg=None) -> np.ndarray:
    t, s = _f64(targets, 4), _f64(sources, 4)
    out = np.zeros((len(t), 4)) if trg is None else _f64(trg).copy()
    _kcheck(lib().exafmm_direct(_p(t), len(t), _p(s), len(s), images, theta, cycle, _p(out)))
    return out


def p2m(P, X, xyzq, M=None):
    x = _f64(xyzq, 4)
    out = np.zeros(P * (P + 1) // 2, np.complex128) if M is None else _c128(M).copy()
    _kcheck(lib().exafmm_kernel_p2m(P, _p(_f64(X)), len(x), _p(x), _p(out)))
    return out


def m2m(P, Xp, Xc, Mc, Mp=None):
    Xc = _f64(Xc).reshape(-1, 3)
    Mc = _c128(Mc).reshape(len(Xc), -1)
    out = np.zeros(P * (P + 1) // 2, np.complex128) if Mp is None else _c128(Mp).copy()
    _kcheck(lib().exafmm_kernel_m2m(P, _p(_f64(Xp)), len(Xc), _p(Xc), _p(Mc), _p(out)))
    return out


def m2l(P, Xi, Xj, Mj, Li=None, Xper=None):
    out = np.zeros(P * (P + 1) // 2, np.complex128) if Li is None else _c128(Li).copy()
    xp = None if Xper is None else _f64(Xper)
    _kcheck(lib().exafmm_kernel_m2l(P, _p(_f64(Xi)), _p(_f64(Xj)), _p(_c128(Mj)), _p(out), _p(xp)))
    return out


def l2l(P, Xc, Xp, Lp, Lc=None):
    out = np.zeros(P * (P + 1) // 2, np.complex128) if Lc is None else _c128(Lc).copy()
    _kcheck(lib().exafmm_kernel_l2l(P, _p(_f64(Xc)), _p(_f64(Xp)), _p(_c128(Lp)), _p(out)))
    return out


def l2p(P, X, L, xyzq, trg=None):
    x = _f64(xyzq, 4)
    out = np.zeros((len(x), 4)) if trg is None else _f64(trg).copy()
    _kcheck(lib().exafmm_kernel_l2p(P, _p(_f64(X)), _p(_c128(L)), len(x), _p(x), _p(out)))
    return out


def p2p(xi, xj, Xper=None, trg=None):
    a, b = _f64(xi, 4), _f64(xj, 4)
    out = np.zeros((len(a), 4)) if trg is None else _f64(trg).copy()
    xp = None if Xper is None else _f64(Xper)
    _kcheck(lib().exafmm_kernel_p2p(len(a), _p(a), len(b), _p(b), _p(xp), _p(out)))
    return out


def drift(x: float, k: int, up: bool = False) -> float:
    return lib().exafmm_drift(float(x), int(k), int(up))


def launch_count() -> int:
    """Kernels the engine has launched in this process."""
    return int(lib().exafmm_launch_count())


class Batch:
    """Many independent systems per call, on a pool of solve contexts (one host
    thread and CUDA stream each)."""

    def __init__(self, P=10, theta=0.4, ncrit=64, nspawn=5000, precision=FP64, device=-1, workers=8, forest=0):
        h = _vp()
        rc = lib().exafmm_batch_create(ctypes.byref(h), P, theta, ncrit, nspawn, precision, device, workers)
        if rc != 0:
            raise FmmError(f"exafmm_batch_create failed ({rc})")
        self._h = h
        if forest:
            self.set_forest(forest)

    def set_forest(self, buckets: int):
        """buckets > 0: each call's systems are solved as at most `buckets` forests
        (groups of whole size classes, one context each); 0: one system per context."""
        if lib().exafmm_batch_set_forest(self._h, int(buckets)) != 0:
            raise FmmError("invalid forest bucket count")

    def set_mixed_policy(self, m2l_fp32=1, p2p_fp32=True, min_level=2, max_dl=3):
        """Fmm.set_mixed_policy for every context of the batch."""
        if lib().exafmm_batch_set_mixed_policy(self._h, int(m2l_fp32), int(p2p_fp32), min_level, max_dl) != 0:
            raise FmmError("invalid mixed policy")

    def set_p2p_candidates(self, candidates):
        """P2P targets-per-lane settings the autotuner tries with every ncrit (default [0])."""
        c = np.ascontiguousarray(candidates, dtype=np.int32)
        if lib().exafmm_batch_set_p2p_candidates(self._h, _p(c), len(c)) != 0:
            raise FmmError("invalid P2P candidates")

    def config_table(self) -> dict:
        """The tuned table: size class -> (ncrit, P2P targets per lane)."""
        buf = np.zeros(3 * 64, dtype=np.int32)
        k = lib().exafmm_batch_config_table(self._h, _p(buf), 64)
        return {int(buf[3 * i]): (int(buf[3 * i + 1]), int(buf[3 * i + 2])) for i in range(k)}

    def set_config_table(self, table: dict):
        t = np.ascontiguousarray([v for c, (n, tp) in sorted(table.items()) for v in (c, n, tp)] or [0],
                                 dtype=np.int32)
        if lib().exafmm_batch_set_config_table(self._h, _p(t), len(table)) != 0:
            raise FmmError("invalid config table")

    def set_ncrit_candidates(self, candidates):
        """The ncrit values the autotuner tries, in order (default 32, 64, 128)."""
        c = np.ascontiguousarray(candidates, dtype=np.int32)
        if lib().exafmm_batch_set_ncrit_candidates(self._h, _p(c), len(c)) != 0:
            raise FmmError("invalid ncrit candidates")

    def elapsed_ms(self) -> float:
        """Forest mode: device time of the last call (first copy in to last copy out)."""
        v = _c_double()
        lib().exafmm_batch_elapsed(self._h, ctypes.byref(v))
        return v.value

    def buckets(self, count: int):
        """Forest mode: (group of each system, ncrit of each group) of the last call."""
        of = np.zeros(max(1, count), dtype=np.int32)
        nc = np.zeros(64, dtype=np.int32)
        k = lib().exafmm_batch_buckets(self._h, _p(of), _p(nc), 64)
        return of[:count], nc[:max(0, k)]

    def bucket_p2p(self) -> np.ndarray:
        """Forest mode: each group's P2P targets per lane in the last call."""
        t = np.zeros(64, dtype=np.int32)
        k = lib().exafmm_batch_bucket_p2p(self._h, _p(t), 64)
        return t[:max(0, k)]

    def close(self):
        if getattr(self, "_h", None):
            lib().exafmm_batch_destroy(self._h)
            self._h = None

    __del__ = close

    def autotune(self, enable: bool):
        lib().exafmm_batch_autotune(self._h, int(enable))

    def ncrit_table(self) -> dict:
        buf = (_c_int * 128)()
        k = lib().exafmm_batch_ncrit_table(self._h, buf, 64)
        return {buf[2 * i]: buf[2 * i + 1] for i in range(k)}

    def set_ncrit_table(self, table: dict):
        pairs = (_c_int * (2 * max(1, len(table))))(*[v for kv in sorted(table.items()) for v in kv])
        if lib().exafmm_batch_set_ncrit_table(self._h, pairs, len(table)) != 0:
            raise FmmError("invalid ncrit table")

    def solve_device(self, sizes, in_ptrs, out_ptrs):
        """Forest mode with device memory: system i's n_i x 4 doubles at in_ptrs[i],
        its results to out_ptrs[i]."""
        k = len(sizes)
        n = (_c_ll * max(1, k))(*[int(v) for v in sizes])
        px = (_vp * max(1, k))(*[int(p) or None for p in in_ptrs])
        po = (_vp * max(1, k))(*[int(p) or None for p in out_ptrs])
        if lib().exafmm_batch_solve(self._h, k, n, px, po) != 0:
            raise FmmError(lib().exafmm_batch_error(self._h).decode())

    def solve(self, systems, outs=None):
        """systems: list of (n_i, 4) float64 arrays; returns the list of (n_i, 4) results."""
        xs = [_f64(x, 4) for x in systems]
        if outs is None:
            outs = [np.zeros((len(x), 4)) for x in xs]
        for o, x in zip(outs, xs):
            assert o.dtype == np.float64 and o.shape == (len(x), 4) and o.flags.c_contiguous
        k = len(xs)
        n = (_c_ll * k)(*[len(x) for x in xs])
        px = (_vp * k)(*[x.ctypes.data for x in xs])
        po = (_vp * k)(*[o.ctypes.data for o in outs])
        if lib().exafmm_batch_solve(self._h, k, n, px, po) != 0:
            raise FmmError(lib().exafmm_batch_error(self._h).decode())
        return outs

    def times(self, count: int) -> np.ndarray:
        t = np.zeros(count)
        lib().exafmm_batch_times(self._h, _p(t))
        return t


def forest_buckets(sizes, buckets: int) -> np.ndarray:
    """The batch's forest grouping of systems of these sizes (host only)."""
    n = np.ascontiguousarray(sizes, dtype=np.int64)
    out = np.zeros(max(1, len(n)), dtype=np.int32)
    k = lib().exafmm_forest_buckets(len(n), _p(n), int(buckets), _p(out))
    if k < 0:
        raise FmmError("invalid forest grouping input")
    return out[:len(n)]


class Server:
    """Asynchronous request server with HBM-budget admission."""

    def __init__(self, device=-1, workers=8, hbm_budget_bytes=150e9):
        h = _vp()
        rc = lib().exafmm_server_create(ctypes.byref(h), device, workers, float(hbm_budget_bytes))
        if rc != 0:
            raise FmmError(f"exafmm_server_create failed ({rc})")
        self._h = h
        self._live = {}

    def close(self):
        if getattr(self, "_h", None):
            lib().exafmm_server_destroy(self._h)
            self._h = None
            self._live.clear()

    __del__ = close

    def submit(self, xyzq, P=10, theta=0.4, ncrit=64, nspawn=5000, precision=FP64, out=None) -> int:
        x = _f64(xyzq, 4)
        o = np.zeros((len(x), 4)) if out is None else out
        assert o.dtype == np.float64 and o.shape == (len(x), 4) and o.flags.c_contiguous
        t = _c_ll()
        rc = lib().exafmm_server_submit(self._h, _p(x), len(x), _p(o), P, theta, ncrit, nspawn, precision,
                                        ctypes.byref(t))
        if rc != 0:
            raise FmmError(f"exafmm_server_submit failed ({rc})")
        self._live[t.value] = (x, o)   # both must outlive the request
        return t.value

    def done(self, ticket: int) -> bool:
        d = _c_int()
        lib().exafmm_server_poll(self._h, ticket, ctypes.byref(d))
        return bool(d.value)

    def wait(self, ticket: int):
        """(results, times) with times = (queue ms, start-to-results ms, submit-to-results ms, device ms)."""
        t = np.zeros(4)
        rc = lib().exafmm_server_wait(self._h, ticket, _p(t))
        x, o = self._live.pop(ticket)
        if rc != 0:
            raise FmmError(lib().exafmm_server_error().decode())
        return o, t

    # ---- device-resident repeat chains ----
    def open_session(self, xyzq, P=10, theta=0.4, ncrit=64, nspawn=5000, precision=FP64) -> int:
        """A chain of solves of one system kept on the device between steps."""
        x = _f64(xyzq, 4)
        sid = _c_ll()
        rc = lib().exafmm_server_open_session(self._h, _p(x), len(x), P, theta, ncrit, nspawn, precision,
                                              ctypes.byref(sid))
        if rc != 0:
            raise FmmError(f"exafmm_server_open_session failed ({rc})")
        self._live[("session", sid.value)] = x
        return sid.value

    def submit_step(self, session: int, sigma=0.0, seed=0, d_xyzq: int | None = None, out=None) -> int:
        """The session's next step: the first solves the opened bodies, later ones
        move them on the device (to d_xyzq, or by a Gaussian step of sigma drawn from
        seed) and solve again."""
        n = len(self._live[("session", session)])
        o = np.zeros((n, 4)) if out is None else out
        assert o.dtype == np.float64 and o.shape == (n, 4) and o.flags.c_contiguous
        t = _c_ll()
        rc = lib().exafmm_server_submit_step(self._h, session, float(sigma), int(seed) & (2**64 - 1),
                                             _vp(d_xyzq) if d_xyzq else None, _p(o), ctypes.byref(t))
        if rc != 0:
            raise FmmError(lib().exafmm_server_error().decode() or f"exafmm_server_submit_step failed ({rc})")
        self._live[t.value] = (None, o)
        return t.value

    def session_bodies(self, session: int) -> np.ndarray:
        x = np.zeros_like(self._live[("session", session)])
        if lib().exafmm_server_session_bodies(self._h, session, _p(x)) != 0:
            raise FmmError(lib().exafmm_server_error().decode())
        return x

    def close_session(self, session: int):
        if lib().exafmm_server_close_session(self._h, session) != 0:
            raise FmmError(lib().exafmm_server_error().decode())
        self._live.pop(("session", session), None)

    def set_mixed_policy(self, m2l_fp32=1, p2p_fp32=True, min_level=2, max_dl=3):
        """Fmm.set_mixed_policy for the server's mixed-precision requests."""
        if lib().exafmm_server_set_mixed_policy(self._h, int(m2l_fp32), int(p2p_fp32), min_level, max_dl) != 0:
            raise FmmError("invalid mixed policy")

    def set_grouping(self, max_requests=64, max_request_bodies=262144, max_group_bodies=4 << 20):
        """Continuous batching of small queued requests with equal parameters into
        one forest solve (max_requests=1: off)."""
        if lib().exafmm_server_set_grouping(self._h, int(max_requests), int(max_request_bodies),
                                            int(max_group_bodies)) != 0:
            raise FmmError("invalid grouping limits")

    def stats(self) -> dict:
        v = np.zeros(6)
        lib().exafmm_server_stats(self._h, _p(v))
        g = _c_ll()
        lib().exafmm_server_grouped(self._h, ctypes.byref(g))
        return dict(in_flight=v[0], held=v[1], peak_admitted=v[2], completed=int(v[3]), queued=int(v[4]),
                    budget=v[5], grouped=int(g.value))
