"""exafmm_get_bounds_noalloc: the bounding box for callers that cannot allocate
device memory (a host framework that owns every device byte through its own
pool, or a latency-bound loop that cannot pay for cudaMalloc/cudaFree).  The
caller brings device buffers for the bodies and the six outputs; the entry
point's only scratch is a small array built into the library.

Checked through the C ABI against the allocating entry point
(exafmm_get_bounds): bit for bit, on two calls in a row, the second on bodies
whose extremes lie inside the first's, so leftover scratch from the first call
would show.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _entry(ex):
    fn = ctypes.CDLL(ex.LIB_PATH).exafmm_get_bounds_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p]
    return fn


def _reference_bounds(ex, x):
    f = ex.Fmm(P=4)
    f.set_bodies(x)
    b = f.get_bounds()
    f.close()
    return b


def test_noalloc_bounds_match_allocating_entry_on_consecutive_calls(ex, datasets):
    import torch
    fn = _entry(ex)
    wide = datasets.plummer(300_000, seed=4)        # extremes out to r = 20
    narrow = datasets.cube(200_000, seed=5) * 0.5   # well inside the first box
    narrow[:, 3] *= 2.0
    out = torch.full((6,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for x in (wide, narrow):
        dx = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        torch.cuda.synchronize()
        rc = fn(dx.data_ptr(), len(x), out.data_ptr(), stream.cuda_stream)
        assert rc == 0
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), _reference_bounds(ex, x))


def test_noalloc_bounds_empty_and_out_of_range(ex):
    import torch
    fn = _entry(ex)
    out = torch.full((6,), 7.0, dtype=torch.float64, device="cuda")
    assert fn(None, 0, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), np.zeros(6))   # BoundBox::getBounds of no bodies
    assert fn(None, -1, out.data_ptr(), None) == 2
    assert fn(None, 1 << 31, out.data_ptr(), None) == 2       # beyond the stated maximum
    assert fn(None, 10, out.data_ptr(), None) == 3            # null bodies


# Child process: only the engine library and the CUDA runtime, no torch, so a
# cudaDeviceReset there invalidates nothing but what the child made itself.
_RESET_CHILD = r"""
import ctypes, sys
import numpy as np
lib = ctypes.CDLL(sys.argv[1])
rt = ctypes.CDLL("libcudart.so.12")
vp, ll = ctypes.c_void_p, ctypes.c_longlong
lib.exafmm_get_bounds_noalloc.argtypes = [vp, ll, vp, vp]
lib.exafmm_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                              ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int]
lib.exafmm_set_bodies.argtypes = [vp, vp, ll]
lib.exafmm_get_bounds.argtypes = [vp, vp]
lib.exafmm_destroy.argtypes = [vp]
rt.cudaMalloc.argtypes = [ctypes.POINTER(vp), ctypes.c_size_t]
rt.cudaMemcpy.argtypes = [vp, vp, ctypes.c_size_t, ctypes.c_int]
rt.cudaFree.argtypes = [vp]

def ref_bounds(x):
    ctx = vp()
    assert lib.exafmm_create(ctypes.byref(ctx), 4, 0.4, 64, 5000, 0, 6.283185307179586, 0, 0) == 0
    assert lib.exafmm_set_bodies(ctx, x.ctypes.data, len(x)) == 0
    b = np.zeros(6)
    assert lib.exafmm_get_bounds(ctx, b.ctypes.data) == 0
    lib.exafmm_destroy(ctx)
    return b

def noalloc_bounds(x):
    dx, db = vp(), vp()
    assert rt.cudaMalloc(ctypes.byref(dx), x.nbytes) == 0 and rt.cudaMalloc(ctypes.byref(db), 48) == 0
    assert rt.cudaMemcpy(dx, x.ctypes.data, x.nbytes, 1) == 0
    rc = lib.exafmm_get_bounds_noalloc(dx, len(x), db, None)
    assert rc == 0, rc
    assert rt.cudaDeviceSynchronize() == 0
    out = np.zeros(6)
    assert rt.cudaMemcpy(out.ctypes.data, db, 48, 2) == 0
    rt.cudaFree(dx); rt.cudaFree(db)
    return out

rng = np.random.default_rng(7)
a = np.ascontiguousarray(np.c_[rng.uniform(-3, 3, (50_000, 3)), rng.uniform(-1, 1, 50_000)])
b = np.ascontiguousarray(np.c_[rng.uniform(-1, 1, (40_000, 3)), rng.uniform(-1, 1, 40_000)])
ra, rb = ref_bounds(a), ref_bounds(b)
assert np.array_equal(noalloc_bounds(a), ra)
# a CUDA error already pending on this thread (a failed allocation) is left
# for its owner: status 5, nothing launched, the error still there afterwards
out6, big = vp(), vp()
assert rt.cudaMalloc(ctypes.byref(out6), 48) == 0   # a valid output, so nothing could go astray
assert rt.cudaMalloc(ctypes.byref(big), 1 << 60) != 0
assert lib.exafmm_get_bounds_noalloc(None, 0, out6, None) == 5
assert rt.cudaGetLastError() != 0 and rt.cudaGetLastError() == 0
assert lib.exafmm_get_bounds_noalloc(None, 0, out6, None) == 0
assert rt.cudaDeviceSynchronize() == 0
rt.cudaFree(out6)
assert rt.cudaDeviceReset() == 0   # a new primary context: the scratch address must be looked up again
assert np.array_equal(noalloc_bounds(b), rb)
assert np.array_equal(noalloc_bounds(a), ra)
print("ok")
"""


def test_noalloc_bounds_after_device_reset_and_with_pending_error(ex):
    import subprocess
    import sys
    r = subprocess.run([sys.executable, "-c", _RESET_CHILD, ex.LIB_PATH], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
