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
