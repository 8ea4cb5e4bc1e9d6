"""The allocation-free subdivision entry point, svp_classify_cells_noalloc, against svp_classify_cells.

Some callers cannot allocate device memory while they run (their device memory belongs to another allocator or a
fixed budget, or an allocation's implicit synchronisation is not acceptable in their loop).  For them the library
keeps the subdivision heaps in a fixed device array.  This test calls both entry points through the C ABI on the
same inputs and requires identical verdicts (the tolerance of every certificate test: bit for bit), on two calls in
a row with different inputs, so that whatever the first call leaves in the shared array cannot change the second.
"""
import ctypes
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def verdict_bytes(lib, name, arrays, n, delta, depth, boxes):
    out = torch.zeros((n, 64), dtype=torch.uint8, device="cuda")
    ptrs = [ctypes.c_void_p(a.data_ptr()) for a in arrays]
    rc = getattr(lib, name)(*ptrs, n, float(delta), depth, boxes, ctypes.c_void_p(out.data_ptr()),
                            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, name
    torch.cuda.synchronize()
    return out.cpu().numpy()


def classify_inputs(delta):
    from seq_vp_3d_b200.certificate import fallback_arrays_device
    g = np.load(os.path.join(GOLDEN, "cells.npz"))
    ok, plo, phi, clo, chi, _ = fallback_arrays_device(g["vertices"], g["spacing"], delta)
    keep = torch.nonzero(ok.bool()).flatten()
    return [t[keep].contiguous() for t in (clo, chi, plo, phi)]


def test_noalloc_matches_allocating_entry_point_twice():
    from seq_vp_3d_b200 import _lib
    lib = _lib.load()
    for delta, depth, boxes in ((0.0, 48, 255), (0.01, 6, 40)):      # two calls in a row, different inputs
        arrays = classify_inputs(delta)
        n = arrays[0].shape[0]
        assert n > 100
        ref = verdict_bytes(lib, "svp_classify_cells", arrays, n, delta, depth, boxes)
        got = verdict_bytes(lib, "svp_classify_cells_noalloc", arrays, n, delta, depth, boxes)
        assert np.array_equal(got, ref), (delta, depth, boxes)


def test_noalloc_rejects_budget_beyond_its_array():
    from seq_vp_3d_b200 import _lib
    lib = _lib.load()
    arrays = classify_inputs(0.0)
    out = torch.zeros((1, 64), dtype=torch.uint8, device="cuda")
    rc = lib.svp_classify_cells_noalloc(*[ctypes.c_void_p(a.data_ptr()) for a in arrays], 1, 0.0, 48, 256,
                                        ctypes.c_void_p(out.data_ptr()), None)
    assert rc == _lib.SVP_EINVAL
    assert "255" in _lib.last_error()
