"""Device plumbing: torch owns device memory and streams; the kernels are libsvp3d's."""
import ctypes
import warnings

import numpy as np
import torch

from . import _lib


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("seq_vp_3d_b200 needs a CUDA device (sm_100a); there is no CPU fallback")


def stream_ptr(stream=None):
    s = torch.cuda.current_stream() if stream is None else stream
    return ctypes.c_void_p(s.cuda_stream)


def ptr(t):
    """Raw device pointer of a contiguous CUDA tensor (or None)."""
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return ctypes.c_void_p(t.data_ptr())


def to_device(a, dtype=torch.float64, device="cuda"):
    """numpy / tensor -> contiguous CUDA tensor of dtype (copies only when needed)."""
    if isinstance(a, torch.Tensor):
        t = a.to(device=device, dtype=dtype)
    else:
        with warnings.catch_warnings():
            # read-only host arrays (frozen states) are only read: the tensor view is copied to the device at once
            warnings.simplefilter("ignore", UserWarning)
            t = torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype)
    return t.contiguous()


def grid_struct(grid):
    """svp_grid of a Grid3D (shape zyx, spacing xyz, axes xyz)."""
    nz, ny, nx = grid.shape
    hx, hy, hz = grid.spacing
    x0, y0, z0 = (float(a[0]) for a in grid.axes)
    return _lib.Grid(nx, ny, nz, hx, hy, hz, x0, y0, z0)
