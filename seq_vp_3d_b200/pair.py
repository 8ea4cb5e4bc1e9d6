"""Device registration pair: the Q1 energy/gradient/metric kernels of libsvp3d behind a small Python class.

A DevicePair owns the frozen device constants of one subproblem (grid, fixed image, spline of the moving image,
u_ref, weights) -- the device half of jd_curl/three_d/problem.py:284 Problem3D.  Every method takes and returns
CUDA tensors (node fields (nz, ny, nx[, 3]) float64, free vectors (3 * n_free,) component-major).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .device import grid_struct, ptr, require_cuda, stream_ptr, to_device

F64 = torch.float64


class DevicePair:
    PRECISIONS = {"plain": 0, "mixed": 1}

    def __init__(self, grid, fixed, moving, u_ref, *, lam, mu, nu, kappa, activation=.05, delta=0., stream=None,
                 precision="plain"):
        require_cuda()
        self.grid = grid
        self.weights = (float(lam), float(mu), float(nu), float(kappa), float(activation), float(delta))
        self._g = grid_struct(grid)
        self._w = _lib.Weights(*self.weights)
        f, m, r = to_device(fixed), to_device(moving), to_device(u_ref)
        if tuple(f.shape) != grid.shape or tuple(m.shape) != grid.shape or tuple(r.shape) != grid.shape + (3,):
            raise ValueError("fixed/moving (nz, ny, nx) and u_ref (nz, ny, nx, 3) required")
        h = ctypes.c_void_p()
        _lib.call("svp_pair_create", ctypes.byref(self._g), ctypes.byref(self._w), ptr(f), ptr(m), ptr(r),
                  ctypes.byref(h), stream_ptr(stream))
        self._h = h
        self.device = f.device
        if precision not in self.PRECISIONS:
            raise ValueError("precision: 'plain' (float64) or 'mixed' (float32 search direction)")
        self.precision = precision
        _lib.call("svp_pair_set_precision", self._h, self.PRECISIONS[precision])
        nz, ny, nx = grid.shape
        self.nnode, self.nfree = nz * ny * nx, (nz - 2) * (ny - 2) * (nx - 2)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().svp_pair_destroy(h)
            except Exception:
                pass
            self._h = None

    # ------------------------------------------------------------------ allocation helpers
    def node(self, comps=0):
        shape = self.grid.shape + ((comps,) if comps else ())
        return torch.empty(shape, dtype=F64, device=self.device)

    def free(self):
        return torch.empty(3 * self.nfree, dtype=F64, device=self.device)

    # ------------------------------------------------------------------ kernels
    def set_reference(self, u_ref, stream=None):
        r = to_device(u_ref)
        _lib.call("svp_pair_set_reference", self._h, ptr(r), stream_ptr(stream))

    def set_spline_coefficients(self, coefficients, stream=None):
        """Use given not-a-knot coefficients (nz, ny, nx) of the moving image on this grid's knots."""
        c = to_device(coefficients)
        if tuple(c.shape) != self.grid.shape:
            raise ValueError("spline coefficients: (nz, ny, nx) required")
        _lib.call("svp_pair_set_spline_coefficients", self._h, ptr(c), stream_ptr(stream))

    def spline_coefficients(self, stream=None):
        out = self.node()
        _lib.call("svp_pair_spline_coefficients", self._h, ptr(out), stream_ptr(stream))
        return out

    def warp(self, u, with_gradient=False, stream=None):
        w = self.node()
        g = self.node(3) if with_gradient else None
        _lib.call("svp_warp", self._h, ptr(u), ptr(w), ptr(g), stream_ptr(stream))
        return w, g

    def sample_points(self, points, with_gradient=True, stream=None):
        pts = to_device(points).reshape(-1, 3).contiguous()
        n = pts.shape[0]
        v = torch.empty(n, dtype=F64, device=self.device)
        g = torch.empty((n, 3), dtype=F64, device=self.device) if with_gradient else None
        _lib.call("svp_sample_points", self._h, ptr(pts), n, ptr(v), ptr(g), stream_ptr(stream))
        return v, g

    def energy(self, u, warped, stream=None):
        """(terms[5] image, proximity, jd, curl, barrier; number of barrier points with J <= delta)."""
        t = (ctypes.c_double * 5)()
        bad = ctypes.c_int64()
        _lib.call("svp_energy", self._h, ptr(u), ptr(warped), t, ctypes.byref(bad), stream_ptr(stream))
        return np.array(t[:]), int(bad.value)

    def energy_difference(self, base_u, base_w, trial_u, trial_w, base_active=None, trial_active=None, stream=None):
        """(E(trial) - E(base), F(trial) - F(base)), cancellation-free; the optional barrier activity masks of the
        two states only skip work (same values)."""
        d = (ctypes.c_double * 2)()
        _lib.call("svp_energy_difference_masked", self._h, ptr(base_u), ptr(base_w), ptr(trial_u), ptr(trial_w),
                  ptr(base_active), ptr(trial_active), d, stream_ptr(stream))
        return d[0], d[1]

    def energy_difference_screened(self, base_u, base_w, trial_u, trial_w, base_active=None, stream=None):
        """energy_difference with the JD/curl penalty differences in float32 (the mixed form's screen): (dE, dF,
        band), dE within band of the float64 difference, dF the float64 call's value."""
        d = (ctypes.c_double * 2)()
        band = ctypes.c_double()
        _lib.call("svp_energy_difference_screened", self._h, ptr(base_u), ptr(base_w), ptr(trial_u), ptr(trial_w),
                  ptr(base_active), d, ctypes.byref(band), stream_ptr(stream))
        return d[0], d[1], band.value

    def cell_mask(self):
        return torch.empty(self.grid.n_cells, dtype=torch.uint8, device=self.device)

    def trial_energy(self, base_u, base_w, trial_u, with_gradient=True, base_active=None, stream=None):
        """Warp and evaluate a trial against its base in one pass: (warped, image_grad or None, terms[5],
        barrier violations, (E(trial) - E(base), F(trial) - F(base)), the trial's barrier activity mask).
        base_active (the base's own mask) limits the base's barrier sweep to the cells where it can contribute;
        the values are the same bits."""
        w = self.node()
        g = self.node(3) if with_gradient else None
        act = self.cell_mask()
        t = (ctypes.c_double * 5)()
        d = (ctypes.c_double * 2)()
        bad = ctypes.c_int64()
        _lib.call("svp_trial_energy_active", self._h, ptr(base_u), ptr(base_w), ptr(trial_u), ptr(w), ptr(g),
                  ptr(base_active), ptr(act), t, d, ctypes.byref(bad), stream_ptr(stream))
        return w, g, np.array(t[:]), int(bad.value), (d[0], d[1]), act

    def trial_energy_screened(self, base_u, base_w, trial_u, with_gradient=True, base_active=None, stream=None):
        """trial_energy with the JD/curl penalties in float32 (the mixed form's energy screen): the same tuple plus
        the error estimate of the E difference (the node terms, the barrier and F are the float64 call's bits)."""
        w = self.node()
        g = self.node(3) if with_gradient else None
        act = self.cell_mask()
        t = (ctypes.c_double * 5)()
        d = (ctypes.c_double * 2)()
        band = ctypes.c_double()
        bad = ctypes.c_int64()
        _lib.call("svp_trial_energy_screened", self._h, ptr(base_u), ptr(base_w), ptr(trial_u), ptr(w), ptr(g),
                  ptr(base_active), ptr(act), t, d, ctypes.byref(band), ctypes.byref(bad), stream_ptr(stream))
        return w, g, np.array(t[:]), int(bad.value), (d[0], d[1]), act, band.value

    def gradient(self, u, warped, image_grad, term="total", out=None, active=None, stream=None):
        out = self.free() if out is None else out
        _lib.call("svp_gradient_masked", self._h, ptr(u), ptr(warped), ptr(image_grad), _lib.TERMS[term],
                  ptr(active), ptr(out), stream_ptr(stream))
        return out

    def outer_gradients(self, u, warped, image_grad, active=None, stream=None):
        gF, gD, gE = self.free(), self.free(), self.free()
        _lib.call("svp_outer_gradients_masked", self._h, ptr(u), ptr(warped), ptr(image_grad), ptr(active), ptr(gF),
                  ptr(gD), ptr(gE), stream_ptr(stream))
        return gF, gD, gE

    def ggn_diagonal(self, u, image_grad, active=None, stream=None):
        out = self.free()
        _lib.call("svp_ggn_diagonal_masked", self._h, ptr(u), ptr(image_grad), ptr(active), ptr(out),
                  stream_ptr(stream))
        return out

    def ggn_hvp(self, u, image_grad, p, stream=None):
        out = self.free()
        _lib.call("svp_ggn_hvp", self._h, ptr(u), ptr(image_grad), ptr(to_device(p)), ptr(out), stream_ptr(stream))
        return out

    def node_min_jd(self, u, extension_activation=None, stats=None, stream=None):
        """Node JD measure (T62); with extension_activation, the T69/T73 face/interior extension on candidate cells
        (stats, a dict, then receives the candidate count)."""
        out = self.node()
        if extension_activation is None:
            _lib.call("svp_node_min_jd", self._h, ptr(u), ptr(out), stream_ptr(stream))
            return out
        cand = ctypes.c_int64()
        _lib.call("svp_node_min_jd_extended", self._h, ptr(u), float(extension_activation), ptr(out),
                  ctypes.byref(cand) if stats is not None else None, stream_ptr(stream))
        if stats is not None:
            stats["candidates"] = stats.get("candidates", 0) + int(cand.value)
        return out

    def jd_root(self, u, p, limit, stream=None):
        """(tau of the first closed27 root in (0, limit] or None, invalid base points)."""
        root = ctypes.c_double()
        bad = ctypes.c_int64()
        _lib.call("svp_jd_root", self._h, ptr(u), ptr(p), float(limit), ctypes.byref(root), ctypes.byref(bad),
                  stream_ptr(stream))
        r = root.value
        return (None if not np.isfinite(r) else r), int(bad.value)

    def poisson_apply(self, a, b, rhs, *, metric="q1", scale=None, sign=1., out=None, stream=None):
        out = self.free() if out is None else out
        _lib.call("svp_poisson_apply", self._h, float(a), float(b), 0 if metric == "q1" else 1, ptr(scale),
                  ptr(rhs), float(sign), ptr(out), stream_ptr(stream))
        return out

    # ------------------------------------------------------------------ vector helpers
    def inject(self, theta, out=None, stream=None):
        out = self.node(3) if out is None else out
        _lib.call("svp_inject", ctypes.byref(self._g), ptr(theta), ptr(out), stream_ptr(stream))
        return out

    def trial_point(self, theta, tau, p, maxima_dev, stream=None):
        """(candidate, u) of a line-search trial in one pass: candidate = theta + tau p with axpy's roundings,
        u = inject(candidate); maxima_dev (two device doubles, e.g. a Scalars slot pair) receives
        (max |candidate - theta|, max |theta|)."""
        cand = torch.empty_like(theta)
        u = self.node(3)
        _lib.call("svp_trial_point", ctypes.byref(self._g), ptr(theta), float(tau), ptr(p), ptr(cand), ptr(u),
                  maxima_dev, stream_ptr(stream))
        return cand, u

    def restrict(self, field, out=None, stream=None):
        out = self.free() if out is None else out
        _lib.call("svp_restrict", ctypes.byref(self._g), ptr(field), ptr(out), stream_ptr(stream))
        return out

    def step_bound(self, u, p, stream=None):
        b = ctypes.c_double()
        _lib.call("svp_step_bound", ctypes.byref(self._g), ptr(u), ptr(p), ctypes.byref(b), stream_ptr(stream))
        return b.value


def dot(a, b, stream=None):
    out = ctypes.c_double()
    _lib.call("svp_dot", ptr(a), ptr(b), a.numel(), ctypes.byref(out), stream_ptr(stream))
    return out.value


def axpy(x, tau, p, out=None, stream=None):
    out = torch.empty_like(x) if out is None else out
    _lib.call("svp_axpy", ptr(x), float(tau), ptr(p), x.numel(), ptr(out), stream_ptr(stream))
    return out


class Scalars:
    """Device slots for the scalars of one step (dots, BB2 products, bounds), gathered with a single copy into pinned
    host memory and one stream synchronisation (libsvp3d's *_dev entry points write the slots stream-ordered)."""

    def __init__(self, n=16, device="cuda"):
        self.dev = torch.zeros(n, dtype=torch.float64, device=device)
        self.host = torch.zeros(n, dtype=torch.float64).pin_memory()

    def slot(self, k):
        return ctypes.c_void_p(self.dev.data_ptr() + 8 * k)

    def dot(self, k, a, b, stream=None):
        _lib.call("svp_dot_dev", ptr(a), ptr(b), a.numel(), self.slot(k), stream_ptr(stream))

    def bb2(self, k, theta, theta_old, g, g_old, p_old, p, stream=None):
        _lib.call("svp_bb2_dots_dev", ptr(theta), ptr(theta_old), ptr(g), ptr(g_old), ptr(p_old), ptr(p),
                  theta.numel(), self.slot(k), stream_ptr(stream))

    def step_dots(self, k, g, p, previous=None, stream=None):
        """Slots k, k+1 = g.g, g.p and, with previous = (theta, theta_old, g_old, p_old), k+2..k+5 = the BB2
        products, in one pass (the values of dot() and bb2())."""
        th, th0, g0, p0 = (None,) * 4 if previous is None else previous
        _lib.call("svp_step_dots_dev", ptr(g), ptr(p), ptr(th), ptr(th0), ptr(g0), ptr(p0), g.numel(), self.slot(k),
                  stream_ptr(stream))

    def max_abs_diff(self, k, a, b, stream=None):
        _lib.call("svp_max_abs_diff_dev", ptr(a), ptr(b), a.numel(), self.slot(k), stream_ptr(stream))

    def step_bound(self, k, pair, u, p, stream=None):
        _lib.call("svp_step_bound_dev", ctypes.byref(pair._g), ptr(u), ptr(p), self.slot(k), stream_ptr(stream))

    def copy_async(self, stream=None):
        """Start the copy of every slot to the host; values() waits for it (usually already done by then, when a
        later call synchronized the stream)."""
        s = torch.cuda.current_stream() if stream is None else stream
        with torch.cuda.stream(s):
            self.host.copy_(self.dev, non_blocking=True)
            self._done = torch.cuda.Event()
            self._done.record(s)

    def values(self):
        self._done.synchronize()
        return self.host.numpy().copy()

    def fetch(self, stream=None):
        """Copy every slot to the host and wait; returns a numpy copy."""
        s = torch.cuda.current_stream() if stream is None else stream
        with torch.cuda.stream(s):
            self.host.copy_(self.dev, non_blocking=True)
        s.synchronize()
        return self.host.numpy().copy()
