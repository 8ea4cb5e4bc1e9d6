"""Rectangular physical grid (mirror of jd_curl/three_d/grid.py:11 Grid3D and :49 make_grid_3d).

Shape is zyx, spacing and axes are xyz; the grid id is the reference's SHA-256 of (sizes, spacing, origins, unit),
so ids agree with the reference for the same arguments.
"""
from dataclasses import dataclass
import hashlib

import numpy as np


_WEIGHT_TOTALS = {}


class InputValidationError(ValueError):
    """A named input violates the numerical or layout contract (jd_curl.validation.InputValidationError)."""


@dataclass(frozen=True)
class Grid3D:
    shape: tuple
    spacing: tuple
    axes: tuple
    trapezoid: tuple
    omega: float
    unit: str
    grid_id: str

    @property
    def interior_shape(self):
        return tuple(n - 2 for n in self.shape)

    @property
    def cell_shape(self):
        return tuple(n - 1 for n in self.shape)

    @property
    def n_free_scalar(self):
        return int(np.prod(self.interior_shape))

    @property
    def n_cells(self):
        return int(np.prod(self.cell_shape))

    @property
    def n_nodes(self):
        return int(np.prod(self.shape))

    def node_weights(self):
        tx, ty, tz = self.trapezoid
        return self.omega * tz[:, None, None] * ty[None, :, None] * tx[None, None, :]

    def node_weight_total(self):
        """Sum of the node weights, accumulated in long double and rounded once; cached per grid id (it costs tens of
        milliseconds on a native grid, and every registration on the grid needs it for its MSE)."""
        total = _WEIGHT_TOTALS.get(self.grid_id)
        if total is None:
            total = float(np.sum(self.node_weights(), dtype=np.longdouble))
            if len(_WEIGHT_TOTALS) >= 64:
                _WEIGHT_TOTALS.clear()
            _WEIGHT_TOTALS[self.grid_id] = total
        return total

    def identity(self):
        x, y, z = self.axes
        out = np.empty(self.shape + (3,))
        out[..., 0], out[..., 1], out[..., 2] = x, y[:, None], z[:, None, None]
        return out


def _count(value, name):
    """A node count: a plain integer of at least 5 (the Q1 cell kernels need interior nodes on every axis)."""
    ok = isinstance(value, (int, np.integer)) and not isinstance(value, bool) and value >= 5
    if not ok:
        raise InputValidationError(f"{name} must be an integer node count >= 5, got {value!r}")
    return int(value)


def _scalar(value, name, *, positive=False):
    ok = isinstance(value, (int, float, np.integer, np.floating)) and not isinstance(value, bool)
    value = float(value) if ok else float("nan")
    if not (ok and np.isfinite(value) and (value > 0 or not positive)):
        kind = "a positive finite" if positive else "a finite"
        raise InputValidationError(f"{name} must be {kind} real number")
    return value


def _axis(count, step, start):
    """Node coordinates start + step * k, k = 0 .. count - 1 (read-only), and the trapezoid weights of the axis."""
    with np.errstate(all="ignore"):
        coords = start + step * np.arange(count, dtype=np.float64)
    if not (np.isfinite(coords).all() and (coords[1:] > coords[:-1]).all()):
        raise InputValidationError("axis coordinates overflow or do not increase strictly")
    weights = np.full(count, 1.0)
    weights[0] = weights[-1] = 0.5
    coords.flags.writeable = weights.flags.writeable = False
    return coords, weights


def make_grid_3d(*, nx, ny, nz, hx, hy, hz, x0=0., y0=0., z0=0., unit="unit"):
    """Grid3D of nx x ny x nz nodes (keyword arguments as the reference's factory, grid.py:49).  The grid id is the
    SHA-256 of repr((sizes, spacings, origins, unit)) with xyz-ordered tuples, the identity the reference assigns to
    the same arguments, so states and certificates carry interchangeable grid ids."""
    counts = tuple(_count(v, k) for k, v in (("nx", nx), ("ny", ny), ("nz", nz)))
    steps = tuple(_scalar(v, k, positive=True) for k, v in (("hx", hx), ("hy", hy), ("hz", hz)))
    starts = tuple(_scalar(v, k) for k, v in (("x0", x0), ("y0", y0), ("z0", z0)))
    if not (isinstance(unit, str) and unit.strip()):
        raise InputValidationError("unit must name the length unit (a nonempty string)")
    axes, weights = zip(*(_axis(n, h, o) for n, h, o in zip(counts, steps, starts)))
    with np.errstate(all="ignore"):
        cell_volume = float(steps[0] * steps[1] * steps[2])
    # the smallest node mass, a corner's omega / 8, must stay a positive finite double
    if not (np.isfinite(cell_volume) and cell_volume * 0.125 > 0):
        raise InputValidationError("cell volume hx * hy * hz (and its corner eighth) must be positive and finite")
    grid_id = hashlib.sha256(repr((counts, steps, starts, unit)).encode()).hexdigest()
    return Grid3D(counts[::-1], steps, tuple(axes), tuple(weights), cell_volume, unit, grid_id)


def grid_from_shape(shape_zyx, spacing_xyz, unit="mm"):
    nz, ny, nx = shape_zyx
    hx, hy, hz = spacing_xyz
    return make_grid_3d(nx=nx, ny=ny, nz=nz, hx=hx, hy=hy, hz=hz, unit=unit)
