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


def _size(n, name):
    if isinstance(n, bool) or not isinstance(n, (int, np.integer)) or n < 5:
        raise InputValidationError(f"{name}: expected an integer >= 5")
    return int(n)


def _real(v, name, positive=False):
    if isinstance(v, bool) or not isinstance(v, (int, float, np.floating, np.integer)):
        raise InputValidationError(f"{name}: expected a real scalar")
    v = float(v)
    if not np.isfinite(v) or (positive and v <= 0):
        raise InputValidationError(f"{name}: must be {'positive and ' if positive else ''}finite")
    return v


def make_grid_3d(*, nx, ny, nz, hx, hy, hz, x0=0., y0=0., z0=0., unit="unit"):
    sizes = tuple(_size(n, name) for n, name in zip((nx, ny, nz), ("nx", "ny", "nz")))
    spacing = tuple(_real(h, name, positive=True) for h, name in zip((hx, hy, hz), ("hx", "hy", "hz")))
    origins = tuple(_real(o, name) for o, name in zip((x0, y0, z0), ("x0", "y0", "z0")))
    if not isinstance(unit, str) or not unit.strip():
        raise InputValidationError("unit: explicit nonempty length unit required")
    axes, mass = [], []
    with np.errstate(over="ignore", under="ignore", invalid="ignore"):
        omega = float(np.prod(spacing))
        for n, h, origin in zip(sizes, spacing, origins):
            axis = origin + h * np.arange(n, dtype=np.float64)
            if not np.all(np.isfinite(axis)) or not np.all(np.diff(axis) > 0):
                raise InputValidationError("coordinates must be finite and strictly increasing")
            axis.flags.writeable = False
            axes.append(axis)
            weights = np.ones(n)
            weights[[0, -1]] = .5
            weights.flags.writeable = False
            mass.append(weights)
    if not np.isfinite(omega) or omega / 8 <= 0:
        raise InputValidationError("grid mass must be positive finite float64, including corners")
    digest = hashlib.sha256(repr((sizes, spacing, origins, unit)).encode()).hexdigest()
    return Grid3D(sizes[::-1], spacing, tuple(axes), tuple(mass), omega, unit, digest)


def grid_from_shape(shape_zyx, spacing_xyz, unit="mm"):
    nz, ny, nx = shape_zyx
    hx, hy, hz = spacing_xyz
    return make_grid_3d(nx=nx, ny=ny, nz=nz, hx=hx, hy=hy, hz=hz, unit=unit)
