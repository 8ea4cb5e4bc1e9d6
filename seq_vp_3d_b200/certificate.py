"""Whole-cell Jacobian-determinant certificate on the B200 (drop-in for jd_curl/three_d/feasibility.py).

Call surface kept from the reference:
  certify_map(u, grid, *, config)                       feasibility.py:393 (and certify_map_owned :558)
  parallel_margins(u, grid, delta)                      compiled_enclosure.py:303
  prescreen_lower_bounds(u, grid, coefficients, cells)  certificate_prescreen.py:125
  fallback_arrays(vertices, spacing, delta, errors)     compiled_fallback.py:330
Every decision is made by libsvp3d's CUDA kernels, bit-identical to the reference CPU certifier (binary64 round to
nearest plus one outward ulp per interval operation, no FMA).  Host numpy inputs are uploaded; CUDA tensors are used
in place.  There is no CPU path.
"""
import ctypes
import hashlib
import threading
from dataclasses import dataclass, replace

import numpy as np
import torch

from . import _lib
from .device import grid_struct, ptr, require_cuda, stream_ptr, to_device
from .grid import InputValidationError

STATUS = ("certified_feasible", "infeasible", "uncertain")
REASONS = ("positive_enclosure_cover", "positive_bernstein_cover", "JACOBIAN_VIOLATION", "arithmetic_uncertain",
           "subdivision_budget", "NONFINITE_STATE", "NONZERO_BOUNDARY", "INVALID_DOMAIN", "unsupported_arithmetic",
           "sample_witness", "subdivision_witness", "box_budget", "depth_budget", "positive_edge_hull",
           "not_checked")
CERTIFICATE_VERSION = "q1-3d-parallel-hoisted-edge-hull-float-bernstein-prescreen-compiled-bernstein-v1"


@dataclass(frozen=True)
class CertificateConfig:
    """Subdivision budgets and the delta of J > delta (feasibility.py:22-117 config family).

    prescreen=True is the reference's PrescreenCertificateConfig execution (hull, float prescreen, interval
    fallback); prescreen=False its CompiledFallback/ParallelEnclosure execution (hull, interval fallback)."""
    delta: float = 0.
    max_depth: int = 48
    max_boxes: int = 255
    tile_size: int = 65536
    prescreen: bool = True

    def __post_init__(self):
        d = float(self.delta)
        if not np.isfinite(d) or d < 0 or d >= 1:
            raise InputValidationError("delta: require 0 <= delta < 1")
        object.__setattr__(self, "delta", 0.0 if d == 0 else d)
        for key, minimum in (("max_depth", 0), ("max_boxes", 1), ("tile_size", 1)):
            v = getattr(self, key)
            if isinstance(v, bool) or not isinstance(v, (int, np.integer)) or v < minimum:
                raise InputValidationError(f"{key}: expected an integer >= {minimum}")
            object.__setattr__(self, key, int(v))
        if self.max_depth > 120:
            raise InputValidationError("adaptive max_depth must be <= 120")


def PrescreenCertificateConfig(delta=.01, max_depth=48, max_boxes=255, tile_size=8192, fallback_workers=8, **_):
    """The reference's default production certificate (feasibility.py:107); fallback_workers has no GPU meaning."""
    return CertificateConfig(delta=delta, max_depth=max_depth, max_boxes=max_boxes, tile_size=tile_size,
                             prescreen=True)


@dataclass(frozen=True)
class FeasibilityResult:
    """feasibility.py:148-179 PrescreenFeasibilityResult fields."""
    status: str
    min_jd_lower_bound: float | None
    min_margin_lower_bound: float | None
    sampled_min_jd: float | None
    n_cells_checked: int
    n_uncertain: int
    n_infeasible: int
    n_boxes: int
    max_depth: int
    witness_cell: int | None
    witness_reference_point: tuple | None
    reason: str
    state_hash: str | None
    grid_id: str
    delta_hex: str
    config: CertificateConfig
    certificate_version: str = CERTIFICATE_VERSION
    n_fast_cells: int = 0
    n_fallback_cells: int = 0
    n_prescreen_cells: int = 0


@dataclass(frozen=True)
class Interval:
    lo: np.ndarray
    hi: np.ndarray


class Certifier:
    """Owned device workspace for one (grid, config) pair (libsvp3d svp_certifier)."""

    def __init__(self, grid, config):
        require_cuda()
        self.grid, self.config = grid, config
        self._g = grid_struct(grid)
        cfg = _lib.CertConfig(config.delta, config.max_depth, config.max_boxes, config.tile_size,
                              1 if config.prescreen else 0, 0)
        handle = ctypes.c_void_p()
        _lib.call("svp_certifier_create", ctypes.byref(self._g), ctypes.byref(cfg), ctypes.byref(handle))
        self._h = handle

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().svp_certifier_destroy(h)
            except Exception:
                pass
            self._h = None

    def run(self, u_dev, stream=None):
        r = _lib.CertResult()
        _lib.call("svp_certify_map", self._h, ptr(u_dev), ctypes.byref(r), stream_ptr(stream))
        return r


_CERTIFIERS = {}
_CERT_LOCK = threading.Lock()


def certifier(grid, config):
    """The workspace of (grid, config) on the current device for the calling host thread: registrations that run
    concurrently on their own threads and streams never share a certificate workspace."""
    key = (grid.grid_id, grid.shape, config, torch.cuda.current_device(), threading.get_ident())
    with _CERT_LOCK:
        c = _CERTIFIERS.get(key)
        if c is None:
            if len(_CERTIFIERS) > 16:
                _CERTIFIERS.clear()
            c = _CERTIFIERS[key] = Certifier(grid, config)
    return c


def result_from_record(r, grid, config, state_hash):
    nan_none = lambda x, has=True: float(x) if has and np.isfinite(x) else None
    point = tuple(float(v) for v in r.witness_point) if np.all(np.isfinite(list(r.witness_point))) else None
    return FeasibilityResult(
        status=STATUS[r.status], min_jd_lower_bound=nan_none(r.min_jd_lower_bound, r.has_min_jd),
        min_margin_lower_bound=nan_none(r.min_margin_lower_bound, r.has_min_jd),
        sampled_min_jd=nan_none(r.sampled_min_jd, r.has_sampled_min), n_cells_checked=int(r.n_cells_checked),
        n_uncertain=int(r.n_uncertain), n_infeasible=int(r.n_infeasible), n_boxes=int(r.n_boxes),
        max_depth=int(r.max_depth), witness_cell=None if r.witness_cell < 0 else int(r.witness_cell),
        witness_reference_point=point, reason=REASONS[r.reason], state_hash=state_hash, grid_id=grid.grid_id,
        delta_hex=float(config.delta).hex(), config=config, n_fast_cells=int(r.n_fast_cells),
        n_fallback_cells=int(r.n_fallback_cells), n_prescreen_cells=int(r.n_prescreen_cells))


def _field(u, grid):
    if isinstance(u, torch.Tensor):
        if tuple(u.shape) != tuple(grid.shape) + (3,):
            raise InputValidationError("u: expected grid.shape + (3,)")
        return to_device(u), None
    a = np.ascontiguousarray(np.asarray(u, dtype=np.float64))
    if a.shape != tuple(grid.shape) + (3,):
        raise InputValidationError("u: expected grid.shape + (3,)")
    return to_device(a), a


def certify_map(u, grid, *, config=None, with_hash=True, stream=None):
    """All cells plus six faces and sampling domain (feasibility.py:393).  Host input is hashed (SHA-256 of its
    C-order bytes) as the reference does; a device tensor is hashed only with with_hash=True (one download)."""
    config = CertificateConfig() if config is None else config
    if not isinstance(config, CertificateConfig):
        raise InputValidationError("config: CertificateConfig required")
    dev, host = _field(u, grid)
    record = certifier(grid, config).run(dev, stream)
    digest = None
    if with_hash:
        if host is None:
            host = dev.detach().cpu().numpy()
        digest = hashlib.sha256(memoryview(host).cast("B")).hexdigest()
    return result_from_record(record, grid, config, digest)


def parallel_margins(u, grid, delta, stream=None):
    """(margin float64[ncell], flag bool[ncell]) of the edge-hull enclosure; numpy out for numpy in."""
    require_cuda()
    dev, host = _field(u, grid)
    n = grid.n_cells
    margin = torch.empty(n, dtype=torch.float64, device=dev.device)
    flag = torch.empty(n, dtype=torch.uint8, device=dev.device)
    g = grid_struct(grid)
    _lib.call("svp_edge_hull_margins", ctypes.byref(g), ptr(dev), float(delta), ptr(margin), ptr(flag),
              stream_ptr(stream))
    if host is not None:
        return margin.cpu().numpy(), flag.cpu().numpy().astype(bool)
    return margin, flag.bool()


def _closed27(spacing):
    from itertools import product
    nodes = (0., .5, 1.)
    points = np.array([(x, y, z) for z, y, x in product(nodes, repeat=3)])
    vertices = [(x, y, z) for z, y, x in product((0, 1), repeat=3)]
    D = np.empty((3, 27, 8))
    for a, vertex in enumerate(vertices):
        factors = [points[:, j] if vertex[j] else 1 - points[:, j] for j in range(3)]
        for j in range(3):
            o = [k for k in range(3) if k != j]
            D[j, :, a] = (1 if vertex[j] else -1) / spacing[j] * factors[o[0]] * factors[o[1]]
    return D


def prescreen_lower_bounds(u, grid, coefficients, cells, *, workers=None, stream=None):
    """Rigorous float Bernstein lower bounds of J over each listed cell (NaN where not finite).

    coefficients must be the grid's closed27 Q1 derivative table (the kernel evaluates that table itself)."""
    D = np.asarray(coefficients, dtype=np.float64)
    if D.shape != (3, 27, 8):
        raise InputValidationError("prescreen: closed27 coefficient table (3, 27, 8) required")
    if not np.array_equal(D.view(np.uint64), _closed27(grid.spacing).view(np.uint64)):
        raise InputValidationError("prescreen: coefficients are not this grid's closed27 table")
    dev, host = _field(u, grid)
    cells_t = to_device(cells, dtype=torch.int64)
    out = torch.full((cells_t.numel(),), float("nan"), dtype=torch.float64, device=dev.device)
    if cells_t.numel():
        g = grid_struct(grid)
        _lib.call("svp_prescreen_lower_bounds", ctypes.byref(g), ptr(dev), ptr(cells_t), cells_t.numel(),
                  ptr(out), stream_ptr(stream))
    return out.cpu().numpy() if host is not None else out


def fallback_arrays_device(vertices, spacing, delta, stream=None):
    """(ok uint8[n], p_lo, p_hi, c_lo, c_hi, samples: (n, 27)) as CUDA tensors."""
    require_cuda()
    v = to_device(vertices)
    if v.dim() != 3 or tuple(v.shape[1:]) != (8, 3):
        raise InputValidationError("vertices: expected (cells,8,3)")
    n = v.shape[0]
    outs = [torch.empty((n, 27), dtype=torch.float64, device=v.device) for _ in range(5)]
    ok = torch.empty(n, dtype=torch.uint8, device=v.device)
    h = (ctypes.c_double * 3)(*[float(x) for x in spacing])
    if n:
        _lib.call("svp_fallback_arrays", ptr(v), n, h, float(delta), *[ptr(o) for o in outs], ptr(ok),
                  stream_ptr(stream))
    return (ok, *outs)


def fallback_arrays(vertices, spacing, delta, errors=None):
    """Drop-in for compiled_fallback.fallback_arrays: (p, coefficients, samples) or None if any cell fails."""
    ok, plo, phi, clo, chi, smp = (t.cpu().numpy() for t in fallback_arrays_device(vertices, spacing, delta))
    if not np.all(ok):
        return None
    shape = (len(ok), 3, 3, 3)
    return (Interval(plo.reshape(shape), phi.reshape(shape)), Interval(clo.reshape(shape), chi.reshape(shape)),
            smp.reshape(shape))


def classify_cells(c_lo, c_hi, p_lo, p_hi, delta, max_depth=48, max_boxes=255, stream=None):
    """Subdivision verdicts (feasibility.py:295 _classify) of n cells: list of dicts."""
    arrs = [to_device(np.asarray(a).reshape(-1, 27) if not isinstance(a, torch.Tensor) else a.reshape(-1, 27))
            for a in (c_lo, c_hi, p_lo, p_hi)]
    n = arrs[0].shape[0]
    out = torch.empty((n, ctypes.sizeof(_lib.CellVerdict)), dtype=torch.uint8, device=arrs[0].device)
    if n:
        _lib.call("svp_classify_cells", *[ptr(a) for a in arrs], n, float(delta), int(max_depth), int(max_boxes),
                  ptr(out), stream_ptr(stream))
    raw = out.cpu().numpy()
    res = []
    for k in range(n):
        v = _lib.CellVerdict.from_buffer_copy(raw[k].tobytes())
        res.append(dict(status=v.status, reason=v.reason, boxes=v.boxes, depth=v.depth,
                        margin=v.margin if v.has_margin else None,
                        witness=tuple(v.witness) if v.has_witness else None))
    return res
