"""Whole-cell Jacobian-determinant certificate on the B200 (drop-in for jd_curl/three_d/feasibility.py).

Call surface kept from the reference:
  certify_map(u, grid, *, config)                       feasibility.py:393 (and certify_map_owned :558)
  parallel_margins(u, grid, delta)                      compiled_enclosure.py:303
  prescreen_lower_bounds(u, grid, coefficients, cells)  certificate_prescreen.py:125
  fallback_arrays(vertices, spacing, delta, errors)     compiled_fallback.py:177
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
BASE_VERSION = "q1-3d-interval-bernstein-v1"
CERTIFICATE_VERSION = "q1-3d-parallel-hoisted-edge-hull-float-bernstein-prescreen-compiled-bernstein-v1"


def _integer(value, name, minimum):
    if isinstance(value, bool) or not isinstance(value, (int, np.integer)) or value < minimum:
        raise InputValidationError(f"{name}: expected an integer >= {minimum}")
    return int(value)


def _require(ok, message):
    if not ok:
        raise InputValidationError(message)


# The certificate configuration family of the reference (feasibility.py:22-121), with its defaults, validation and
# isinstance structure: code that picks an execution with isinstance(config, ...) reads these classes the same way.
# Each class selects a GPU execution: the bare class and AdaptiveCertificateConfig prove every cell by interval
# Bernstein subdivision (depth-first for the bare class, lowest bound first for the adaptive one); the Enclosure family
# runs the edge-hull preproof first; PrescreenCertificateConfig adds the float Bernstein prescreen.  The compiled,
# parallel and worker-count fields name the reference's CPU executions, whose results are the same; on the GPU they
# select nothing.
@dataclass(frozen=True)
class CertificateConfig:
    delta: float = .01
    max_depth: int = 12
    max_boxes: int = 255
    tile_size: int = 8192

    def __post_init__(self):
        try:
            d = float(self.delta)
        except (TypeError, ValueError):
            raise InputValidationError("delta: finite real required") from None
        _require(np.isfinite(d), "delta: finite real required")
        _require(0 <= d < 1, "delta: require 0 <= delta < 1")
        object.__setattr__(self, "delta", 0.0 if d == 0 else d)     # one spelling of zero (-0.0 -> +0.0)
        for key, minimum in (("max_depth", 0), ("max_boxes", 1), ("tile_size", 1)):
            object.__setattr__(self, key, _integer(getattr(self, key), key, minimum))

    # GPU execution selected by the class (svp_cert_config.prescreen / .execution)
    @property
    def hull(self):
        return isinstance(self, EnclosureCertificateConfig)

    @property
    def prescreen(self):
        return isinstance(self, PrescreenCertificateConfig)

    @property
    def depth_first(self):
        return not isinstance(self, AdaptiveCertificateConfig)


@dataclass(frozen=True)
class AdaptiveCertificateConfig(CertificateConfig):
    """Lowest-lower-bound-first subdivision with a deeper budget."""
    max_depth: int = 48
    policy: str = "lowest_bound_first_v1"

    def __post_init__(self):
        super().__post_init__()
        _require(self.policy == "lowest_bound_first_v1", "unsupported adaptive certificate policy")
        _require(self.max_depth <= 120, "adaptive max_depth must be <= 120")


@dataclass(frozen=True)
class EnclosureCertificateConfig(AdaptiveCertificateConfig):
    """Edge-hull whole-cell preproof, then the adaptive subdivision of the cells it leaves."""
    prepass: str = "edge_hull_v1"

    def __post_init__(self):
        super().__post_init__()
        _require(self.prepass == "edge_hull_v1", "unsupported enclosure prepass")


@dataclass(frozen=True)
class CompiledEnclosureCertificateConfig(EnclosureCertificateConfig):
    kernel: str = "numba-directed-edge-hull-v1"

    def __post_init__(self):
        super().__post_init__()
        _require(self.kernel in ("numba-directed-edge-hull-v1", "numba-hoisted-edge-hull-v1"),
                 "unsupported compiled enclosure kernel")


@dataclass(frozen=True)
class ParallelEnclosureCertificateConfig(CompiledEnclosureCertificateConfig):
    kernel: str = "numba-parallel-hoisted-edge-hull-v1"
    fallback_workers: int = 8

    def __post_init__(self):
        EnclosureCertificateConfig.__post_init__(self)
        _require(self.kernel == "numba-parallel-hoisted-edge-hull-v1",
                 "parallel certificate requires the parallel hoisted kernel")
        object.__setattr__(self, "fallback_workers", _integer(self.fallback_workers, "fallback_workers", 1))


@dataclass(frozen=True)
class CompiledFallbackCertificateConfig(ParallelEnclosureCertificateConfig):
    fallback_kernel: str = "numba-bernstein-fallback-v1"

    def __post_init__(self):
        super().__post_init__()
        _require(self.fallback_kernel == "numba-bernstein-fallback-v1", "unsupported compiled fallback kernel")


@dataclass(frozen=True)
class PrescreenCertificateConfig(CompiledFallbackCertificateConfig):
    """Hull preproof, the rigorous float Bernstein prescreen of the cells it leaves, then the interval fallback."""
    prescreen_kernel: str = "numba-float-bernstein-apriori-v1"

    def __post_init__(self):
        super().__post_init__()
        _require(self.prescreen_kernel == "numba-float-bernstein-apriori-v1", "unsupported prescreen kernel")


def certificate_version(config):
    """The record's certificate_version for a config (feasibility.py:123-137)."""
    if isinstance(config, PrescreenCertificateConfig):
        return CERTIFICATE_VERSION
    if isinstance(config, CompiledFallbackCertificateConfig):
        return "q1-3d-parallel-hoisted-edge-hull-compiled-bernstein-v1"
    if isinstance(config, ParallelEnclosureCertificateConfig):
        return "q1-3d-parallel-hoisted-edge-hull-bernstein-v1"
    if isinstance(config, CompiledEnclosureCertificateConfig):
        if config.kernel == "numba-hoisted-edge-hull-v1":
            return "q1-3d-hoisted-edge-hull-bernstein-v1"
        return "q1-3d-compiled-edge-hull-bernstein-v1"
    if isinstance(config, EnclosureCertificateConfig):
        return "q1-3d-edge-hull-bernstein-v1"
    return BASE_VERSION


def execution_of(config):
    """(prescreen, execution flags) of svp_cert_config for a config object -- ours or the reference's own classes,
    read by the fields that distinguish them (prepass: edge hull; prescreen_kernel: prescreen; policy: adaptive)."""
    hull = hasattr(config, "prepass")
    prescreen = hasattr(config, "prescreen_kernel")
    adaptive = hasattr(config, "policy")
    flags = (0 if hull else 1) | (0 if adaptive else 2)
    return (1 if prescreen else 0), flags


# The GPU production configuration of the native loop: the prescreen execution with the budgets the reference's
# native route passes (delta 0, depth 48, 255 boxes, tiles of 65536 cells).
NATIVE_CERTIFICATE = PrescreenCertificateConfig(delta=0., max_depth=48, max_boxes=255, tile_size=65536)


@dataclass(frozen=True)
class FeasibilityResult:
    """feasibility.py:148-179 FeasibilityResult fields plus the Enclosure/Prescreen counts (0 where the config's
    execution has no such stage)."""
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
    certificate_version: str = BASE_VERSION
    n_fast_cells: int = 0
    n_fallback_cells: int = 0
    n_prescreen_cells: int = 0


@dataclass(frozen=True)
class Interval:
    lo: np.ndarray
    hi: np.ndarray


class Certifier:
    """Owned device workspace for one (grid, config) pair (libsvp3d svp_certifier).  directed=True selects the
    directed-rounding arithmetic of the mixed form (valid enclosures at least as tight as the reference's)."""

    def __init__(self, grid, config, directed=False):
        require_cuda()
        self.grid, self.config, self.directed = grid, config, bool(directed)
        self._g = grid_struct(grid)
        prescreen, execution = execution_of(config)
        execution |= 4 if directed else 0          # SVP_CERT_DIRECTED
        cfg = _lib.CertConfig(config.delta, config.max_depth, config.max_boxes, config.tile_size, prescreen, execution)
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


def certifier(grid, config, directed=False):
    """The workspace of (grid, config) on the current device for the calling host thread: registrations that run
    concurrently on their own threads and streams never share a certificate workspace."""
    key = (grid.grid_id, grid.shape, config, bool(directed), torch.cuda.current_device(), threading.get_ident())
    with _CERT_LOCK:
        c = _CERTIFIERS.get(key)
        if c is None:
            if len(_CERTIFIERS) > 16:
                _CERTIFIERS.clear()
            c = _CERTIFIERS[key] = Certifier(grid, config, directed)
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
        delta_hex=float(config.delta).hex(), config=config, certificate_version=certificate_version(config),
        n_fast_cells=int(r.n_fast_cells),
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


def certify_map(u, grid, *, config=None, with_hash=True, stream=None, directed=False):
    """All cells plus six faces and sampling domain (feasibility.py:393).  Host input is hashed (SHA-256 of its
    C-order bytes) as the reference does; a device tensor is hashed only with with_hash=True (one download)."""
    config = CertificateConfig() if config is None else config
    if not isinstance(config, CertificateConfig):
        raise InputValidationError("config: CertificateConfig required")
    dev, host = _field(u, grid)
    record = certifier(grid, config, directed).run(dev, stream)
    digest = None
    if with_hash:
        if host is None:
            host = dev.detach().cpu().numpy()
        digest = hashlib.sha256(memoryview(host).cast("B")).hexdigest()
    return result_from_record(record, grid, config, digest)


def parallel_margins(u, grid, delta, stream=None, directed=False):
    """(margin float64[ncell], flag bool[ncell]) of the edge-hull enclosure; numpy out for numpy in."""
    require_cuda()
    dev, host = _field(u, grid)
    n = grid.n_cells
    margin = torch.empty(n, dtype=torch.float64, device=dev.device)
    flag = torch.empty(n, dtype=torch.uint8, device=dev.device)
    g = grid_struct(grid)
    _lib.call("svp_edge_hull_margins_directed" if directed else "svp_edge_hull_margins", ctypes.byref(g), ptr(dev),
              float(delta), ptr(margin), ptr(flag), stream_ptr(stream))
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


def fallback_arrays_device(vertices, spacing, delta, stream=None, directed=False):
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
        _lib.call("svp_fallback_arrays_directed" if directed else "svp_fallback_arrays", ptr(v), n, h, float(delta),
                  *[ptr(o) for o in outs], ptr(ok), stream_ptr(stream))
    return (ok, *outs)


def fallback_arrays(vertices, spacing, delta, errors=None):
    """Drop-in for compiled_fallback.fallback_arrays: (p, coefficients, samples) or None if any cell fails."""
    ok, plo, phi, clo, chi, smp = (t.cpu().numpy() for t in fallback_arrays_device(vertices, spacing, delta))
    if not np.all(ok):
        return None
    shape = (len(ok), 3, 3, 3)
    return (Interval(plo.reshape(shape), phi.reshape(shape)), Interval(clo.reshape(shape), chi.reshape(shape)),
            smp.reshape(shape))


def classify_cells(c_lo, c_hi, p_lo, p_hi, delta, max_depth=48, max_boxes=255, depth_first=False, stream=None,
                   directed=False):
    """Subdivision verdicts (feasibility.py:295 _classify) of n cells: list of dicts.  depth_first selects the bare
    CertificateConfig's order (a stack, left child first); the default is the adaptive lowest-bound-first order."""
    arrs = [to_device(np.asarray(a).reshape(-1, 27) if not isinstance(a, torch.Tensor) else a.reshape(-1, 27))
            for a in (c_lo, c_hi, p_lo, p_hi)]
    n = arrs[0].shape[0]
    out = torch.empty((n, ctypes.sizeof(_lib.CellVerdict)), dtype=torch.uint8, device=arrs[0].device)
    if n:
        _lib.call("svp_classify_cells_policy", *[ptr(a) for a in arrs], n, float(delta), int(max_depth),
                  int(max_boxes), (1 if depth_first else 0) | (2 if directed else 0), ptr(out), stream_ptr(stream))
    raw = out.cpu().numpy()
    res = []
    for k in range(n):
        v = _lib.CellVerdict.from_buffer_copy(raw[k].tobytes())
        res.append(dict(status=v.status, reason=v.reason, boxes=v.boxes, depth=v.depth,
                        margin=v.margin if v.has_margin else None,
                        witness=tuple(v.witness) if v.has_witness else None))
    return res
