"""Float32 pyramid pre-optimizer and its certified hand-over to the native solve (the config-2 route).

Mirrors jd_curl/three_d/preopt.py:506 preoptimize (levels 8/4/2/1, Adam on the float32 pre-objective, the step
capped at `cap` voxels, Gaussian-smoothed gradient and field), preopt.py:617 boundary_taper, multiresolution.py:45
four_level_grids / :55 prolong_displacement, nifti.py:128 downsample_array and multiresolution.py:111
prepare_transfer_problem (the first certified scale 0.9^k of the tapered seed).  The pre-optimizer is an
UNCERTIFIED initializer: its output becomes a formal state only through the certificate of the transfer, exactly as
in the reference.  Every iteration runs on the device (libsvp3d svp_pre_level); the host touches a level's record
floats once per level.
"""
import ctypes
from dataclasses import asdict, dataclass
from time import perf_counter

import numpy as np
import torch

from . import _lib
from . import certificate as cert_mod
from .device import ptr, require_cuda, stream_ptr, to_device
from .grid import InputValidationError, make_grid_3d

FACTORS = (8, 4, 2, 1)
PREOPT_POLICY = "fp32-preopt-v1"
TRANSFER_ALPHAS = tuple(.9 ** k for k in range(7))      # multiresolution.py:89 TRANSFER_BACKTRACK_ALPHAS
TERMS = ("data", "geometry", "floor", "curvature", "min_det", "total")


@dataclass(frozen=True)
class PreoptConfig:
    """preopt.py:32 PreoptConfig (same fields and defaults)."""
    iterations: tuple = (80, 80, 60, 40)
    lr: float = .25
    cap: float = .5
    sigma_grad: float = 1.
    sigma_field: float = 0.
    mu: tuple = (1., 1., .1, .03)
    alpha: tuple = (1e-3, 1e-3, 1e-3, 0.)
    kappa_pre: float = 10.
    j0: float = .2
    seconds: float = 8.
    beta1: float = .9
    beta2: float = .99
    eps: float = 1e-8

    def __post_init__(self):
        if len(self.iterations) != 4 or any(int(n) != n or n < 0 for n in self.iterations):
            raise InputValidationError("preopt iterations: four nonnegative integers")
        for name in ("lr", "cap", "kappa_pre", "j0", "seconds", "beta1", "beta2", "eps"):
            v = float(getattr(self, name))
            if not np.isfinite(v) or v <= 0:
                raise InputValidationError(f"preopt {name}: positive finite")
        if self.sigma_grad < 0 or self.sigma_field < 0 or not (self.beta1 < 1 and self.beta2 < 1) or self.j0 >= 1:
            raise InputValidationError("preopt: sigma >= 0, betas < 1, j0 < 1")
        for name in ("mu", "alpha"):
            vals = getattr(self, name)
            if len(vals) != 4 or any(not np.isfinite(v) or v < 0 for v in vals):
                raise InputValidationError(f"preopt {name}: four finite nonnegative numbers")
        if any(m <= 0 for m in self.mu):
            raise InputValidationError("preopt mu: positive")


# The reference's documented native run (docs/usage.md 3.1: --pre-optimizer "fp32-v1:iterations=50/50/100/60,
# lr=0.5,cap=0.5,sigma_grad=1,sigma_field=1,mu=1/1/0.01/0.003,alpha=1e-3/1e-3/1e-3/0,kappa_pre=10,j0=0.2,seconds=60,
# taper=4").
NATIVE_PREOPT = PreoptConfig(iterations=(50, 50, 100, 60), lr=.5, cap=.5, sigma_grad=1., sigma_field=1.,
                             mu=(1., 1., .01, .003), alpha=(1e-3, 1e-3, 1e-3, 0.), kappa_pre=10., j0=.2, seconds=60.)
NATIVE_TAPER = 4


def coarse_grid(grid, shape_zyx):
    """nifti.py:112: the same node-centre FOV on a coarser node count."""
    if any(n < 5 or n > old for n, old in zip(shape_zyx, grid.shape)):
        raise InputValidationError("target axes must be >=5 and no larger than source")
    spacing = tuple((axis[-1] - axis[0]) / (n - 1) for axis, n in zip(grid.axes, shape_zyx[::-1]))
    return make_grid_3d(nx=shape_zyx[2], ny=shape_zyx[1], nz=shape_zyx[0], hx=spacing[0], hy=spacing[1],
                        hz=spacing[2], x0=grid.axes[0][0], y0=grid.axes[1][0], z0=grid.axes[2][0], unit=grid.unit)


def four_level_grids(native):
    """multiresolution.py:45: levels 8/4/2/1 preserving the physical node-centre FOV."""
    if native.unit != "mm":
        raise InputValidationError("four-level registration requires a physical mm grid")
    shapes = [tuple((n - 2 + s) // s + 1 for n in native.shape) for s in FACTORS]
    if any(n < 5 for shape in shapes for n in shape):
        raise InputValidationError("all four levels need >=5 nodes on every axis")
    return tuple(coarse_grid(native, shape) for shape in shapes[:-1]) + (native,)


def _prolong_tables(source, target):
    """Per-axis (left index, weight) of multiresolution.py:55 prolong_displacement, in z, y, x order."""
    lefts, weights = [], []
    for old, new, h in zip(source.axes[::-1], target.axes[::-1], source.spacing[::-1]):
        tol = 32 * np.finfo(float).eps * max(1., np.max(np.abs(old)), np.max(np.abs(new)))
        if len(new) < len(old) or not np.allclose(old[[0, -1]], new[[0, -1]], rtol=0., atol=tol):
            raise InputValidationError("transfer must refine the same physical FOV")
        t = (new - old[0]) / h
        t[0], t[-1] = 0., len(old) - 1
        if np.any(t[1:-1] <= 0) or np.any(t[1:-1] >= len(old) - 1):
            raise InputValidationError("target interior is not inside the source FOV")
        left = np.floor(t).astype(np.int64)
        left[-1] = len(old) - 2
        lefts.append(left)
        weights.append(t - left)
    return np.concatenate(lefts).astype(np.int32), np.concatenate(weights)


def prolong_displacement(u, source, target, stream=None):
    """Q1 transfer of a device displacement (source.shape + (3,)) onto the finer target grid (device)."""
    left, weight = _prolong_tables(source, target)
    out = torch.empty(target.shape + (3,), dtype=torch.float64, device=u.device)
    sz, sy, sx = source.shape
    tz, ty, tx = target.shape
    _lib.call("svp_field_prolong", ptr(u), sz, sy, sx, ptr(out), tz, ty, tx,
              left.ctypes.data_as(ctypes.c_void_p), weight.ctypes.data_as(ctypes.c_void_p), stream_ptr(stream))
    return out


def downsample(image, source, target, stream=None):
    """nifti.py:128 downsample_array on the device (image: device float64, source.shape)."""
    out = torch.empty(target.shape, dtype=torch.float64, device=image.device)
    nz, ny, nx = source.shape
    mz, my, mx = target.shape
    _lib.call("svp_image_downsample", ptr(image), nz, ny, nx, ptr(out), mz, my, mx, stream_ptr(stream))
    return out


def pre_energy_grad(fixed32, moving32, grid, u_int, mu, alpha, kappa, j0, stream=None):
    """(terms dict, gradient) of the float32 pre-objective at u_int (3, D-2, H-2, W-2) voxels (device)."""
    D, H, W = grid.shape
    grad = torch.empty_like(u_int)
    t = (ctypes.c_float * 6)()
    hx, hy, hz = grid.spacing
    _lib.call("svp_pre_energy_grad", ptr(fixed32), ptr(moving32), D, H, W, hx, hy, hz, ptr(u_int), float(mu),
              float(alpha), float(kappa), float(j0), ptr(grad), t, stream_ptr(stream))
    return dict(zip(TERMS, (float(v) for v in t))), grad


def preoptimize(fixed, moving, grid, config=None, stream=None):
    """preopt.py:506: (u float64 (nz, ny, nx, 3) in mm with zero faces, on the device; record).  Uncertified."""
    require_cuda()
    config = PreoptConfig() if config is None else config
    dev = torch.device("cuda")
    f64, m64 = to_device(fixed), to_device(moving)
    started = perf_counter()
    grids = four_level_grids(grid)
    levels, u_mm, cap_total = [], None, 0
    for level, lg in enumerate(grids):
        tick = perf_counter()
        if level == 3:
            F, M = f64, m64
        else:
            F, M = downsample(f64, grid, lg, stream), downsample(m64, grid, lg, stream)
        h = np.array(lg.spacing)
        if u_mm is None:
            u_int = torch.zeros((3,) + lg.interior_shape, dtype=torch.float32, device=dev)
        else:
            seed = prolong_displacement(u_mm, grids[level - 1], lg, stream)
            vox = seed[1:-1, 1:-1, 1:-1].permute(3, 0, 1, 2) / torch.as_tensor(h, device=dev)[:, None, None, None]
            u_int = vox.to(torch.float32).contiguous()
        m, v = torch.zeros_like(u_int), torch.zeros_like(u_int)
        prm = _lib.PreParams(config.mu[level], config.alpha[level], config.kappa_pre, config.j0, config.lr, config.cap,
                             config.sigma_grad, config.sigma_field, config.beta1, config.beta2, config.eps)
        first, last = (ctypes.c_float * 6)(), (ctypes.c_float * 6)()
        hits = ctypes.c_int64()
        D, H, W = lg.shape
        n_it = int(config.iterations[level])
        F32, M32 = F.to(torch.float32).contiguous(), M.to(torch.float32).contiguous()
        if n_it:
            _lib.call("svp_pre_level", ptr(F32), ptr(M32), D, H, W, *lg.spacing, ctypes.byref(prm), 0, n_it,
                      ptr(u_int), ptr(m), ptr(v), first, last, ctypes.byref(hits), stream_ptr(stream))
            if not np.isfinite(last[5]):
                raise FloatingPointError("preopt: nonfinite pre-objective")
        out = torch.zeros(lg.shape + (3,), dtype=torch.float64, device=dev)
        out[1:-1, 1:-1, 1:-1] = u_int.double().permute(1, 2, 3, 0) * torch.as_tensor(h, device=dev)
        u_mm = out
        cap_total += hits.value
        levels.append(dict(level=level, shrink_factor=FACTORS[level], shape_zyx=list(lg.shape), iterations=n_it,
                           seconds=perf_counter() - tick,
                           first=dict(zip(TERMS, (float(x) for x in first))) if n_it else None,
                           last=dict(zip(TERMS, (float(x) for x in last))) if n_it else None))
    record = dict(policy=PREOPT_POLICY, config=asdict(config), device="cuda", dtype="float32", levels=levels,
                  cap_hits=int(cap_total), stopped=None, seconds=perf_counter() - started,
                  role="uncertified_preoptimizer_initializer_NOT_outer_commit")
    return u_mm, record


def boundary_taper(u, grid, L=4):
    """preopt.py:617: nodes within L of a face scale linearly to zero on the face.  Returns (tapered u, weights),
    the weights on the input's side (a device u gets them formed on the device from the three axis profiles: the
    same products in the same order as the host form)."""
    rs = []
    for n in grid.shape:
        k = np.arange(n)
        rs.append(np.minimum(np.minimum(k, n - 1 - k) / float(L), 1.))
    if torch.is_tensor(u):
        r = [torch.as_tensor(a, device=u.device) for a in rs]
        w = r[0][:, None, None] * r[1][None, :, None] * r[2][None, None, :]
    else:
        w = rs[0][:, None, None] * rs[1][None, :, None] * rs[2][None, None, :]
    return (w[..., None] * u), w


def transfer(seed, grid, certificate_config=None):
    """multiresolution.py:111 prepare_transfer_problem: the first scale alpha in 0.9^k (k = 0..6) whose
    alpha * seed the whole-cell certificate proves (J > 0 on every closed cell).  Returns (field or None, report)."""
    # the reference's transfer default (multiresolution.py:127): the edge-hull execution with strict J > 0
    config = cert_mod.EnclosureCertificateConfig(delta=0.) if certificate_config is None else certificate_config
    if not isinstance(config, cert_mod.EnclosureCertificateConfig) or config.delta != 0.:
        raise InputValidationError("transfer recovery requires whole-cell strict JD>0 certification")
    certifier = cert_mod.certifier(grid, config)
    attempts = []
    started = perf_counter()
    for index, alpha in enumerate(TRANSFER_ALPHAS):
        field = seed if index == 0 else (alpha * seed)
        rec = certifier.run(field.contiguous())
        proof = cert_mod.result_from_record(rec, grid, config, None)
        attempts.append(dict(attempt_index=index, alpha=alpha, status=proof.status, reason=proof.reason,
                             min_jd_lower_bound=proof.min_jd_lower_bound))
        if proof.status == "certified_feasible":
            return field, dict(status="ready", attempts=attempts, accepted_alpha=alpha,
                               displacement_loss_fraction=1 - alpha, elapsed_seconds=perf_counter() - started,
                               role="initializer_only_NOT_outer_commit")
        if proof.reason not in ("JACOBIAN_VIOLATION", "subdivision_budget", "INVALID_DOMAIN"):
            break
    return None, dict(status="rejected", attempts=attempts, accepted_alpha=None,
                      elapsed_seconds=perf_counter() - started, role="initializer_only_NOT_outer_commit")


def register_pair(fixed, moving, grid, weights, *, preopt=NATIVE_PREOPT, taper=NATIVE_TAPER, outer=200,
                  inner_config=None, certificate_config=None, precision="plain"):
    """The config-2 route: pyramid pre-optimization, boundary taper, certified transfer, then the certified native
    proximal solve from the transferred field (which is also its proximal reference).  Returns
    (SequentialResult, record).  Without a certified transfer the native solve starts from u = 0."""
    from .solver import PGConfig3D, Registration, SequentialConfig3D, solve_sequential
    record = {}
    field = None
    if preopt is not None:
        raw, record["preopt"] = preoptimize(fixed, moving, grid, preopt)
        seed, _ = boundary_taper(raw, grid, taper)
        field, record["transfer"] = transfer(seed.contiguous(), grid)
    reg = Registration(grid, fixed, moving, **weights, u_ref=None if field is None else field,
                       certificate_config=certificate_config, precision=precision)
    theta0 = None if field is None else reg.pair.restrict(field)
    res = solve_sequential(reg, theta0, config=SequentialConfig3D(max_iterations=outer),
                           inner_config=PGConfig3D() if inner_config is None else inner_config)
    return res, record
