"""B200Backend: the reference loop's `backend=` plug-in, served by libsvp3d's sm_100a kernels.

jd_curl's solvers take a GPU plug-in through one argument, `backend=`:
  jd_curl/three_d/sequential.py:165 solve_sequential(problem, theta, ..., backend=...)
  jd_curl/three_d/solvers/poisson_gradient.py:1090 solve_poisson_gradient(problem, theta, ..., backend=...)
The reference fills it with backends/accelerated.py:363 AcceleratedHybridBackend (Torch + Triton).  This class has
the same call surface, so that loop runs unchanged on a B200 with this library doing the work:

  evaluate_trial(problem, theta, *, certificate_observer, witness_observer)  accelerated.py:1667
  promote_trial(problem, trial)                                               accelerated.py:2851
  gradient(lin, target)                                                       accelerated.py:923, hybrid.py:69
  poisson(inverse) -> object with apply / prepare_equilibrated / apply_equilibrated    hybrid.py:77, :225-286
  diagonal(lin), diagonal_launch(lin)                                         hybrid.py:81-91
  node_min_jd(lin, *, extension_activation, stats, compiled)                 hybrid.py:98
  global_jd_root(lin, direction, limit)                                       hybrid.py:93
  linearize(lin) -> gradient() / diagonal() / hvp(p)                          hybrid.py:59
  stable_energy_reduction(problem, base, trial, *, outer_only, required_reduction)   accelerated.py:3114
  stable_energy_reductions(problem, base, trial, *, required_reduction)      accelerated.py:3121
  outer_gradient_vectors(lin), outer_norms(lin, omega)                        accelerated.py:3126, :3164
  cpu_state(problem, state, *, promote)                                       accelerated.py:2924
  device.upload / device.download / device.synchronize                        backends/torch_ops.py Device

States cross the boundary as the reference's own types (TrialState3D, AcceptedState3D, FeasibilityResult,
EnergyTerms3D, EnergyReduction, InvalidTrial), with host numpy arrays, exactly as the reference's plug-in returns
them; the jd_curl package is imported from the caller's environment when a method first needs one of its types.
Device copies of every state this backend evaluated stay resident (u, warped image, image gradient, barrier
activity mask), keyed by the state's eval_id, so a gradient or a comparison does not upload them again.

Decisions follow the reference's CPU rules: comparisons return the stable differences with the 16 eps max(E)
resolution of energy_comparison.py:117-122, and a comparison within a few resolutions of its decision threshold, or
a gradient norm within 1% of the forcing target (the reference plug-in's own rule, hybrid.py:69-75), is redone by
the reference's CPU functions on the same states.  Everything else runs on the GPU; there is no CPU fallback for
missing hardware (constructing the backend without CUDA raises).
"""
from collections import OrderedDict
import hashlib
from time import perf_counter

import numpy as np
import torch

from . import _lib
from . import certificate as cert_mod
from .device import require_cuda, to_device
from .grid import make_grid_3d
from .pair import DevicePair

BACKEND_ID = "b200-sm100a-libsvp3d-float64"
EPS = float(np.finfo(float).eps)
# a GPU comparison this close (in resolutions) to its decision is redone by the reference CPU comparison
CRITICAL_RESOLUTIONS = 4.
# gradient norms within this factor of the forcing target are recomputed on the CPU (hybrid.py:72)
GRADIENT_RECHECK = 1.01


def _jd():
    """The reference package's types and helpers (imported on first use from the caller's environment)."""
    from jd_curl.three_d import feasibility as F
    from jd_curl.three_d import residuals as R
    from jd_curl import energy_comparison as EC
    from jd_curl.three_d import energy_comparison as EC3
    from jd_curl.three_d import linearization as L
    from jd_curl.types import InvalidTrial
    from jd_curl.validation import StateMismatchError, InputValidationError, require_finite_result
    from jd_curl.three_d.solvers.common import gradient_norm_mass
    return dict(F=F, R=R, EC=EC, EC3=EC3, L=L, InvalidTrial=InvalidTrial, StateMismatchError=StateMismatchError,
                InputValidationError=InputValidationError, require_finite_result=require_finite_result,
                gradient_norm_mass=gradient_norm_mass)


def _frozen(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    a.flags.writeable = False
    return a


class Device:
    """upload / download / synchronize of the reference's backends/torch_ops.py Device, on the current CUDA device."""

    def __init__(self, device="cuda"):
        require_cuda()
        self.device = torch.device(device)

    def upload(self, a):
        return to_device(a, device=self.device)

    def download(self, t):
        return t.detach().cpu().numpy()

    def synchronize(self):
        torch.cuda.synchronize(self.device)


class _Pending:
    """diagonal_launch's result: the device work is queued; result() checks and downloads (hybrid.py:195)."""

    def __init__(self, backend, tensor):
        self._backend, self._tensor = backend, tensor

    def result(self):
        t, self._tensor = self._tensor, None
        return self._backend._checked_diagonal(t)


class _Linearized:
    """Device view of one reference Linearization3D (hybrid.py:59 linearize): derivative kernels of its state."""

    def __init__(self, backend, lin):
        self.backend, self.lin = backend, lin
        self.pair, self.state = backend._bind(lin.problem), backend._device_state(lin.problem, lin.state, promote=True)

    def gradient(self, term="total"):
        s = self.state
        return self.pair.gradient(s["u"], s["warped"], s["image_grad"], term=term, active=s["active"])

    def diagonal(self):
        s = self.state
        return self.pair.ggn_diagonal(s["u"], s["image_grad"], active=s["active"])

    def hvp(self, p):
        s = self.state
        return self.pair.ggn_hvp(s["u"], s["image_grad"], self.backend.device.upload(p))


class _Poisson:
    """The object backend.poisson(inverse) returns (hybrid.py:210 _HostPoisson): inverse.apply on the device, with the
    reference's a, b and metric, plus the pre-scaled equilibrated form prepare/apply_equilibrated."""

    METRICS = {"q1": 0, "seven_point": 1, "seven-point": 1}

    def __init__(self, backend, inverse):
        self.backend, self.inverse = backend, inverse
        metric = getattr(inverse, "metric", "q1")
        if metric not in self.METRICS:
            raise _jd()["InputValidationError"](f"Poisson metric {metric!r} is not served by this backend")
        self.a, self.b, self.metric = float(inverse.a), float(inverse.b), metric
        self.grid = inverse.grid
        self._scale = None

    @property
    def shape(self):
        return self.inverse.shape

    def _pair(self):
        return self.backend._grid_pair(self.grid)

    def apply(self, rhs):
        b = self.backend
        started = perf_counter()
        x = self._pair().poisson_apply(self.a, self.b, b.device.upload(np.asarray(rhs, dtype=np.float64).ravel()),
                                       metric=self.metric)
        out = b.device.download(x)
        _jd()["require_finite_result"](out, "Poisson inverse")
        b._time("poisson", started)
        return out

    def prepare_equilibrated(self, scale, gradient):
        """(device scale, device gradient) for apply_equilibrated, or None when s * g is not finite."""
        dev = self.backend.device
        if self._scale is None or self._scale[0] is not scale:
            self._scale = (scale, dev.upload(scale))
        g = dev.upload(gradient)
        if not bool(torch.isfinite(self._scale[1] * g).all()):
            return None
        return self._scale[1], g

    def apply_equilibrated(self, prepared, between=None):
        """-(s * M^-1 (s * g)) on the device: (direction, True), or ("x", M^-1 (s * g)) when it is not finite."""
        b = self.backend
        started = perf_counter()
        s, g = prepared
        out = self._pair().poisson_apply(self.a, self.b, g, metric=self.metric, scale=s, sign=-1.)
        if between is not None:
            between()
        finite = bool(torch.isfinite(out).all())
        if not finite:
            x = self._pair().poisson_apply(self.a, self.b, s * g, metric=self.metric)
            b._time("poisson", started)
            return "x", b.device.download(x)
        host = b.device.download(out)
        b._time("poisson", started)
        return host, True


class B200Backend:
    """Drop-in `backend=` of jd_curl's sequential / PG solvers on one B200 (see the module docstring)."""

    def __init__(self, device="cuda", *, max_states=6):
        self.device = Device(device)
        self.backend_id = BACKEND_ID
        self.evaluation_backend_id = BACKEND_ID
        self.timings = {}
        self.cpu_gradient_checks = 0
        self.comparison_counts = dict(gpu=0, cpu=0)
        self.last_comparison = {}             # read by the reference loops for their attempt rows
        self._max_states = int(max_states)
        self._states = OrderedDict()          # eval_id -> device fields of an evaluated state
        self._pairs = {}                      # (grid id, image ids, weights, activation, delta) -> DevicePair
        self._bound = {}                      # id(pair) -> problem_id whose u_ref the pair holds
        self._grids = {}                      # grid id -> our Grid3D
        self._certifiers = {}

    # ------------------------------------------------------------------ bookkeeping
    def _time(self, name, started):
        self.timings[name] = self.timings.get(name, 0.) + perf_counter() - started

    def _grid(self, grid):
        g = self._grids.get(grid.grid_id)
        if g is None:
            nz, ny, nx = grid.shape
            hx, hy, hz = grid.spacing
            x0, y0, z0 = (float(a[0]) for a in grid.axes)
            g = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=hx, hy=hy, hz=hz, x0=x0, y0=y0, z0=z0, unit=grid.unit)
            if g.grid_id != grid.grid_id:
                raise _jd()["StateMismatchError"]("grid id differs from the reference's for the same arguments")
            self._grids[grid.grid_id] = g
        return g

    @staticmethod
    def _supported(problem):
        err = _jd()["InputValidationError"]
        if problem.barrier_location != "closed27_uniform" or problem.barrier_activation is None:
            raise err("B200Backend serves the closed27 localized barrier route")
        if getattr(problem, "barrier_basis", "samples") != "samples":
            raise err("B200Backend serves the sampled barrier (barrier_basis='samples')")
        if getattr(problem, "curvature_weight", 0.) or getattr(problem, "data_weight", None) is not None:
            raise err("B200Backend serves the default energy (no curvature term, unit data weights)")
        if getattr(problem, "active_weights", None) is not None:
            raise err("B200Backend does not serve active-set weights")

    def _pair_key(self, problem):
        w = problem.weights
        return (problem.grid.grid_id, problem.sampler.image_id, id(problem.fixed_image), w.lam, w.mu, w.nu, w.kappa,
                float(problem.barrier_activation), float(problem.certificate_config.delta))

    def _bind(self, problem):
        """The device pair of this problem's images and weights, holding this problem's reference u_ref."""
        self._supported(problem)
        key = self._pair_key(problem)
        pair = self._pairs.get(key)
        if pair is None:
            grid = self._grid(problem.grid)
            w = problem.weights
            coeff = np.asarray(problem.sampler._spline.c, dtype=np.float64)
            pair = DevicePair(grid, problem.fixed_image, coeff, problem.controls.u_ref, lam=w.lam, mu=w.mu, nu=w.nu,
                              kappa=w.kappa, activation=problem.barrier_activation,
                              delta=problem.certificate_config.delta)
            # the reference sampler's own coefficients (the device prefilter of `coeff` above is replaced)
            pair.set_spline_coefficients(coeff)
            if len(self._pairs) >= 4:
                self._pairs.clear()
                self._bound.clear()
            self._pairs[key] = pair
            self._bound[id(pair)] = problem.problem_id
        elif self._bound.get(id(pair)) != problem.problem_id:
            pair.set_reference(problem.controls.u_ref)
            self._bound[id(pair)] = problem.problem_id
        return pair

    def _grid_pair(self, grid):
        for key, pair in self._pairs.items():
            if key[0] == grid.grid_id:
                return pair
        raise _jd()["StateMismatchError"]("Poisson apply before any state of this grid was evaluated")

    def _certifier(self, problem):
        config = problem.certificate_config
        key = (problem.grid.grid_id, config)
        c = self._certifiers.get(key)
        if c is None:
            c = self._certifiers[key] = cert_mod.Certifier(self._grid(problem.grid), config)
        return c

    def _remember(self, eval_id, fields):
        self._states[eval_id] = fields
        self._states.move_to_end(eval_id)
        while len(self._states) > self._max_states:
            self._states.popitem(last=False)

    def _device_state(self, problem, state, promote=False):
        """Device fields of a reference state (uploaded once if this backend did not evaluate it)."""
        s = self._states.get(state.eval_id)
        if s is None:
            s = dict(u=self.device.upload(state.u), warped=self.device.upload(state.warped), image_grad=None,
                     active=None)
            self._remember(state.eval_id, s)
        else:
            self._states.move_to_end(state.eval_id)
        if promote and s["image_grad"] is None:
            ig = getattr(state, "image_grad", None)
            s["image_grad"] = (self.device.upload(ig) if ig is not None else
                               self._bind(problem).warp(s["u"], with_gradient=True)[1])
        return s

    # ------------------------------------------------------------------ certificate record in the reference's type
    def _record(self, problem, rec, state_hash):
        F = _jd()["F"]
        config = problem.certificate_config
        mine = cert_mod.result_from_record(rec, self._grid(problem.grid), config, state_hash)
        common = dict(status=mine.status, min_jd_lower_bound=mine.min_jd_lower_bound,
                      min_margin_lower_bound=mine.min_margin_lower_bound, sampled_min_jd=mine.sampled_min_jd,
                      n_cells_checked=mine.n_cells_checked, n_uncertain=mine.n_uncertain,
                      n_infeasible=mine.n_infeasible, n_boxes=mine.n_boxes, max_depth=mine.max_depth,
                      witness_cell=mine.witness_cell, witness_reference_point=mine.witness_reference_point,
                      reason=mine.reason, state_hash=state_hash, grid_id=problem.grid.grid_id,
                      delta_hex=config.delta.hex(), config=config,
                      certificate_version=F.certificate_version(config))
        if isinstance(config, F.PrescreenCertificateConfig):
            return F.PrescreenFeasibilityResult(**common, n_fast_cells=mine.n_fast_cells,
                                                n_fallback_cells=mine.n_fallback_cells,
                                                n_prescreen_cells=mine.n_prescreen_cells)
        if isinstance(config, F.EnclosureCertificateConfig):
            return F.EnclosureFeasibilityResult(**common, n_fast_cells=mine.n_fast_cells,
                                                n_fallback_cells=mine.n_fallback_cells)
        return F.FeasibilityResult(**common)

    # ------------------------------------------------------------------ evaluation (accelerated.py:1667, :2851)
    def evaluate_trial(self, problem, theta, *, certificate_observer=None, witness_observer=None):
        """Certify, sample and evaluate theta: TrialState3D, or InvalidTrial with the reference's reasons
        (residuals.py:209-236)."""
        J = _jd()
        started = perf_counter()
        theta = np.asarray(theta, dtype=np.float64)
        if theta.shape != (3 * problem.grid.n_free_scalar,):
            raise J["InputValidationError"]("theta: expected shape (3 * n_free,)")
        bad = ~np.isfinite(theta)
        if bad.any():
            return J["InvalidTrial"]("NONFINITE_STATE", "nonfinite free displacement", int(bad.sum()))
        theta = _frozen(theta.copy())
        pair = self._bind(problem)
        u_dev = pair.inject(self.device.upload(theta))
        rec = self._certifier(problem).run(u_dev)
        u = _frozen(self.device.download(u_dev))
        certificate = self._record(problem, rec, hashlib.sha256(memoryview(u).cast("B")).hexdigest())
        if certificate_observer is not None:
            certificate_observer(certificate)
        if certificate.status != "certified_feasible":
            reason = "FEASIBILITY_UNCERTAIN" if certificate.status == "uncertain" else certificate.reason
            self._time("evaluate_trial", started)
            return J["InvalidTrial"](reason, "trial not certified: " + certificate.reason,
                                     certificate.n_uncertain + certificate.n_infeasible)
        warped_dev, grad_dev = pair.warp(u_dev, with_gradient=True)
        terms, violations = pair.energy(u_dev, warped_dev)
        if violations or not np.all(np.isfinite(terms)):
            self._time("evaluate_trial", started)
            return J["InvalidTrial"]("NONFINITE_STATE",
                                     "floating barrier-point evaluation contradicts feasible certificate", 1)
        energy = J["R"].EnergyTerms3D(*(float(t) for t in terms))
        eval_id = hashlib.sha256((problem.problem_id + certificate.state_hash).encode()).hexdigest()
        self._remember(eval_id, dict(u=u_dev, warped=warped_dev, image_grad=grad_dev, active=None))
        state = J["R"].TrialState3D(theta, u, _frozen(self.device.download(warped_dev)), energy, certificate,
                                    problem.problem_id, eval_id)
        self._time("evaluate_trial", started)
        return state

    def promote_trial(self, problem, trial):
        """AcceptedState3D with the physical image gradient at X + u (residuals.py:238)."""
        J = _jd()
        J["R"].validate_state(problem, trial)
        started = perf_counter()
        s = self._device_state(problem, trial)
        if s["image_grad"] is None:
            warped, s["image_grad"] = self._bind(problem).warp(s["u"], with_gradient=True)
            if not torch.equal(warped, s["warped"]):
                raise J["StateMismatchError"]("promoted sampler value changed from certified trial")
        out = J["R"].AcceptedState3D(trial.theta, trial.u, trial.warped, trial.energy, trial.certificate,
                                     trial.problem_id, trial.eval_id, _frozen(self.device.download(s["image_grad"])))
        self._time("promote_trial", started)
        return out

    def cpu_state(self, problem, state, *, promote=True):
        """The reference's CPU evaluation (and promotion) of the same theta (accelerated.py:2924)."""
        R = _jd()["R"]
        trial = R.evaluate_trial(problem, state.theta)
        if isinstance(trial, _jd()["InvalidTrial"]) or not promote:
            return trial
        return R.promote_trial(problem, trial)

    # ------------------------------------------------------------------ derivatives
    def linearize(self, lin):
        return _Linearized(self, lin)

    def gradient(self, lin, target):
        """Total gradient on the free nodes (host), recomputed by the reference CPU gradient when its norm is within
        1% of the forcing target (hybrid.py:69-75)."""
        J = _jd()
        started = perf_counter()
        g = self.device.download(self.linearize(lin).gradient())
        J["require_finite_result"](g, "device gradient")
        if J["gradient_norm_mass"](g, lin.problem.grid.omega) <= GRADIENT_RECHECK * target:
            self.cpu_gradient_checks += 1
            g = J["L"].energy_gradient(lin)
        self._time("gradient", started)
        return g

    def outer_gradient_vectors(self, lin):
        """(gF, gD, gE) host vectors of one joint cell pass (linearization.py:217)."""
        started = perf_counter()
        dl = self.linearize(lin)
        s = dl.state
        out = tuple(self.device.download(v) for v in
                    dl.pair.outer_gradients(s["u"], s["warped"], s["image_grad"], active=s["active"]))
        for v in out:
            _jd()["require_finite_result"](v, "device outer gradient")
        self._time("outer_gradient_vectors", started)
        return out

    def outer_norms(self, lin, omega):
        norm = _jd()["gradient_norm_mass"]
        return tuple(norm(g, omega) for g in self.outer_gradient_vectors(lin))

    def _checked_diagonal(self, t):
        if not bool(torch.isfinite(t).all()) or not bool((t > 0).all()):
            raise FloatingPointError("invalid device GGN diagonal")
        return self.device.download(t)

    def diagonal(self, lin):
        """Device GGN diagonal (free vector) of the state's frozen barrier GGN (linearization.py:357)."""
        t = self.linearize(lin).diagonal()
        if not bool(torch.isfinite(t).all()) or not bool((t > 0).all()):
            raise FloatingPointError("invalid device GGN diagonal")
        return t

    def diagonal_launch(self, lin):
        return _Pending(self, self.linearize(lin).diagonal())

    def node_min_jd(self, lin, *, extension_activation=None, stats=None, compiled=False):
        """Node JD measure (host, full grid shape), with the T69/T73 face/interior extension when asked
        (solvers/jd_affine.py:205)."""
        started = perf_counter()
        dl = self.linearize(lin)
        out = self.device.download(dl.pair.node_min_jd(dl.state["u"], extension_activation, stats))
        self._time("node_min_jd", started)
        return out

    def global_jd_root(self, lin, direction, limit):
        """(first closed27 root in units of limit or inf, invalid base points, points evaluated)."""
        dl = self.linearize(lin)
        root, invalid = dl.pair.jd_root(dl.state["u"], self.device.upload(direction), float(limit))
        points = 27 * lin.problem.grid.n_cells
        return (np.inf if root is None else root / float(limit)), invalid, points

    def poisson(self, inverse):
        return _Poisson(self, inverse)

    # ------------------------------------------------------------------ comparisons (accelerated.py:3062-3124)
    def _differences(self, problem, base, trial):
        pair = self._bind(problem)
        b, t = self._device_state(problem, base), self._device_state(problem, trial)
        return pair.energy_difference(b["u"], b["warped"], t["u"], t["warped"], b["active"], t["active"])

    def _compare(self, problem, base, trial, *, outer_only, joint, required):
        J = _jd()
        for state in (base, trial):
            J["R"].validate_state(problem, state)
        dE, dF = self._differences(problem, base, trial)

        def reduction(difference, is_outer):
            energy = max(s.energy.outer if is_outer else s.energy.total for s in (base, trial))
            return J["EC"].EnergyReduction(float(-difference), float(16 * EPS * energy))

        out = ((reduction(dE, False), reduction(dF, True)) if joint else
               (reduction(dF if outer_only else dE, outer_only),))
        critical = any(not np.isfinite(r.actual) or abs(r.actual) <= CRITICAL_RESOLUTIONS * r.resolution or
                       abs(r.certified - required) <= CRITICAL_RESOLUTIONS * r.resolution for r in out)
        if critical:
            # the decision is within a few resolutions of its threshold: the reference's CPU comparison decides
            self.comparison_counts["cpu"] += 1
            out = (J["EC3"].stable_energy_reductions(problem, base, trial) if joint else
                   (J["EC3"].stable_energy_reduction(problem, base, trial, outer_only=outer_only),))
            path = "cpu"
        else:
            self.comparison_counts["gpu"] += 1
            path = "gpu"
        self.last_comparison = dict(path=path, reason="critical_margin" if critical else "resolved",
                                    required_reduction=required, guard=[r.resolution for r in out])
        return out if joint else out[0]

    def stable_energy_reduction(self, problem, base, trial, *, outer_only=False, required_reduction=0.):
        started = perf_counter()
        if not isinstance(outer_only, bool):
            raise _jd()["InputValidationError"]("outer_only must be boolean")
        r = self._compare(problem, base, trial, outer_only=outer_only, joint=False,
                          required=float(required_reduction))
        self._time("stable_energy_reduction", started)
        return r

    def stable_energy_reductions(self, problem, base, trial, *, required_reduction=0.):
        started = perf_counter()
        r = self._compare(problem, base, trial, outer_only=False, joint=True, required=float(required_reduction))
        self._time("stable_energy_reductions", started)
        return r
