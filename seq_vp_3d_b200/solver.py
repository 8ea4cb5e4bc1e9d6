"""Device-resident certified proximal registration loop on one B200.

Mirrors the reference's default native route:
  jd_curl/three_d/sequential.py:165 _solve_sequential (SequentialReuseConfig3D: forcing eta0 sqrt(min(GF, G0)/G0),
      threshold 1e-8 + 1e-6 G0, joint E/F stable commit, self-reference refresh)
  jd_curl/three_d/solvers/poisson_gradient.py:1090 solve_poisson_gradient (ConservativePGConfig3D: metric
      P^-1 = S~ M^-1 S~ with the image shift, GGN equilibration and JD-affine damping; BB2 steps clipped to
      [1e-8, 10]; 0.9 x the domain bound; witness-cell cubic JD prediction; stable Armijo c1 = 1e-4 with halving
      backtracking (<= 25); the resolution exit)
State (u, warped image, image gradient, gradients, directions) stays on the device; the host sees scalars only,
plus the few witness cells of the JD predictor.  Every accepted state is certified by the GPU certificate, which
is bit-identical to the reference CPU certifier.
"""
from collections import OrderedDict, namedtuple
from dataclasses import dataclass, field
from itertools import product
from time import perf_counter

import numpy as np
import torch

from . import certificate as cert_mod
from .device import to_device
from .pair import DevicePair, Scalars, dot

EPS = float(np.finfo(float).eps)
InvalidTrial = namedtuple("InvalidTrial", "reason detail count")
FAST_COSINE_SCREEN = 1e-6
# the mixed form's float32 energy screen: runtime float64 checks (the first SCREEN_CHECKS screened evaluations and
# every SCREEN_RECHECK-th) and the decision margin in bands
SCREEN_CHECKS = 3
SCREEN_RECHECK = 50
SCREEN_MARGIN = 2.
JD_AFFINE_FLOOR = 1e-12
T62_POLICY = "image_shift_ggn_equilibrated_jd_affine_v1"
T69_POLICY = "image_shift_ggn_equilibrated_jd_affine_v2"   # T62 + face/interior extension once a certificate was uncertain
T73_POLICY = "image_shift_ggn_equilibrated_jd_affine_v3"   # T62 + face/interior extension always (the native default)
METRIC_POLICIES = (T62_POLICY, T69_POLICY, T73_POLICY)


@dataclass(frozen=True)
class PGConfig3D:
    """ConservativePGConfig3D fields of the default route (solvers/poisson_gradient.py:24-236)."""
    max_iterations: int = 5
    initial_step: float = 1.
    step_min: float = 1e-8
    step_max: float = 10.
    max_backtracks: int = 25
    c1: float = 1e-4
    step_tol: float = 1e-12
    stall_steps: int = 5
    jd_step_safety: float = .9
    metric_policy: str = T73_POLICY
    shift_factor: float = 1.
    jd_affine_activation: float = .25
    resolution_exit: bool = True

    def __post_init__(self):
        if self.metric_policy not in METRIC_POLICIES:
            raise ValueError(f"metric_policy: one of {METRIC_POLICIES}")


@dataclass(frozen=True)
class SequentialConfig3D:
    """SequentialReuseConfig3D (sequential.py:29-63)."""
    max_iterations: int = 3
    eta0: float = .01
    step_tol: float = 1e-12
    stall_steps: int = 5


@dataclass
class State:
    theta: torch.Tensor
    u: torch.Tensor
    warped: torch.Tensor
    energy: np.ndarray                 # image, proximity, jd, curl, barrier
    certificate: object
    eval_id: int
    image_grad: torch.Tensor = None    # set by promotion
    norms: tuple = None                # (GF, GD, GE) when computed with the final gradient
    differences: tuple = None          # ((base eval_id, reference version), (dE, dF)) from the one-pass trial
    active: object = None              # per-cell barrier activity mask (from the state's own trial evaluation)
    band: float = 0.                   # error estimate of the screened (float32) dE in `differences`; 0: float64

    @property
    def total(self):
        return float(((((self.energy[0] + self.energy[1]) + self.energy[2]) + self.energy[3]) + self.energy[4]))

    @property
    def outer(self):
        return float(self.energy[0] + self.energy[4])


@dataclass
class InnerResult:
    state: State
    status: str
    reason: str
    gradient_norm: float
    target: float
    accepted_steps: int
    history: list


@dataclass
class SequentialResult:
    status: str
    reason: str
    initial_state: State
    final_state: State
    history: list
    GF_initial: float
    GF_final: float
    GF_threshold: float
    native_mse: float
    final_mse: float
    counts: dict
    elapsed_seconds: float
    timings: dict = field(default_factory=dict)

    @property
    def certified(self):
        return self.final_state is not None and self.final_state.certificate.status == "certified_feasible"


class Registration:
    """One frozen registration problem on the device (problem.py:333 make_problem): grid, images, weights, the
    localized closed27 barrier (activation 0.05), the certificate configuration and the proximal reference."""

    def __init__(self, grid, fixed, moving, *, lam, mu, nu, kappa, activation=.05, u_ref=None,
                 certificate_config=None, precision="plain"):
        self.grid = grid
        self.config = cert_mod.NATIVE_CERTIFICATE if certificate_config is None else certificate_config
        self.delta = self.config.delta
        self.weights = dict(lam=lam, mu=mu, nu=nu, kappa=kappa)
        self.activation = activation
        u_ref = torch.zeros(grid.shape + (3,), dtype=torch.float64, device="cuda") if u_ref is None else u_ref
        self.pair = DevicePair(grid, fixed, moving, u_ref, lam=lam, mu=mu, nu=nu, kappa=kappa,
                               activation=activation, delta=self.delta, precision=precision)
        # the mixed form proves J > delta in the directed-rounding arithmetic (enclosures at least as tight)
        self.certifier = cert_mod.certifier(grid, self.config, directed=precision == "mixed")
        # the mixed form's float32 energy screen of line-search trials (backends/accelerated.py:66-77 screens the
        # same way): decisions within SCREEN_MARGIN bands of a threshold are taken on float64 differences, and the
        # first SCREEN_CHECKS screened evaluations and every SCREEN_RECHECK-th are also evaluated in float64; one
        # difference outside its band switches the screen off for this registration
        self.screen = dict(on=precision == "mixed", evaluations=0, checks=0, band_hits=0, violations=0,
                           max_error_over_band=0.)
        self.q_sum = grid.node_weight_total()
        self.length = float(np.linalg.norm([a[-1] - a[0] for a in grid.axes]))
        self._eval = 0
        self._reference_version = 0
        self.scalars = Scalars(16)
        ref = self.certify(to_device(u_ref))
        if ref.status != "certified_feasible":
            raise ValueError(f"u_ref: not certified feasible ({ref.reason})")
        self.reference_certificate = ref

    # ------------------------------------------------------------------ evaluation (residuals.py:209, :238)
    def certify(self, u):
        rec = self.certifier.run(u)
        return cert_mod.result_from_record(rec, self.grid, self.config, None)

    def evaluate_trial(self, theta, observer=None, base=None, u=None):
        """Certify, warp and evaluate theta (u: its injected field, when the caller has it).  With the line search's
        base, the trial is warped (with its image gradient, so promotion is free) and evaluated against the base in
        one pass, and the stable base -> trial differences are kept for stable_reductions (bitwise the separate
        passes' values)."""
        u = self.pair.inject(theta) if u is None else u
        c = self.certify(u)
        if observer is not None:
            observer(c)
        if c.status != "certified_feasible":
            reason = ("NONFINITE_STATE" if c.reason == "NONFINITE_STATE" else
                      "FEASIBILITY_UNCERTAIN" if c.status == "uncertain" else c.reason)
            return InvalidTrial(reason, "trial not certified: " + c.reason, c.n_uncertain + c.n_infeasible)
        grad = diff = active = None
        if base is None:
            warped, _ = self.pair.warp(u)
            terms, bad = self.pair.energy(u, warped)
        elif self.screen["on"]:
            warped, grad, terms, bad, diff, active, band = self.pair.trial_energy_screened(base.u, base.warped, u,
                                                                                           base_active=base.active)
        else:
            warped, grad, terms, bad, diff, active = self.pair.trial_energy(base.u, base.warped, u,
                                                                            base_active=base.active)
        if bad or not np.all(np.isfinite(terms)):
            return InvalidTrial("NONFINITE_STATE", "floating barrier-point evaluation contradicts feasible certificate", 1)
        self._eval += 1
        state = State(theta, u, warped, terms, c, self._eval, image_grad=grad, active=active)
        if diff is not None:
            state.differences = ((base.eval_id, self._reference_version), diff)
            if base is not None and self.screen["on"]:
                state.band = band
                self._screen_check(base, state)
        return state

    def _verify(self, base, trial, dE, band):
        """The screen's runtime check, on the first SCREEN_CHECKS screened evaluations and every SCREEN_RECHECK-th:
        the float64 (dE, dF) of the two states, or None when no check is due.  A screened dE outside its band ends
        screening for this registration."""
        sc = self.screen
        sc["evaluations"] += 1
        k = sc["evaluations"]
        if not (k <= SCREEN_CHECKS or k % SCREEN_RECHECK == 0):
            return None
        sc["checks"] += 1
        exact = self.pair.energy_difference(base.u, base.warped, trial.u, trial.warped, base.active, trial.active)
        err = abs(dE - exact[0])
        if band > 0:
            sc["max_error_over_band"] = max(sc["max_error_over_band"], err / band)
        if err > band:
            sc["violations"] += 1
            sc["on"] = False
        return exact

    def _screen_check(self, base, trial):
        """The runtime check of a screened trial evaluation: a checked trial keeps the float64 differences."""
        exact = self._verify(base, trial, trial.differences[1][0], trial.band)
        if exact is not None:
            trial.differences = (trial.differences[0], exact)
            trial.band = 0.

    def promote_trial(self, state):
        if state.image_grad is None:
            _, state.image_grad = self.pair.warp(state.u, with_gradient=True)
        return state

    def prepare_base(self, theta):
        s = self.evaluate_trial(theta)
        return s if isinstance(s, InvalidTrial) else self.promote_trial(s)

    def set_reference(self, state):
        """Self-reference refresh (problem.py:397 make_self_reference; sequential.py:347): u_ref = u of a certified
        state; that state's proximity/JD/curl penalties become exactly zero."""
        self.pair.set_reference(state.u)
        self._reference_version += 1
        self.reference_certificate = state.certificate
        e = state.energy.copy()
        e[1:4] = 0.
        state.energy = e
        state.norms = None if state.norms is None else (state.norms[0], state.norms[1], state.norms[0])
        return state

    # ------------------------------------------------------------------ derivatives
    def gnorm(self, g):
        return self.norm_of(dot(g, g))

    def norm_of(self, gg):
        """The norm sqrt(max(g.g, 0)) / sqrt(omega) from the dot product."""
        return float(np.sqrt(max(float(gg), 0.)) / np.sqrt(self.grid.omega))

    def outer_norms(self, state):
        if state.norms is None:
            gF, gD, gE = self.pair.outer_gradients(state.u, state.warped, state.image_grad, state.active)
            state.norms = (self.gnorm(gF), self.gnorm(gD), self.gnorm(gE))
        return state.norms

    def stable_reductions(self, base, trial, required=None):
        """(E, F) EnergyReduction pairs (actual, resolution) (energy_comparison.py:135).  A screened (float32) E
        difference -- the trial's own from its evaluation against this base, or, for any other pair of states in the
        mixed form (the outer commit's start and candidate), svp_energy_difference_screened -- is replaced by the
        float64 one when the decision it feeds (certified = actual - resolution against 0 and `required`, |actual|
        against the resolution) lies within SCREEN_MARGIN bands; F is float64 in both."""
        cached = trial.differences
        use_cache = cached is not None and cached[0] == (base.eval_id, self._reference_version)
        band = 0.
        if use_cache:
            (dE, dF), band = cached[1], trial.band
        elif self.screen["on"]:
            dE, dF, band = self.pair.energy_difference_screened(base.u, base.warped, trial.u, trial.warped,
                                                                base.active)
            exact = self._verify(base, trial, dE, band)
            if exact is not None:
                (dE, dF), band = exact, 0.
        else:
            dE, dF = self.pair.energy_difference(base.u, base.warped, trial.u, trial.warped, base.active,
                                                 trial.active)
        rE = 16 * EPS * max(base.total, trial.total)
        rF = 16 * EPS * max(base.outer, trial.outer)
        if band > 0:
            actual, margin = -dE, SCREEN_MARGIN * band
            edges = (rE, -rE) + ((required + rE,) if required is not None else ())
            if not np.isfinite(actual) or min(abs(actual - e) for e in edges) <= margin:
                self.screen["band_hits"] += 1
                dE, dF = self.pair.energy_difference(base.u, base.warped, trial.u, trial.warped, base.active,
                                                     trial.active)
                if use_cache:
                    trial.differences = (cached[0], (dE, dF))
                    trial.band = 0.
        return (-dE, rE), (-dF, rF)

    def step_ratio(self, candidate, theta):
        """(max|candidate - theta| / max(length, max|theta|), whether the two vectors are equal): the maximum is
        zero exactly when every entry is equal (finite vectors; -0 equals +0, as torch.equal has it)."""
        from . import _lib
        import ctypes
        from .device import ptr, stream_ptr
        out = (ctypes.c_double * 2)()
        _lib.call("svp_max_abs_diff", ptr(candidate), ptr(theta), candidate.numel(), out, stream_ptr())
        return float(out[0] / max(self.length, out[1])), out[0] == 0.

    def metric(self, base, config, memory=None):
        """(a, b, S~) of the T62 conservative metric (solvers/poisson_gradient.py:400 _pg_metric_inverse)."""
        import ctypes
        from . import _lib
        from .device import ptr, stream_ptr
        lam, mu, nu = self.weights["lam"], self.weights["mu"], self.weights["nu"]
        alpha = ctypes.c_double()
        _lib.call("svp_image_shift", self.pair._h, ptr(base.image_grad), float(config.shift_factor),
                  ctypes.byref(alpha), stream_ptr())
        a, b = lam + alpha.value, mu / 2 + nu / 2
        inv_h2 = sum(1 / h ** 2 for h in self.grid.spacing)
        m = self.grid.omega * (a + b * (8 / 9) * inv_h2)
        d = self.pair.ggn_diagonal(base.u, base.image_grad, base.active)
        # solvers/poisson_gradient.py:486: T73 always, T69 once this level has seen an undetermined certificate
        extend = config.metric_policy == T73_POLICY or (
            config.metric_policy == T69_POLICY and memory is not None and memory.uncertain > 0)
        node = self.pair.node_min_jd(base.u, config.jd_affine_activation if extend else None)
        scale = self.pair.free()
        bad = ctypes.c_int64()
        _lib.call("svp_pg_scale", self.pair._h, ptr(d), ptr(node), float(m), float(config.jd_affine_activation),
                  JD_AFFINE_FLOOR, ptr(scale), ctypes.byref(bad), stream_ptr())
        if bad.value:
            raise FloatingPointError("T62 scale must be finite and positive")
        return a, b, scale


# ------------------------------------------------------------------------------------------ JD step prediction
def _cofactor(F):
    out = np.empty(F.shape)
    for r, j, k in ((0, 1, 2), (1, 2, 0), (2, 0, 1)):
        for c, l, m in ((0, 1, 2), (1, 2, 0), (2, 0, 1)):
            out[..., r, c] = F[..., j, l] * F[..., k, m] - F[..., j, m] * F[..., k, l]
    return out


def first_root_before(c, limit):
    """solvers/jd_step.py:19: floating first root of c0 + c1 t + c2 t^2 + c3 t^3 on (0, limit], or None."""
    c = np.asarray(c, dtype=float)
    with np.errstate(over="ignore", invalid="ignore"):
        c = c * np.array([1., limit, limit ** 2, limit ** 3])
    if not np.all(np.isfinite(c)) or c[0] <= 0:
        raise FloatingPointError("invalid cubic predictor base/coefficients")
    if c[0] > np.abs(c[1:]).sum():
        return None
    poly = np.trim_zeros(c[::-1], trim="f")
    if len(poly) == 1:
        return None
    try:
        roots = np.roots(poly / np.max(np.abs(poly)))
    except np.linalg.LinAlgError as error:
        raise FloatingPointError("cubic root failure") from error
    cand = [float(r.real) for r in roots if 0 < r.real <= 1 and abs(r.imag) <= 1e-8 * max(1., abs(r.real))]
    return None if not cand else min(cand) * limit


class JDStepMemory:
    """Bounded recent witnesses of failed certificates (solvers/jd_step.py:88): the first root of
    det(A + tau V) - delta at each witness cell's closed27 and witness points caps the next trial step."""
    CLOSED27 = [(x, y, z) for z, y, x in product((0., .5, 1.), repeat=3)]
    VERTICES = [(x, y, z) for z, y, x in product((0, 1), repeat=3)]

    def __init__(self, grid):
        self.grid = grid
        self.points = OrderedDict()
        self.uncertain = 0

    def certificate(self, c):
        if c.status == "uncertain":
            self.uncertain += 1
        if c.status == "infeasible" and c.witness_cell is not None and c.witness_reference_point is not None:
            key = (int(c.witness_cell), tuple(float(x) for x in c.witness_reference_point))
            self.points[key] = None
            self.points.move_to_end(key)
            if len(self.points) > 128:
                self.points.popitem(last=False)

    def predict(self, base_u, direction, limit, safety, delta):
        if not self.points:
            return limit
        grid = self.grid
        nz, ny, nx = grid.shape
        cz, cy, cx = grid.cell_shape
        cells = sorted({c for c, _ in self.points})
        # gather the witness cells' vertex data (8 nodes each) from the device
        node_ids = []
        for c in cells:
            z0, y0, x0 = c // (cx * cy), (c // cx) % cy, c % cx
            node_ids.append([((z0 + vz) * ny + y0 + vy) * nx + x0 + vx for vx, vy, vz in self.VERTICES])
        node_ids = np.array(node_ids)
        idx = torch.as_tensor(node_ids.ravel(), device=base_u.device)
        U = base_u.reshape(-1, 3)[idx].cpu().numpy().reshape(len(cells), 8, 3)
        fz, fy, fx = nz - 2, ny - 2, nx - 2
        z, y, x = np.unravel_index(node_ids, grid.shape)
        free = (z > 0) & (z < nz - 1) & (y > 0) & (y < ny - 1) & (x > 0) & (x < nx - 1)
        # free-vector index of each vertex; boundary vertices are clipped into range and masked to zero below
        flat = ((np.clip(z - 1, 0, fz - 1) * fy + np.clip(y - 1, 0, fy - 1)) * fx + np.clip(x - 1, 0, fx - 1))
        nf = fz * fy * fx
        pid = torch.as_tensor(np.stack([flat + r * nf for r in range(3)], -1).ravel(), device=direction.device)
        Pv = direction[pid].cpu().numpy().reshape(len(cells), 8, 3) * free[..., None]
        minimum = None
        try:
            for k, c in enumerate(cells):
                pts = list(self.CLOSED27) + [p for cc, p in self.points if cc == c and p not in self.CLOSED27]
                pts = np.asarray(pts)
                D = np.empty((3, len(pts), 8))
                for a, vertex in enumerate(self.VERTICES):
                    fac = [pts[:, j] if vertex[j] else 1 - pts[:, j] for j in range(3)]
                    for j in range(3):
                        o = [m for m in range(3) if m != j]
                        D[j, :, a] = (1 if vertex[j] else -1) / grid.spacing[j] * fac[o[0]] * fac[o[1]]
                A = np.einsum("jqa,ar->qrj", D, U[k]) + np.eye(3)
                V = np.einsum("jqa,ar->qrj", D, Pv[k])
                C = np.stack((np.linalg.det(A) - delta, np.sum(_cofactor(A) * V, axis=(-2, -1)),
                              np.sum(A * _cofactor(V), axis=(-2, -1)), np.linalg.det(V)), axis=-1)
                for row in C:
                    r = first_root_before(row, limit)
                    if r is not None:
                        minimum = r if minimum is None else min(r, minimum)
        except (FloatingPointError, OverflowError):
            return limit
        return limit if minimum is None else min(limit, safety * minimum)


# ------------------------------------------------------------------------------------------ inner PG solve
def _protect(config, value):
    return min(config.step_max, max(config.step_min, value))


def _bb2(reg, config, theta, g, p, previous):
    """(proposal, rule) of solvers/poisson_gradient.py:785 _step_proposal_fast."""
    import ctypes
    from . import _lib
    from .device import ptr, stream_ptr
    if previous is None:
        return _protect(config, config.initial_step), "initial"
    th0, g0, p0, tau0 = previous
    out = (ctypes.c_double * 4)()
    _lib.call("svp_bb2_dots", ptr(theta), ptr(th0), ptr(g), ptr(g0), ptr(p0), ptr(p), theta.numel(), out,
              stream_ptr())
    return _bb2_rule(config, previous, out[:])


def _bb2_rule(config, previous, dots):
    """The BB2 rule set on the secant products (s.y, s.s, y.y, y.iy) of svp_bb2_dots."""
    if previous is None:
        return _protect(config, config.initial_step), "initial"
    tau0 = previous[3]
    fallback = _protect(config, 2 * min(tau0, config.step_max / 2))
    sy, ss, yy2, yiy = (float(v) for v in dots)
    if not all(np.isfinite([sy, ss, yy2, yiy])):
        return fallback, "fallback_nonfinite_secant"
    if sy <= 0:
        return fallback, "fallback_nonpositive_curvature"
    ns, ny = np.sqrt(ss), np.sqrt(yy2)
    screened = ns > 0 and ny > 0 and ns * ny >= 2. ** -900 and sy / (ns * ny) > FAST_COSINE_SCREEN
    if not screened and sy / (ns * ny) <= 1e-12:
        return fallback, "fallback_small_curvature"
    if yiy <= 0:
        return fallback, "fallback_nonpositive_metric_curvature"
    proposal = sy / yiy
    if not np.isfinite(proposal) or proposal <= 0:
        return fallback, "fallback_nonpositive_step"
    return _protect(config, proposal), "bb2"


def _failed_status(attempts):
    reasons = {a["reason"] for a in attempts}
    if reasons == {"INVALID_DOMAIN"}:
        return "domain_blocked"
    if reasons == {"FEASIBILITY_UNCERTAIN"}:
        return "feasibility_uncertain"
    if reasons == {"JACOBIAN_VIOLATION"}:
        return "feasibility_blocked"
    if reasons and all(r.startswith("NONFINITE") for r in reasons):
        return "nonfinite_evaluation"
    return "line_search_failed"


def _precision_evidence(attempts, untruncated):
    if not attempts or not untruncated:
        return False
    for a in attempts:
        if a["reason"] != "ENERGY_RESOLUTION" or not a["valid"] or a["accepted"] or a["resolution"] is None:
            return False
    return all(np.isfinite(a["actual"]) and a["resolution"] >= 0 and abs(a["actual"]) <= a["resolution"]
               for a in attempts)


def solve_pg(reg, base, *, target, config, memory, timings=None):
    """One frozen-reference subproblem (solvers/poisson_gradient.py:1090)."""
    history, accepted_steps, small_steps = [], 0, 0
    previous, metric = None, None
    pending = None          # the next step's gradient, launched as soon as its state was accepted
    G = None

    def finish(status, reason):
        return InnerResult(base, status, reason, G, target, accepted_steps, history)

    S = reg.scalars
    while True:
        final = accepted_steps >= config.max_iterations
        if final:
            # the last gradient of the solve: the joint outer triple (same gE), reused by the outer norms
            gF, gD, g = reg.pair.outer_gradients(base.u, base.warped, base.image_grad, base.active)
            S.dot(0, g, g)
            S.dot(1, gF, gF)
            S.dot(2, gD, gD)
            v = S.fetch()
            G = reg.norm_of(v[0])
            base.norms = (reg.norm_of(v[1]), reg.norm_of(v[2]), G)
            if G <= target:
                return finish("converged_gradient", "GRADIENT_TARGET")
            if small_steps >= config.stall_steps:
                return finish("stagnated", "SMALL_ACCEPTED_STEPS")
            return finish("max_iterations", "ACCEPTED_STEP_BUDGET")
        # One batch of device work and one synchronisation per step: the gradient and its norm, (the metric on the
        # first step,) the direction, the slope, the BB2 secant products and the domain bound.  The decisions below
        # are taken in the reference's order on the same values.
        g = pending if pending is not None else reg.pair.gradient(base.u, base.warped, base.image_grad,
                                                                  active=base.active)
        pending = None
        metric_error = None
        if metric is None:
            try:
                metric = reg.metric(base, config, memory)
            except FloatingPointError as exc:
                metric_error = exc
        if metric_error is None:
            a, b, scale = metric
            p = reg.pair.poisson_apply(a, b, g, scale=scale, sign=-1.)
            # |g|^2, the slope g.p and the BB2 products in one pass
            S.step_dots(0, g, p, None if previous is None else (base.theta, previous[0], previous[1], previous[2]))
            S.step_bound(6, reg.pair, base.u, p)
        else:
            S.dot(0, g, g)
        v = S.fetch()
        G = reg.norm_of(v[0])
        if G <= target:
            return finish("converged_gradient", "GRADIENT_TARGET")
        if small_steps >= config.stall_steps:
            return finish("stagnated", "SMALL_ACCEPTED_STEPS")
        if metric_error is not None:
            return finish("nonfinite_evaluation", str(metric_error))
        slope = float(v[1])
        if not np.isfinite(slope):
            return finish("nonfinite_evaluation", "PG directional derivative")
        if slope >= 0:
            return finish("non_descent_direction", "NON_DESCENT_DIRECTION")
        proposal, rule = _bb2_rule(config, previous, v[2:6])
        bound = float(v[6])
        if bound <= 0:
            return finish("domain_blocked", "NO_POSITIVE_DOMAIN_STEP")
        tau = min(proposal, .9 * bound)
        tau = memory.predict(base.u, p, tau, config.jd_step_safety, reg.delta)
        untruncated = tau == proposal
        attempts = []
        exit_floor = 15 * EPS * base.total if config.resolution_exit else None
        global_attempts = 0
        accepted = False
        for attempt in range(config.max_backtracks + 1):
            required = -config.c1 * tau * slope
            # candidate, its field and the step ratio's maxima in one pass; the maxima's copy completes under the
            # trial's own synchronisations
            candidate, u_trial = reg.pair.trial_point(base.theta, tau, p, S.slot(7))
            S.copy_async()
            trial = reg.evaluate_trial(candidate, observer=memory.certificate, base=base, u=u_trial)
            valid = not isinstance(trial, InvalidTrial)
            actual = resolution = None
            if valid:
                v = S.values()
                relative = float(v[7] / max(reg.length, v[8]))
                (actual, resolution), _ = reg.stable_reductions(base, trial, required)
                certified = actual - resolution
                accepted = certified > 0 and certified >= required
                reason = ("ACCEPTED" if accepted else "ENERGY_RESOLUTION" if abs(actual) <= resolution
                          else "NO_STRICT_DECREASE" if actual < 0 else "ARMIJO_REJECTED")
            else:
                reason = trial.reason
            if accepted:
                reg.promote_trial(trial)
                if accepted_steps + 1 < config.max_iterations:
                    # the next iteration is not the final one, so it starts from this state's gradient: launch it
                    # now, the bookkeeping below runs while the GPU computes it
                    pending = reg.pair.gradient(trial.u, trial.warped, trial.image_grad, active=trial.active)
            exit_stop = False
            if (config.resolution_exit and not accepted and not reason.startswith("NONFINITE")
                    and global_attempts + 1 <= config.max_backtracks):
                if reason == "JACOBIAN_VIOLATION":
                    next_tau = min(.5 * tau, memory.predict(base.u, p, tau, config.jd_step_safety, reg.delta))
                else:
                    next_tau = .5 * tau
                exit_stop = next_tau * abs(slope) <= exit_floor
            row = dict(iteration=accepted_steps, attempt=attempt + 1, accepted=bool(accepted), reason=reason,
                       valid=valid, tau=tau, proposal=proposal, rule=rule, bound=bound, actual=actual,
                       resolution=resolution, energy_base=base.total,
                       energy_trial=trial.total if valid else None, gradient_norm=G, slope=slope)
            history.append(row)
            attempts.append(row)
            if reason.startswith("NONFINITE"):
                return finish("nonfinite_evaluation", reason)
            if accepted:
                small_steps = small_steps + 1 if relative <= config.step_tol else 0
                previous = (base.theta, g, p, tau)
                base = trial
                accepted_steps += 1
                break
            global_attempts += 1
            if global_attempts > config.max_backtracks:
                break
            if exit_stop:
                break
            if reason == "JACOBIAN_VIOLATION":
                tau = min(.5 * tau, memory.predict(base.u, p, tau, config.jd_step_safety, reg.delta))
            else:
                tau *= .5
        if not accepted:
            evidence = _precision_evidence(attempts, untruncated)
            return finish("precision_stagnated" if evidence else _failed_status(attempts), attempts[-1]["reason"])


# ------------------------------------------------------------------------------------------ outer loop
def solve_sequential(reg, theta0=None, *, config=None, inner_config=None, budget=None):
    """Certified proximal outer iteration (sequential.py:165) from theta0 (default: zero displacement)."""
    config = SequentialConfig3D() if config is None else config
    inner_config = PGConfig3D() if inner_config is None else inner_config
    started = perf_counter()
    theta0 = torch.zeros(3 * reg.grid.n_free_scalar, dtype=torch.float64, device="cuda") if theta0 is None else theta0
    memory = JDStepMemory(reg.grid)
    counts = dict(outer_accepted=0, inner_calls=0, trials=0, reference_refreshes=0)
    history = []

    def mse(state):
        return float(2 * state.energy[0] / reg.q_sum)

    raw = reg.prepare_base(theta0)
    if isinstance(raw, InvalidTrial):
        return SequentialResult("invalid_initial_state", raw.reason, None, None, history, None, None, None, None,
                                None, counts, perf_counter() - started)
    current = raw
    if not (current.energy[1] == 0. and current.energy[2] == 0. and current.energy[3] == 0.):
        current = reg.set_reference(current)            # initial self reference
        counts["reference_refreshes"] += 1
    initial = current
    native = mse(current)
    GF, GD, GE = reg.outer_norms(current)
    G0 = GF
    threshold = 1e-8 + 1e-6 * G0
    small_steps = 0

    def done(status, reason):
        counts["screen"] = dict(reg.screen)
        return SequentialResult(status, reason, initial, current, history, G0, GF, threshold, native, mse(current),
                                counts, perf_counter() - started)

    while True:
        if budget is not None and budget():
            return done("outer_time_budget", "WALL_BUDGET; last formal state only, not convergence")
        if GF <= threshold:
            return done("converged_regularized_gradient", "Feasible F=D+B gradient criterion, not global optimality")
        if small_steps >= config.stall_steps:
            return done("outer_stagnated", "Small accepted steps with nonzero outer gradient")
        if counts["outer_accepted"] >= config.max_iterations:
            return done("outer_max_iterations", "Outer budget exhausted; not convergence")
        start = current
        eta = config.eta0 if G0 == 0 else config.eta0 * np.sqrt(min(GF, G0) / G0)
        target = float(eta * GF)
        counts["inner_calls"] += 1
        inner = solve_pg(reg, start, target=target, config=inner_config, memory=memory)
        counts["trials"] += len(inner.history)
        candidate = inner.state
        accepted, reason = False, "INNER_FAILED_NOT_COMMITTED"
        GFa = GDa = GEa = None
        total = fixed = None
        if True:
            GFa, GDa, GEa = reg.outer_norms(candidate)
            relative, same = reg.step_ratio(candidate.theta, start.theta)
            total, fixed = reg.stable_reductions(start, candidate)
            cert = (total[0] - total[1]) > 0 and (fixed[0] - fixed[1]) > 0
            eligible = inner.status in ("converged_gradient", "max_iterations", "stagnated")
            accepted = bool(eligible and cert and not same)
            reason = ("ACCEPTED" if accepted else "INNER_FAILED_NOT_COMMITTED" if not eligible
                      else "NO_PROGRESS" if same else "DESCENT_CERTIFICATE_FAILED")
        history.append(dict(outer_i=len(history), accepted=accepted, reason=reason, inner_status=inner.status,
                            inner_accepted_steps=inner.accepted_steps, inner_history=inner.history,
                            E_start=start.total, E_candidate=candidate.total, F_start=start.outer,
                            F_candidate=candidate.outer, GF_before=GF, GF_candidate=GFa, forcing_target=target,
                            actual_reduction_E=None if total is None else total[0],
                            actual_reduction_F=None if fixed is None else fixed[0],
                            elapsed_seconds=perf_counter() - started))
        if accepted:
            counts["outer_accepted"] += 1
            current, GF, GD, GE = candidate, GFa, GDa, GEa
            small_steps = small_steps + 1 if relative <= config.step_tol else 0
        else:
            if inner.status == "precision_stagnated":
                return done("outer_precision_stagnated", reason)
            if inner.status in ("domain_blocked", "feasibility_blocked", "feasibility_uncertain"):
                return done("outer_" + inner.status, inner.reason)
            if inner.status not in ("converged_gradient", "max_iterations", "stagnated"):
                return done("outer_inner_failed", inner.status + ": " + inner.reason)
            return done("outer_no_progress" if reason == "NO_PROGRESS" else "outer_candidate_rejected", reason)
        if GF <= threshold or counts["outer_accepted"] >= config.max_iterations or small_steps >= config.stall_steps:
            continue
        current = reg.set_reference(current)
        counts["reference_refreshes"] += 1
        GE = GF
