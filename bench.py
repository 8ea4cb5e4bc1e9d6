#!/usr/bin/env python
"""Certified registration pairs per hour at 160x192x224 on B200 GPUs: the plain FP64 form and the mixed form.

One step = one complete certified registration of a seeded head-phantom pair (the 160x192x224 synthetic workload):
float32 8/4/2/1 pyramid pre-optimizer, boundary taper, certified transfer, then the certified proximal loop for
--outer outer steps (5 accepted PG steps each), every accepted state proven J > 0 on every closed cell by the GPU
certificate.  `value`: pairs/hour of the primary form (--form) with the images already in HBM, kernel timers off;
`e2e`: the same through the public API with the images in pinned host memory and the certified displacement + warped
image copied back every step; `latency_s`: p50/p95/p99 of the timed pairs.  `forms` holds the other form timed on
--compare-steps pairs and the mixed/plain ratio with the final MSEs reached.  `roofline` comes from a separate pair
run with the per-kernel CUDA-event timers on.

CPU legs (rank 0, N = 1, skipped with --no-cpu): `cpu_baseline`, the reference's own CPU implementation (the jd_curl
package installed under baseline/_ref, Numba on every host core) timed per component on a z-slab of the workload and
extrapolated per pair (the oracle port where the package is absent), and `parity`, the checker: the final certified
field of the last timed pair re-certified by the C restatement of the reference certifier (every record field
bitwise), and the energy terms (full size), DST-I apply (full size), spline coefficients (full size), warped image,
gradient, GGN diagonal and node JD measure (on a z-slab of the full-size state) diffed against the numpy oracle.

Multi-GPU: one process per GPU, independent pairs per rank (replicas only: registrations are independent units and
the path has no exchange step); value = all ranks' pairs / max-over-ranks time.

--impl reference: the reference's CPU implementation of the path on the host cores (rank 0 only), each step a
bounded sample: the per-component table is measured once in the first warm-up step, then every step re-times one
component (in rotation) on a z-slab and reports the pairs/hour the table extrapolates to.
"""
import os
import sys

# the reference arm's libraries use every host core (set before numpy / numba are imported)
if "--impl" in sys.argv[:-1] and sys.argv[sys.argv.index("--impl") + 1] == "reference":
    for _k in ("NUMBA_NUM_THREADS", "OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ.setdefault(_k, str(os.cpu_count() or 1))

import argparse
import json
import subprocess
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "certified pairs/hour @160x192x224 ({} form, 1 B200 per pair)"
SMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
# component calls per outer step of the default route (5 accepted PG steps with one trial each, as the reference's
# own run of the seeded pairs shows, plus the outer comparison, the self-reference refresh and its base): used only
# by the CPU extrapolation
PER_OUTER = dict(evaluate=6, compare=6, promote=6, gradient=5, outer=1, ggn=1, node_jd=1, certify=1, direction=5)


def parse():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--outer", type=int, default=200, help="outer steps per registration (config 2: 200)")
    ap.add_argument("--form", choices=("plain", "mixed"), default="mixed",
                    help="primary form: mixed (float32 direction bulk on CUDA and tensor cores, float64 energies and "
                         "decisions, directed-rounding certificate) or plain (float64 throughout, certificates "
                         "bit-identical to the reference's); the other form is timed beside it (--compare-steps)")
    ap.add_argument("--compare-steps", type=int, default=3,
                    help="pairs of the other form timed for the mixed/plain ratio (0: skip)")
    ap.add_argument("--concurrency", type=int, default=1,
                    help="serving form: registrations in flight at once (each on its own stream); a step is one "
                         "round of that many pairs, value = all pairs / time, with p50/p95/p99 latency")
    ap.add_argument("--preopt", action=argparse.BooleanOptionalAction, default=True,
                    help="config-2 route: float32 8/4/2/1 pyramid pre-optimizer + certified transfer before the "
                         "native steps")
    ap.add_argument("--shape", default="160,192,224", help="nx,ny,nz")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU legs (baseline timing and parity checker)")
    ap.add_argument("--cpu-planes", type=int, default=5, help="node planes of the CPU baseline's z-slab")
    ap.add_argument("--parity-planes", type=int, default=8, help="node planes of the parity checker's z-slab")
    ap.add_argument("--profile", action="store_true", help="per-kernel device times to stderr")
    ap.add_argument("--serve", default=None, metavar="RATES",
                    help="open-loop serving sweep: comma-separated arrival rates in requests/hour (Poisson arrivals); "
                         "requests mix the grids 96^3, 128x144x128, 160x192x160, 160x192x224 with 25%% 48^3, each a "
                         "seeded blob pair with a fixed outer-step budget (--serve-outer)")
    ap.add_argument("--serve-requests", type=int, default=16, help="requests per arrival rate")
    ap.add_argument("--serve-outer", type=int, default=50, help="outer-step budget per served request")
    ap.add_argument("--serve-slots", type=int, default=4, help="registrations in flight at most")
    return ap.parse_args()


class Clocks:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons while the timed region runs."""

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={SMI_FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for name, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return dict(sm_mhz=float(np.median(sm)) if sm else None, sm_max_mhz=mx, reasons=sorted(reasons),
                    samples=len(sm))


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return p["hbm_gbs"], "measured"
    return 6650., "fallback"


# ------------------------------------------------------------------------------------------ algorithmic counts
# FP64 operations per cell of the cell kernels, counted from their source (csrc/q1.cu, csrc/q1_common.cuh):
# one grad-u column = 30 (3 components x (2 bilinear lerps of 3 + final lerp and 1/h of 4)); det = 17; cofactor+det
# = 35; curl = 3; sq_change = 20; compensated add = 8.  Barrier-active points add a few hundred more (not counted).
FLOP_PER_CELL = {
    # edges 108 + reference sweep (45 columns + 27 x (det + curl)) 1890 + Gauss sweep2 (126 columns) 3780
    # + 27 x (2 det + 2 curl + 4 stable changes + trial energy) 4833 + the trial's closed sweep (45 columns) 1350
    # + 27 x det 459 (the base's closed sweep runs only in cells near the activation: not counted)
    "cell_trial_kernel": 12420,
    "cell_diff_kernel": 15006,
    # edges 72 + ref sweep 1890 + Gauss sweep (45 columns) 1350 + 27 x 31 + closed sweep 1350 + 27 x det 459
    "cell_energy_kernel": 5958,
    # edges 72 + soft sweep2 3780 + 27 x 94 (cofactor, det, curls, fluxes) + adjoint scatter 693
    # + barrier sweep 1350 + 27 x det 459
    "cell_grad_kernel": 8892,
    # edges 36 + Gauss sweep 1350 + 27 x (cofactor 35 + 8 vertices x 30) + closed sweep 1350 + 27 x det 459
    # + the state-independent curl term 24
    "cell_ggn_diag_kernel": 10644,
    "cell_min_jd_kernel": 2009,
}
FP64_PEAK_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12     # nominal: 148 SMs x 64 FP64 FMA/clk x 2 x 1965 MHz
# float32 operations per cell of the mixed form's cell kernels (the float64 barrier of the flagged cells runs in its
# own kernels and is not counted here)
FLOP32_PER_CELL = {
    # edges 108 + reference sweep 1890 + Gauss sweep2 3780 + 27 x (2 det + 2 curl + 3 curl residual pairs
    # (squares, stable change, magnitudes) + 8 weighted sums) 2700 + the trial's closed sweep 1350 + 27 x det 459
    # (the base's closed sweep runs only where the base may be active: not counted)
    "cell_trial32_kernel": 10287,
    # edges 72 + soft sweep2 3780 + 27 x 94 (cofactor, det, curls, fluxes) + adjoint scatter 693
    "cell_grad32_kernel": 7083,
    # edges 36 + Gauss sweep 1350 + 27 x (cofactor 35 + 8 vertices x 30) + the curl constants 24
    "cell_ggn_diag32_kernel": 8835,
}
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12    # nominal: 148 SMs x 128 FP32 FMA/clk x 2 x 1965 MHz
# DRAM bytes (read + write) per cell measured by ncu on the 160x192x96 pair (2,885,055 cells; profiles/
# traffic_cell_trial_edge_hull_warp_160x192x96.md); scaled to a launch by the cells it processes (traffic grows with
# the cell count: every launch streams its fields once, plus neighbour re-reads of the same order)
TRAFFIC_PER_CELL = {"cell_trial_kernel": (325667584 + 1371392) / 2885055,
                    # full size, 160x192x224 (6,772,287 cells; profiles/cell_kernels_head_pair_160x192x224.md)
                    "cell_trial32_kernel": (813766656 + 19263232) / 6772287,
                    "edge_hull_kernel": (74312512 + 8776576) / 2885055,
                    "warp_trial_kernel_grad": (312493568 + 74758400) / 2885055}


def kernel_counts(shape):
    """(algorithmic HBM bytes, FP64 FLOP) per launch of the hot kernels: each input field read once, outputs written
    once; FLOP from FLOP_PER_CELL (cell kernels) or the GEMM count (DST-I passes, averaged over the passes)."""
    nx, ny, nz = shape
    nn, nc, nf = nx * ny * nz, (nx - 1) * (ny - 1) * (nz - 1), (nx - 2) * (ny - 2) * (nz - 2)
    f = [nx - 2, ny - 2, nz - 2]
    # one folded DST-I pass along an axis of length n: 2 (ceil(n/2)^2 + floor(n/2)^2) FLOP per line, 3 nf / n lines
    dst = [2 * (((n + 1) // 2) ** 2 + (n // 2) ** 2) * 3 * nf / n for n in f]
    c = lambda name: FLOP_PER_CELL[name] * nc
    return {
        # base u, trial u, u_ref: 24 B/node each
        "cell_trial_kernel": (3 * 24 * nn, c("cell_trial_kernel")),
        # the mixed form's screened trial: the same fields in, float32 sweeps; the barrier flags and the mask out
        "cell_trial32_kernel": (3 * 24 * nn + 2 * nc, None),
        "cell_diff_kernel": (3 * 24 * nn, c("cell_diff_kernel")),
        "cell_energy_kernel": (2 * 24 * nn, c("cell_energy_kernel")),
        # u, u_ref in; 24 doubles per cell out (one locals buffer; two for the outer triple)
        "cell_grad_kernel": (2 * 24 * nn + 192 * nc, c("cell_grad_kernel")),
        "gather_kernel": (192 * nc + nn * (24 + 24 + 8 + 8 + 24) + 3 * 8 * nf, None),
        "cell_ggn_diag_kernel": (24 * nn + 192 * nc, c("cell_ggn_diag_kernel")),
        # mixed form: the same float64 inputs, float32 locals out
        "cell_grad32_kernel": (2 * 24 * nn + 96 * nc, None),
        "cell_ggn_diag32_kernel": (24 * nn + 96 * nc, None),
        "edge_hull_kernel": (24 * nn + 9 * nc, None),
        # trial u, base u, base warped, fixed, u_ref in; warped (+ gradient) out; coefficients cache resident
        "warp_trial_kernel_grad": ((24 + 24 + 8 + 8 + 24 + 8 + 24) * nn, None),
        "warp_trial_kernel": ((24 + 24 + 8 + 8 + 24 + 8) * nn, None),
        "warp_kernel": ((24 + 8) * nn, None),
        "warp_kernel_grad": ((24 + 8 + 24) * nn, None),
        # folded input read once, output written once (+ the scale / denominator arrays where fused)
        "dst_left_kernel": (2 * 3 * 8 * nf, (dst[1] + dst[2]) / 2),
        "dst_right_kernel": (2 * 3 * 8 * nf, dst[0]),
        "node_diff_kernel": (2 * (24 + 8) * nn + 8 * nn + 24 * nn, None),
        "node_energy_kernel": ((24 + 8 + 8 + 24) * nn, None),
        "precheck_kernel": (24 * nn, None),
        "cell_min_jd_kernel": (24 * nn + 8 * nc, c("cell_min_jd_kernel")),
    }


# kernels timed for the profile and the phase split only: their work depends on the state (the certificate stages
# run on the cells the edge hull leaves unproven, the node-measure extension on candidate cells)
STATE_DEPENDENT_KERNELS = ("prescreen_kernel", "fallback_grid_kernel", "classify_kernel", "jd_extension_kernel",
                           "jd_root_kernel", "cell_ggn_hvp_kernel", "cell_trial_barrier_kernel",
                           "cell_grad_barrier32_kernel", "cell_ggn_barrier32_kernel", "cell_grad_barrier_kernel",
                           "cell_ggn_barrier_kernel", "cell_trial_diff_kernel")


class Ranks:
    """One process per GPU (RANK, WORLD_SIZE, LOCAL_RANK from the launcher's environment) and the two collectives the
    bench takes: a barrier around every timed region and the maximum over ranks of its device time.  Registrations
    are independent replicas, so nothing else crosses ranks.  backend "nccl" on the GPUs; the CPU tests run the same
    code over "gloo" with device "cpu"."""

    def __init__(self, backend="nccl", device="cuda", timeout_s=600):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.device = device
        if self.world > 1:
            import torch.distributed as dist
            from datetime import timedelta
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max(self, x):
        """The maximum of x over the ranks (every rank gets it)."""
        if self.world == 1:
            return x
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


def whole_job_rate(pairs_per_rank, seconds, world):
    """Whole-job pairs/hour: every rank registers pairs_per_rank pairs; seconds is the max over ranks."""
    return world * pairs_per_rank / seconds * 3600.


def phase_summary(phase, timers):
    """Host-clock seconds of one pair's pre-optimizer, transfer and certified loop, the device time of the loop's
    timed kernels and the loop's remainder: host control, syncs and launch gaps."""
    if not phase:
        return None
    out = dict(phase)
    loop = sum(ms for name, (_, ms) in timers.items() if not name.startswith(("pre_", "adam"))) / 1e3
    out["loop_kernels_s"] = loop
    out["loop_host_gap_s"] = out["certified_loop_s"] - loop
    return out


# ------------------------------------------------------------------------------------------ CPU legs
def slab_state(ugt, z0, planes):
    """A certified state on a z-slab of the workload: the ground-truth in-plane displacement at half strength, tapered
    to zero on the slab's z faces (x and y faces are already zero)."""
    taper = np.sin(np.pi * np.arange(planes) / (planes - 1))[:, None, None]
    u = np.zeros((planes,) + ugt.shape[1:])
    u[..., 0] = .5 * ugt[z0:z0 + planes, ..., 0] * taper
    u[..., 1] = .5 * ugt[z0:z0 + planes, ..., 1] * taper
    return np.ascontiguousarray(u)


def reference_package():
    """The reference's own package (jd_curl) installed under baseline/_ref, or None.  It needs nibabel only for NIfTI
    I/O, so a stub module stands in for it."""
    import types
    path = os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(path, "jd_curl")):
        return None
    sys.modules.setdefault("nibabel", types.ModuleType("nibabel"))
    if path not in sys.path:
        sys.path.append(path)
    try:
        import jd_curl
        return jd_curl
    except Exception:
        return None


class CpuTable:
    """Per-component seconds of the reference CPU path on a z-slab of the workload, re-timed one component at a time,
    and the pairs/hour they extrapolate to: seconds per pair = outer x (sum_c count_c x t_c x cell planes of the
    volume / cell planes of the slab + the full-size DST-I directions).  Uses the reference's own package (kind
    "reference") or, where it is absent, the oracle port (kind "port")."""

    def __init__(self, shape, fixed, moving, ugt, weights, planes, outer):
        nx, ny, nz = shape
        self.shape, self.outer, self.planes = shape, outer, planes
        z0 = nz // 2 - planes // 2
        self.scale = (nz - 1) / (planes - 1)
        self.u = slab_state(ugt, z0, planes)
        self.fixed, self.moving = fixed[z0:z0 + planes], moving[z0:z0 + planes]
        self.weights = weights
        self.rhs = np.random.default_rng(1).normal(size=3 * (nx - 2) * (ny - 2) * (nz - 2))
        self.ref = reference_package()
        self.kind = "reference" if self.ref is not None else "port"
        self.cores = int(os.environ.get("NUMBA_NUM_THREADS", os.cpu_count() or 1)) if self.ref else 1
        self.t = {}
        self._base = None
        if self.ref is not None:
            from jd_curl.three_d.grid import make_grid_3d
            from jd_curl.three_d.problem import Weights3D, make_problem
            from jd_curl.three_d.feasibility import PrescreenCertificateConfig
            from jd_curl.three_d.boundary import restrict_free
            g = make_grid_3d(nx=nx, ny=ny, nz=planes, hx=1., hy=1., hz=1., unit="mm")
            self.cfg = PrescreenCertificateConfig(delta=0., max_depth=48, max_boxes=255, tile_size=65536,
                                                  fallback_workers=max(1, os.cpu_count() or 1))
            self.P = make_problem(grid=g, fixed_image=self.fixed, moving_image=self.moving,
                                  u_ref=np.zeros(g.shape + (3,)), weights=Weights3D(**weights),
                                  certificate_config=self.cfg, barrier_location="closed27_uniform",
                                  barrier_activation=.05)
            self.theta = restrict_free(self.u, g)
            self.full = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=1., hy=1., hz=1., unit="mm")
        else:
            from oracle import q1 as Q
            g = Q.make_grid((planes, ny, nx), (1., 1., 1.))
            self.P = Q.make_problem(g, self.fixed, self.moving, np.zeros(g.shape + (3,)), weights["lam"],
                                    weights["mu"], weights["nu"], weights["kappa"])
            self.full = Q.make_grid((nz, ny, nx), (1., 1., 1.))

    def _reference_component(self, name):
        from jd_curl.three_d.residuals import evaluate_trial, promote_trial
        from jd_curl.three_d.linearization import (build_linearization, energy_gradient, outer_gradient_vectors,
                                                   barrier_ggn_diagonal)
        from jd_curl.three_d.energy_comparison import stable_energy_reduction
        from jd_curl.three_d.poisson import build_poisson_inverse
        from jd_curl.three_d.solvers.jd_affine import node_min_jd
        from jd_curl.three_d.feasibility import certify_map
        P = self.P
        if self._base is None:
            trial = evaluate_trial(P, self.theta)
            if not hasattr(trial, "energy"):
                raise RuntimeError(f"CPU baseline state not certified: {trial}")
            self._base = promote_trial(P, trial)
            w = self.weights
            self._inverse = build_poisson_inverse(self.full, a=w["lam"], b=w["mu"] / 2 + w["nu"] / 2, metric="q1")
        base = self._base
        t0 = time.perf_counter()
        if name == "evaluate":
            evaluate_trial(P, self.theta)
        elif name == "promote":
            promote_trial(P, base)
        elif name == "compare":
            stable_energy_reduction(P, base, base)
        elif name == "gradient":
            energy_gradient(build_linearization(P, base))
        elif name == "outer":
            outer_gradient_vectors(build_linearization(P, base))
        elif name == "ggn":
            barrier_ggn_diagonal(build_linearization(P, base))
        elif name == "node_jd":
            node_min_jd(P, base, extension_activation=.25)
        elif name == "certify":
            certify_map(base.u, P.grid, config=self.cfg)
        elif name == "direction":
            inverse = self._inverse
            t0 = time.perf_counter()            # the inverse is built once per inner solve: only its apply counts
            inverse.apply(self.rhs)
        return time.perf_counter() - t0

    def _port_component(self, name):
        from oracle import cert as oc
        from oracle import q1 as Q
        P, u = self.P, self.u
        if self._base is None:
            self._base = Q.warp(P, u, True)
        w, gi = self._base
        t0 = time.perf_counter()
        if name == "evaluate":
            oc.certify_map(u, (1., 1., 1.), 0.0)
            Q.energy(P, u, Q.warp(P, u)[0])
        elif name == "promote":
            Q.warp(P, u, True)
        elif name == "compare":
            Q.differences(P, np.zeros_like(u), w, u, w)
        elif name in ("gradient", "outer"):
            Q.gradient(P, u, w, gi)
        elif name == "ggn":
            Q.ggn_diagonal(P, u, gi)
        elif name == "node_jd":
            Q.node_min_jd(P, u, .25)
        elif name == "certify":
            oc.certify_map(u, (1., 1., 1.), 0.0)
        elif name == "direction":
            Q.poisson_apply(self.full, self.weights["lam"], .03, self.rhs)
        return time.perf_counter() - t0

    def time(self, name):
        self.t[name] = (self._reference_component if self.ref is not None else self._port_component)(name)
        return self.t[name]

    def all(self):
        for name in PER_OUTER:
            self.time(name)

    def seconds_per_pair(self):
        per_outer = sum(PER_OUTER[k] * self.t[k] * (1. if k == "direction" else self.scale) for k in PER_OUTER)
        return per_outer * self.outer

    def sample(self):
        nx, ny, nz = self.shape
        what = (f"the reference package (jd_curl, Numba threads = {self.cores})" if self.ref is not None
                else "the oracle port (numpy, one thread)")
        comps = ", ".join(f"{k} {self.t[k]:.3g} s x {PER_OUTER[k]}" for k in PER_OUTER if k in self.t)
        return (f"{what} per component on a {nx}x{ny}x{self.planes} z-slab of the workload (a certified state: the "
                f"ground-truth in-plane field at half strength), x{self.scale:.1f} cell planes to the volume, DST-I "
                f"at full size; per outer step: {comps}; x{self.outer} outer steps = {self.seconds_per_pair():.1f} s "
                f"per pair (pre-optimizer not counted)")


def parity_check(grid, fixed, moving, weights, u_dev, planes):
    """parity_leg with its failure recorded in the result (the bench line is still printed)."""
    try:
        return parity_leg(grid, fixed, moving, weights, u_dev, planes)
    except Exception as exc:       # a checker failure is a result, not a crash of the measurement
        return {"pass": False, "error": f"{type(exc).__name__}: {exc}"}


def parity_leg(grid, fixed, moving, weights, u_dev, planes):
    """The checker leg: the final certified field of the run against the oracle (the C restatement of the reference
    certifier and the numpy restatement of the energy path), outside every timed region.  Returns a dict of
    equalities and maximal relative errors (normwise for vectors)."""
    import torch
    from oracle import cert as oc
    from oracle import q1 as Q
    from seq_vp_3d_b200 import certificate as cert_mod
    from seq_vp_3d_b200.pair import DevicePair
    started = time.perf_counter()
    nz, ny, nx = grid.shape
    u = u_dev.detach().cpu().numpy()
    out = {}
    # certificate: every record field of the GPU certify_map equals the C oracle's (PrescreenCertificateConfig)
    cfg = cert_mod.NATIVE_CERTIFICATE
    r = cert_mod.result_from_record(cert_mod.certifier(grid, cfg).run(u_dev), grid, cfg, None)
    nan = float("nan")
    gi = np.array([cert_mod.STATUS.index(r.status), cert_mod.REASONS.index(r.reason), r.n_cells_checked,
                   r.n_uncertain, r.n_infeasible, r.n_boxes, r.max_depth,
                   -1 if r.witness_cell is None else r.witness_cell, r.n_fast_cells, r.n_fallback_cells,
                   r.n_prescreen_cells, r.min_jd_lower_bound is not None, r.sampled_min_jd is not None])
    gf = np.array([nan if r.min_jd_lower_bound is None else r.min_jd_lower_bound,
                   nan if r.min_margin_lower_bound is None else r.min_margin_lower_bound,
                   nan if r.sampled_min_jd is None else r.sampled_min_jd,
                   *(r.witness_reference_point or (nan, nan, nan))])
    t0 = time.perf_counter()
    oi, of = oc.certify_map(u, grid.spacing, cfg.delta, max_depth=cfg.max_depth, max_boxes=cfg.max_boxes,
                            tile_size=cfg.tile_size)
    bits = lambda a: np.where(np.isnan(a), 0., a).view(np.uint64)
    out["certificate_record_equal"] = bool(np.array_equal(gi, oi) and np.array_equal(np.isnan(gf), np.isnan(of))
                                           and np.array_equal(bits(gf), bits(of)))
    out["certificate"] = dict(status=r.status, min_jd_lower_bound=r.min_jd_lower_bound, n_fast_cells=r.n_fast_cells,
                              n_prescreen_cells=r.n_prescreen_cells, n_fallback_cells=r.n_fallback_cells,
                              oracle_seconds=time.perf_counter() - t0)
    # the energy path on a pair with the identity reference (proximity, JD and curl terms all nonzero)
    pair = DevicePair(grid, fixed, moving, torch.zeros_like(u_dev), **weights)
    og = Q.make_grid((nz, ny, nx), grid.spacing)
    coeff_o = Q.spline_coefficients(moving, og)
    rel = lambda a, b: float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))
    out["spline_coefficients_rel"] = rel(pair.spline_coefficients().cpu().numpy(), coeff_o)
    warped, image_grad = pair.warp(u_dev, with_gradient=True)
    terms, _ = pair.energy(u_dev, warped)
    g_dev = pair.gradient(u_dev, warped, image_grad, term="total")
    a, b = weights["lam"], weights["mu"] / 2 + weights["nu"] / 2
    x_full = pair.poisson_apply(a, b, g_dev).cpu().numpy()
    d_full = pair.ggn_diagonal(u_dev, image_grad).cpu().numpy()
    node = pair.node_min_jd(u_dev, .25).cpu().numpy()
    g_full, w_g, ig_g = g_dev.cpu().numpy(), warped.cpu().numpy(), image_grad.cpu().numpy()
    # the mixed form's float32 kernels on the same state, against these float64 values (the oracle-checked ones)
    mp = DevicePair(grid, fixed, moving, torch.zeros_like(u_dev), precision="mixed", **weights)
    mixed = dict(gradient_rel=rel(mp.gradient(u_dev, warped, image_grad, term="total").cpu().numpy(), g_full),
                 ggn_diagonal_rel=rel(mp.ggn_diagonal(u_dev, image_grad).cpu().numpy(), d_full),
                 dst_apply_rel=rel(mp.poisson_apply(a, b, g_dev).cpu().numpy(), x_full),
                 energy_terms_rel=0.0)
    rd = cert_mod.result_from_record(cert_mod.certifier(grid, cfg, directed=True).run(u_dev), grid, cfg, None)
    mixed["certificate_directed"] = dict(status=rd.status, same_status=rd.status == r.status,
                                         min_jd_lower_bound=rd.min_jd_lower_bound,
                                         bound_at_least_plain=bool(rd.min_jd_lower_bound is not None and
                                                                   r.min_jd_lower_bound is not None and
                                                                   rd.min_jd_lower_bound >= r.min_jd_lower_bound))
    mixed["note"] = ("float32 gradient / GGN diagonal / DST-I against the float64 path on the final state; the "
                     "energies of record are float64 in both forms (energy_terms_rel); the mixed form screens its E "
                     "differences in float32 and retakes them in float64 near every decision (result.screen)")
    out["mixed_form_errors"] = mixed
    del pair, mp, warped, image_grad, g_dev
    # DST-I apply at full size
    out["dst_apply_rel"] = rel(x_full, Q.poisson_apply(og, a, b, g_full))
    # energy terms at full size (cell terms and node terms by z-slabs on every host core, summed in long double)
    out["energy_terms_rel"] = _oracle_energy(u, fixed, coeff_o, og, weights, terms)
    # a z-slab of node planes [lo, hi): its interior nodes see only slab cells, so their values are the full field's
    z0 = nz // 2 - planes // 2
    lo, hi = z0 - 1, z0 + planes - 1
    sg = Q.make_grid((hi - lo, ny, nx), grid.spacing)
    pts = og.identity()[lo:hi] + u[lo:hi]
    v, gr = Q.spline_sample(coeff_o, og, pts.reshape(-1, 3), True)
    v, gr = v.reshape(sg.shape), gr.reshape(sg.shape + (3,))
    out["warp_rel"] = max(rel(w_g[lo:hi], v), rel(ig_g[lo:hi], gr))
    P = Q.Problem(sg, fixed[lo:hi], None, np.zeros_like(u[lo:hi]), weights["lam"], weights["mu"], weights["nu"],
                  weights["kappa"])
    sl = lambda vec: vec.reshape(3, nz - 2, ny - 2, nx - 2)[:, lo:hi - 2]
    out["gradient_rel"] = rel(sl(g_full), Q.gradient(P, u[lo:hi], v, gr))
    out["ggn_diagonal_rel"] = rel(sl(d_full), Q.ggn_diagonal(P, u[lo:hi], gr))
    out["node_jd_rel"] = rel(node[lo + 1:hi - 1], Q.node_min_jd(P, u[lo:hi], .25)[0][1:-1])
    out["slab"] = f"node planes {lo}..{hi - 1} of {nz} (x {nx}, y {ny}); interior planes {lo + 1}..{hi - 2} compared"
    out["max_rel"] = float(max(out[k] for k in list(out) if k.endswith("_rel")))
    out["tolerance"] = 1e-12
    out["pass"] = bool(out["certificate_record_equal"] and out["max_rel"] <= 1e-12)
    out["seconds"] = time.perf_counter() - started
    return out


def _energy_slab(args):
    """(image, proximity, jd, curl, barrier) partial sums of cell planes [c0, c1) and node planes [c0, n1) of the
    full-size state, in long double (a worker of _oracle_energy)."""
    c0, c1, n1, u, fixed, coeff_path, shape, spacing, w = args
    from oracle import q1 as Q
    coeff = np.load(coeff_path, mmap_mode="r")
    nz, ny, nx = shape
    og = Q.make_grid(shape, spacing)
    sg = Q.make_grid((c1 - c0 + 1, ny, nx), spacing)
    P = Q.Problem(sg, None, None, np.zeros_like(u), w["lam"], w["mu"], w["nu"], w["kappa"])
    jd, cu, bar = Q.cell_terms(P, u)
    m = n1 - c0
    pts = og.identity()[c0:n1] + u[:m]
    v, _ = Q.spline_sample(np.asarray(coeff), og, pts.reshape(-1, 3), False)
    q = og.node_weights()[c0:n1]
    image = .5 * np.sum(q * (v.reshape(q.shape) - fixed[:m]) ** 2, dtype=np.longdouble)
    prox = .5 * w["lam"] * np.sum(q[..., None] * u[:m] ** 2, dtype=np.longdouble)
    return np.array([image, prox, jd, cu, bar], dtype=np.longdouble)


def _oracle_energy(u, fixed, coeff, og, weights, gpu_terms):
    """Max relative error of the GPU's five energy terms against the oracle's at full size, the oracle's sums split
    into z-slabs over a spawn process pool on the host cores."""
    import multiprocessing as mp
    import tempfile
    from concurrent.futures import ProcessPoolExecutor
    nz = u.shape[0]
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "coeff.npy")
        np.save(path, coeff)
        jobs = []
        for c0 in range(0, nz - 1, 8):
            c1 = min(c0 + 8, nz - 1)
            n1 = c1 + 1 if c1 == nz - 1 else c1
            jobs.append((c0, c1, n1, np.ascontiguousarray(u[c0:c1 + 1]), np.ascontiguousarray(fixed[c0:n1]), path,
                         u.shape[:3], og.spacing, weights))
        workers = max(1, min(len(jobs), os.cpu_count() or 1))
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            total = np.zeros(5, dtype=np.longdouble)
            for part in ex.map(_energy_slab, jobs):
                total += part
    ref = total.astype(np.float64)
    return float(np.max(np.abs(np.asarray(gpu_terms) - ref) / np.maximum(np.abs(ref), 1e-300)))


# ------------------------------------------------------------------------------------------ serving form
def serving_bench(args, grid, weights, shape, config, world, rank, local):
    """--concurrency K: K registrations in flight through the serving form (own streams and threads); a step is one
    round of K distinct pairs (seeds seed .. seed + K - 1).  value = pairs / device time of the timed rounds;
    latency percentiles from submission to certified result; e2e = the same rounds from pinned host images with the
    certified u copied back to pinned host memory."""
    import torch
    from seq_vp_3d_b200.preopt import NATIVE_PREOPT, register_pair
    from seq_vp_3d_b200.serve import RegistrationServer
    from seq_vp_3d_b200.solver import PGConfig3D
    from seq_vp_3d_b200.synthetic import head_pair
    nx, ny, nz = shape
    K = args.concurrency
    host = [head_pair((nz, ny, nx), (1., 1., 1.), seed=args.seed + rank * K + k)[:2] for k in range(K)]
    dev = [(torch.from_numpy(f).cuda(), torch.from_numpy(m).cuda()) for f, m in host]
    pinned = [(torch.from_numpy(f).pin_memory(), torch.from_numpy(m).pin_memory()) for f, m in host]
    outs = [torch.empty(grid.shape + (3,), dtype=torch.float64).pin_memory() for _ in range(K)]

    def run(fixed, moving, g, w, out=None):
        res, _ = register_pair(fixed, moving, g, w, preopt=NATIVE_PREOPT if args.preopt else None,
                               outer=args.outer, inner_config=PGConfig3D(), precision=args.form)
        if out is not None:
            out.copy_(res.final_state.u, non_blocking=True)
        return res

    def rounds(srv, n, inputs, copy_back):
        results = []
        for _ in range(n):
            futs = [srv.submit(f, m, grid, dict(weights, **({"out": outs[k]} if copy_back else {})))
                    for k, (f, m) in enumerate(inputs)]
            results += [fu.result() for fu in futs]
        return results

    def runner(fixed, moving, g, w):
        w = dict(w)
        out = w.pop("out", None)
        return run(fixed, moving, g, w, out)

    stream = torch.cuda.current_stream()
    with RegistrationServer(slots=K, run=runner) as srv:
        rounds(srv, args.warmup, dev, False)
        srv.latencies.clear()
        torch.cuda.synchronize()
        with Clocks(local) as clocks:
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            results = rounds(srv, args.steps, dev, False)
            torch.cuda.synchronize()
            end.record(stream)
            end.synchronize()
        seconds = start.elapsed_time(end) / 1e3
        lat = srv.percentiles()
        torch.cuda.synchronize()
        e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_start.record(stream)
        rounds(srv, args.steps, pinned, True)
        torch.cuda.synchronize()
        e_end.record(stream)
        e_end.synchronize()
        e2e_seconds = e_start.elapsed_time(e_end) / 1e3
    pairs = K * args.steps
    if rank == 0:
        r = results[-1]
        line = dict(metric=METRIC.format(args.form) + f", serving {K} in flight", value=pairs / seconds * 3600.,
                    unit="pairs/hour", n_gpus=world, steps=args.steps, warmup=args.warmup,
                    ms_per_step=seconds * 1e3 / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
                    dtype="f64", data="synthetic", config=dict(config, concurrency=K, pairs_per_step=K),
                    latency_s=lat,
                    e2e=dict(value=pairs / e2e_seconds * 3600., unit="pairs/hour",
                             h2d_bytes_per_step=K * 2 * host[0][0].nbytes,
                             d2h_bytes_per_step=K * outs[0].numel() * 8),
                    clocks=clocks.summary(), certified=all(x.certified for x in results),
                    result=dict(status=r.status, outer_accepted=r.counts["outer_accepted"], final_mse=r.final_mse))
        print(json.dumps(line))
    return 0


SERVE_GRIDS = ((96, 96, 96), (128, 144, 128), (160, 192, 160), (160, 192, 224))   # nx, ny, nz


def serve_sweep(args, world, rank, local):
    """Open-loop serving: for each arrival rate, --serve-requests requests arrive at Poisson times (exponential
    gaps, seeded) and are admitted by the server as slots and HBM footprint allow; each request registers a seeded
    blob pair (the 32^3 generator at its grid) for a fixed outer-step budget and returns only a certified field.
    Reports, per rate, the latency from arrival to certified result (p50/p95/p99) and the pairs/hour delivered."""
    import torch
    from seq_vp_3d_b200.grid import make_grid_3d
    from seq_vp_3d_b200.preopt import NATIVE_PREOPT, register_pair
    from seq_vp_3d_b200.serve import RegistrationServer
    from seq_vp_3d_b200.synthetic import blob_pair, default_weights
    rates = [float(r) for r in args.serve.split(",")]
    rng = np.random.default_rng(args.seed)
    # the request mix: 25% 48^3, the rest uniform over the four grids; a pool of distinct seeded pairs per grid
    kinds = [(48, 48, 48) if rng.random() < .25 else SERVE_GRIDS[rng.integers(len(SERVE_GRIDS))]
             for _ in range(args.serve_requests)]
    pool = {}
    for k, shape in enumerate(kinds):
        nx, ny, nz = shape
        if shape not in pool:
            pool[shape] = []
        if len(pool[shape]) < 2:
            f, m, _ = blob_pair((nz, ny, nx), (1., 1., 1.), seed=args.seed + 1000 * len(pool[shape]) + nx + ny + nz)
            grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=1., hy=1., hz=1., unit="mm")
            pool[shape].append((torch.from_numpy(f).cuda(), torch.from_numpy(m).cuda(), grid,
                                default_weights((nz, ny, nx), (1., 1., 1.))))
    requests = [pool[shape][k % len(pool[shape])] for k, shape in enumerate(kinds)]

    def run(fixed, moving, grid, weights):
        res, _ = register_pair(fixed, moving, grid, weights, preopt=NATIVE_PREOPT if args.preopt else None,
                               outer=args.serve_outer, precision=args.form)
        return res

    rows = []
    with RegistrationServer(slots=args.serve_slots, run=run) as srv:
        for f, m, grid, w in requests[:2]:          # warm-up: library set-up and pools
            srv.submit(f, m, grid, w).result()
        with Clocks(local) as clocks:
            for rate in rates:
                gaps = rng.exponential(3600. / rate, size=len(requests))
                srv.latencies.clear()
                t0 = time.perf_counter()
                futures, due = [], t0
                for (f, m, grid, w), gap in zip(requests, gaps):
                    due += gap
                    wait = due - time.perf_counter()
                    if wait > 0:
                        time.sleep(wait)
                    futures.append(srv.submit(f, m, grid, w))
                results = [fu.result() for fu in futures]
                span = time.perf_counter() - t0
                lat = srv.percentiles()
                rows.append(dict(rate_per_hour=rate, requests=len(requests), pairs_per_hour=len(requests) / span * 3600.,
                                 latency_s=lat, certified=all(r.certified for r in results),
                                 mean_final_mse=float(np.mean([r.final_mse for r in results]))))
    if rank == 0:
        best = max(rows, key=lambda r: r["pairs_per_hour"])
        line = dict(metric=METRIC.format(args.form) + ", open-loop serving sweep", value=best["pairs_per_hour"],
                    unit="pairs/hour", n_gpus=world, steps=len(rates), warmup=2,
                    ms_per_step=None, higher_is_better=True, scaling="weak", vs_baseline=None,
                    dtype="f64" if args.form == "plain" else "f32+f64", data="synthetic",
                    config=dict(workload="open-loop Poisson arrivals of seeded blob pairs, grids 96^3 / 128x144x128 / "
                                         "160x192x160 / 160x192x224 with 25% 48^3, pre-optimizer + certified loop",
                                outer_steps=args.serve_outer, slots=args.serve_slots,
                                mix={f"{a}x{b}x{c}": kinds.count((a, b, c)) for a, b, c in set(kinds)}),
                    sweep=rows, clocks=clocks.summary())
        print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------ reference arm
def reference_arm(args, shape, config):
    from seq_vp_3d_b200.synthetic import default_weights, head_pair
    nx, ny, nz = shape
    weights = default_weights((nz, ny, nx), (1., 1., 1.))
    fixed, moving, ugt = head_pair((nz, ny, nx), (1., 1., 1.), seed=args.seed)
    table = CpuTable(shape, fixed, moving, ugt, weights, args.cpu_planes, args.outer)
    names = list(PER_OUTER)
    t_all = time.perf_counter()
    for w in range(max(1, args.warmup)):
        if w == 0:
            table.all()                 # compiles the reference's Numba kernels and fills the table
        else:
            table.time(names[w % len(names)])
    vals, seconds = [], []
    for k in range(args.steps):
        t0 = time.perf_counter()
        table.time(names[k % len(names)])
        seconds.append(time.perf_counter() - t0)
        vals.append(3600. / table.seconds_per_pair())
    value = float(np.mean(vals))
    line = dict(metric=METRIC.format(args.form), value=value, unit="pairs/hour", n_gpus=args.gpus, steps=args.steps,
                warmup=args.warmup, ms_per_step=3.6e6 / value, higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="f64", data="synthetic", config=config, impl="reference",
                cpu_baseline=dict(value=value, unit="pairs/hour", cores=table.cores, kind=table.kind,
                                  sample=table.sample(), components_s=table.t),
                e2e=dict(value=value, unit="pairs/hour", h2d_bytes_per_step=0, d2h_bytes_per_step=0),
                sample_seconds_per_step=float(np.mean(seconds)) if seconds else None,
                wall_seconds=time.perf_counter() - t_all)
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------ main
def main():
    args = parse()
    shape = tuple(int(v) for v in args.shape.split(","))
    nx, ny, nz = shape
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    from seq_vp_3d_b200.synthetic import default_weights, head_pair
    weights = default_weights((nz, ny, nx), (1., 1., 1.))
    start = ("float32 8/4/2/1 pyramid pre-optimizer, taper, certified transfer, then" if args.preopt else "from u=0:")
    forms = {"plain": "plain FP64", "mixed": "mixed (float32 bulk, float64 decisions and certificate)"}
    config = {"workload": f"head phantom pair {nx}x{ny}x{nz} (x fastest), 1 mm, float64, certified proximal loop "
                          f"{start} {args.outer} outer steps x 5 PG steps (T73 metric)",
              "grid_nodes": nx * ny * nz, "outer_steps": args.outer, "inner_steps": 5, "form": forms[args.form],
              "l2_policy": "inputs larger than L2 (6.9M-node fields, 55-165 MB each)"}
    if args.impl == "reference":
        if rank != 0:
            return 0
        return reference_arm(args, shape, config)

    import torch
    torch.cuda.set_device(local)
    ranks = Ranks("nccl", "cuda")
    import ctypes
    from seq_vp_3d_b200 import _lib
    from seq_vp_3d_b200.grid import make_grid_3d
    from seq_vp_3d_b200.preopt import register_pair
    from seq_vp_3d_b200.solver import PGConfig3D, Registration, SequentialConfig3D, solve_sequential

    fixed, moving, ugt = head_pair((nz, ny, nx), (1., 1., 1.), seed=args.seed + rank)
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=1., hy=1., hz=1., unit="mm")
    f_dev = torch.from_numpy(fixed).cuda()
    m_dev = torch.from_numpy(moving).cuda()
    outer_cfg, inner_cfg = SequentialConfig3D(max_iterations=args.outer), PGConfig3D()
    stream = torch.cuda.current_stream()
    phases = []

    def step(f, m, form):
        if args.preopt:
            res, record = register_pair(f, m, grid, weights, outer=args.outer, inner_config=inner_cfg,
                                        precision=form)
        else:
            reg = Registration(grid, f, m, **weights, precision=form)
            res, record = solve_sequential(reg, config=outer_cfg, inner_config=inner_cfg), {}
        if not res.certified:
            raise RuntimeError(f"registration ended without a certified state: {res.status}")
        phases.append(dict(preopt_s=record.get("preopt", {}).get("seconds"),
                           transfer_s=record.get("transfer", {}).get("elapsed_seconds"),
                           certified_loop_s=res.elapsed_seconds))
        return res

    def barrier():
        ranks.barrier()
        torch.cuda.synchronize()

    max_over_ranks = ranks.max

    def launches():
        n = ctypes.c_int64()
        _lib.call("svp_counters", ctypes.byref(n))
        return n.value

    def timed_pairs(form, count, f, m, copy_back=None):
        """count pairs bracketed by barriers and CUDA events: (max-over-ranks seconds, per-pair seconds, results).
        With copy_back, each pair's images come from the pinned host buffers f, m and its certified u and warped
        image go back to the pinned buffers copy_back, inside the timed region."""
        barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        marks = [torch.cuda.Event(enable_timing=True) for _ in range(count)]
        start.record(stream)
        results = []
        for k in range(count):
            if copy_back is None:
                res = step(f, m, form)
            else:
                res = step(f.to("cuda", non_blocking=True), m.to("cuda", non_blocking=True), form)
                copy_back[0].copy_(res.final_state.u, non_blocking=True)
                copy_back[1].copy_(res.final_state.warped, non_blocking=True)
            marks[k].record(stream)
            results.append(res)
        end.record(stream)
        barrier()
        edges = [start] + marks
        per_pair = [edges[k].elapsed_time(edges[k + 1]) / 1e3 for k in range(count)]
        return max_over_ranks(start.elapsed_time(end) / 1e3), per_pair, results

    if args.concurrency > 1:
        return serving_bench(args, grid, weights, shape, config, world, rank, local)
    if args.serve:
        return serve_sweep(args, world, rank, local)

    for _ in range(args.warmup):
        step(f_dev, m_dev, args.form)
    # ---------------------------------------------------------------- timed: device-resident inputs, timers off
    n0 = launches()
    with Clocks(local) as clocks:
        seconds, per_pair, results = timed_pairs(args.form, args.steps, f_dev, m_dev)
    n1 = launches()
    value = whole_job_rate(args.steps, seconds, world)
    # ---------------------------------------------------------------- e2e: public API from pinned host buffers
    f_host = torch.from_numpy(fixed).pin_memory()
    m_host = torch.from_numpy(moving).pin_memory()
    u_out = torch.empty(grid.shape + (3,), dtype=torch.float64).pin_memory()
    w_out = torch.empty(grid.shape, dtype=torch.float64).pin_memory()
    e2e_seconds, _, _ = timed_pairs(args.form, args.steps, f_host, m_host, copy_back=(u_out, w_out))
    e2e_value = whole_job_rate(args.steps, e2e_seconds, world)
    h2d = 2 * fixed.nbytes
    d2h = u_out.numel() * 8 + w_out.numel() * 8
    # ---------------------------------------------------------------- the other form, for the mixed/plain ratio
    other = "mixed" if args.form == "plain" else "plain"
    compare = None
    if args.compare_steps > 0:
        step(f_dev, m_dev, other)
        o_seconds, _, o_results = timed_pairs(other, args.compare_steps, f_dev, m_dev)
        o_value = whole_job_rate(args.compare_steps, o_seconds, world)
        by = {args.form: (value, results[-1], args.steps), other: (o_value, o_results[-1], args.compare_steps)}
        compare = {k: dict(value=v, ms_per_pair=3.6e6 / v * world, pairs=n, final_mse=r.final_mse,
                           certified=bool(r.certified), outer_accepted=r.counts["outer_accepted"])
                   for k, (v, r, n) in by.items()}
        compare["mixed_over_plain"] = by["mixed"][0] / by["plain"][0]
        compare["final_mse_rel_diff"] = (abs(by["mixed"][1].final_mse - by["plain"][1].final_mse)
                                         / by["plain"][1].final_mse)
    # ---------------------------------------------------------------- one more pair with the kernel timers on
    _lib.call("svp_timers_enable", 1)
    step(f_dev, m_dev, args.form)
    torch.cuda.synchronize()
    timers = {}
    for name in (*kernel_counts(shape), *STATE_DEPENDENT_KERNELS):
        cnt, ms = ctypes.c_int64(), ctypes.c_double()
        _lib.call("svp_timer_read", name.encode(), ctypes.byref(cnt), ctypes.byref(ms))
        if cnt.value:
            timers[name] = (cnt.value, ms.value)
    _lib.call("svp_timers_enable", 0)
    timer_phase = phases[-1]

    if rank == 0:
        counts = kernel_counts(shape)
        counted = {k: v for k, v in timers.items() if k in counts}
        dominant = max(counted, key=lambda k: counted[k][1]) if counted else None
        hbm, kind = peaks()
        roofline = None
        if dominant:
            cnt, ms = timers[dominant]
            per_launch_s = ms / 1e3 / cnt
            nbytes, flop = counts[dominant]
            achieved = nbytes / per_launch_s / 1e9
            ncell = (nx - 1) * (ny - 1) * (nz - 1)
            traffic = TRAFFIC_PER_CELL[dominant] * ncell if dominant in TRAFFIC_PER_CELL else None
            roofline = dict(kernel=dominant, bound="hbm", achieved=achieved, peak=hbm, unit="GB/s",
                            frac=achieved / hbm, traffic=traffic, peak_source=kind, launches=cnt,
                            avg_launch_ms=ms / cnt, algorithmic_bytes_per_launch=nbytes,
                            share_of_loop=ms / 1e3 / (timer_phase["certified_loop_s"] or 1.),
                            timing="CUDA events on the launch stream, one separate pair with the timers on")
            if flop:
                # the cell kernels are FP64-pipe bound: their FLOP rate against the nominal FP64 peak
                roofline["fp64"] = dict(flop_per_launch=flop, achieved_tflops=flop / per_launch_s / 1e12,
                                        peak_tflops=FP64_PEAK_TFLOPS, frac=flop / per_launch_s / 1e12 / FP64_PEAK_TFLOPS,
                                        peak_source="nominal (148 SMs x 64 FP64 FMA/clk x 2 x 1965 MHz)")
            if dominant in FLOP32_PER_CELL:
                # the mixed form's float32 cell kernels: their counted float32 rate against the nominal FP32 peak
                flop32 = FLOP32_PER_CELL[dominant] * ncell
                roofline["fp32"] = dict(flop_per_launch=flop32, achieved_tflops=flop32 / per_launch_s / 1e12,
                                        peak_tflops=FP32_PEAK_TFLOPS,
                                        frac=flop32 / per_launch_s / 1e12 / FP32_PEAK_TFLOPS,
                                        peak_source="nominal (148 SMs x 128 FP32 FMA/clk x 2 x 1965 MHz)")
        if args.profile:
            total = sum(v[1] for v in timers.values())
            for k, (c, ms) in sorted(timers.items(), key=lambda kv: -kv[1][1]):
                print(f"[profile] {k:24s} launches={c:7d} total={ms:10.1f} ms avg={ms / c:8.3f} ms "
                      f"share={ms / total:6.3f}", file=sys.stderr)
            r = results[-1]
            print(f"[profile] pair: status={r.status} outer={r.counts['outer_accepted']} trials={r.counts['trials']} "
                  f"mse {r.native_mse:.6g} -> {r.final_mse:.6g} GF {r.GF_initial:.4g} -> {r.GF_final:.4g}",
                  file=sys.stderr)
        cpu = parity = None
        if world == 1 and not args.no_cpu:
            table = CpuTable(shape, fixed, moving, ugt, weights, args.cpu_planes, args.outer)
            table.all()
            cpu = dict(value=3600. / table.seconds_per_pair(), unit="pairs/hour", cores=table.cores,
                       kind=table.kind, sample=table.sample(), components_s=table.t)
            parity = parity_check(grid, fixed, moving, weights, results[-1].final_state.u, args.parity_planes)
        r = results[-1]
        lat = {f"p{q}": float(np.percentile(per_pair, q)) for q in (50, 95, 99)}
        line = dict(metric=METRIC.format(args.form), value=value, unit="pairs/hour", n_gpus=world, steps=args.steps,
                    warmup=args.warmup, ms_per_step=seconds * 1e3 / args.steps, higher_is_better=True,
                    scaling="weak", vs_baseline=None, dtype="f64" if args.form == "plain" else "f32+f64",
                    data="synthetic", config=config, latency_s=lat,
                    e2e=dict(value=e2e_value, unit="pairs/hour", h2d_bytes_per_step=h2d, d2h_bytes_per_step=d2h),
                    gpu_launches=int(n1 - n0), roofline=roofline, cpu_baseline=cpu, clocks=clocks.summary(),
                    forms=compare, parity=parity,
                    result=dict(status=r.status, certified=bool(r.certified), outer_accepted=r.counts["outer_accepted"],
                                trials=r.counts["trials"], native_mse=r.native_mse, final_mse=r.final_mse,
                                GF_initial=r.GF_initial, GF_final=r.GF_final, screen=r.counts.get("screen")),
                    phases=phase_summary(timer_phase, timers))
        print(json.dumps(line))
    ranks.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
