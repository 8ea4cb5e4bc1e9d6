#!/usr/bin/env python
"""Certified registration pairs per hour at 160x192x224 on B200 GPUs (plain FP64 form).

One step = one complete certified registration of a seeded head-phantom pair (the 160x192x224 synthetic workload):
device pair setup (spline prefilter, constants), then the certified proximal loop from u = 0 for --outer outer steps
(5 accepted PG steps each), every accepted state proven J > 0 on every closed cell by the GPU certificate.
`value`: pairs/hour with the images already in HBM; `e2e`: the same through the public API with the images in
pinned host memory and the certified displacement + warped image copied back every step.

Multi-GPU: one process per GPU, independent pairs per rank (replicas only: registrations are independent units and
the path has no exchange step); value = all ranks' pairs / max-over-ranks time.

--impl reference: the reference's CPU implementation of the path restated in oracle/ (the reference is Python and
is not installed on the GPU host) timed on the host cores on a bounded sample, extrapolated per pair.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "certified pairs/hour @160x192x224 ({} form, 1 B200 per pair)"
SMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
# counts per outer step of the default route (5 accepted PG steps, one trial each on these pairs, as in the
# reference's own run of the small seeded pair): used only by the CPU extrapolation
PER_OUTER = dict(trials=5, gradients=5, outer_triples=1, directions=5, metric_builds=1, certificates=5)


def parse():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--outer", type=int, default=200, help="outer steps per registration (config 2: 200)")
    ap.add_argument("--form", choices=("plain", "mixed"), default="plain",
                    help="plain: float64 throughout; mixed: float32 search direction (gradient, GGN diagonal, DST-I) "
                         "with float64 energies, decisions and certificate")
    ap.add_argument("--concurrency", type=int, default=1,
                    help="serving form: registrations in flight at once (each on its own stream); a step is one "
                         "round of that many pairs, value = all pairs / time, with p50/p95/p99 latency")
    ap.add_argument("--preopt", action=argparse.BooleanOptionalAction, default=True,
                    help="config-2 route: float32 8/4/2/1 pyramid pre-optimizer + certified transfer before the "
                         "native steps")
    ap.add_argument("--shape", default="160,192,224", help="nx,ny,nz")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--cpu-slab", type=int, default=4, help="z-planes of the CPU baseline sample")
    ap.add_argument("--profile", action="store_true", help="per-kernel device times to stderr")
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
# DRAM bytes (read + write) per cell measured by ncu on the 160x192x96 pair (2,885,055 cells; profiles/
# traffic_cell_trial_edge_hull_warp_160x192x96.md); scaled to a launch by the cells it processes (traffic grows with
# the cell count: every launch streams its fields once, plus neighbour re-reads of the same order)
TRAFFIC_PER_CELL = {"cell_trial_kernel": (325667584 + 1371392) / 2885055,
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
        "cell_diff_kernel": (3 * 24 * nn, c("cell_diff_kernel")),
        "cell_energy_kernel": (2 * 24 * nn, c("cell_energy_kernel")),
        # u, u_ref in; 24 doubles per cell out (one locals buffer; two for the outer triple)
        "cell_grad_kernel": (2 * 24 * nn + 192 * nc, c("cell_grad_kernel")),
        "gather_kernel": (192 * nc + nn * (24 + 24 + 8 + 8 + 24) + 3 * 8 * nf, None),
        "cell_ggn_diag_kernel": (24 * nn + 192 * nc, c("cell_ggn_diag_kernel")),
        # mixed form: the same float64 inputs, float32 locals out (the FLOP counts above are float32 operations here)
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
                           "jd_root_kernel", "cell_ggn_hvp_kernel")


def phase_summary(phases, timers, steps):
    """Mean host-clock seconds per pair of the pre-optimizer, the transfer and the certified loop, the device time of
    the FP64 kernels (all inside the certified loop) and the loop's remainder: host control, syncs and launch gaps."""
    if not phases:
        return None
    mean = lambda key: (None if phases[0][key] is None else float(np.mean([p[key] for p in phases])))
    out = {k: mean(k) for k in ("preopt_s", "transfer_s", "certified_loop_s")}
    fp64 = sum(ms for name, (_, ms) in timers.items() if not name.startswith(("pre_", "adam"))) / 1e3 / steps
    out["fp64_kernels_s"] = fp64
    out["loop_host_gap_s"] = out["certified_loop_s"] - fp64
    return out


# ------------------------------------------------------------------------------------------ CPU baseline
def cpu_baseline(shape, fixed, moving, weights, slab, outer):
    """Time the oracle (the reference's CPU algorithm restated) per component on a z-slab of the pair and extrapolate
    to one registration with PER_OUTER counts x outer steps.  Returns (pairs/hour, cores, sample text, seconds)."""
    from oracle import cert as oc
    from oracle import q1 as Q
    nx, ny, nz = shape
    zs = min(slab, nz)
    sub = (zs, ny, nx)
    rng = np.random.default_rng(1)
    g = Q.make_grid(sub, (1., 1., 1.))
    P = Q.make_problem(g, fixed[:zs], moving[:zs], np.zeros(sub + (3,)), weights["lam"], weights["mu"],
                       weights["nu"], weights["kappa"])
    u = np.zeros(sub + (3,))
    u[1:-1, 1:-1, 1:-1] = rng.normal(size=(zs - 2, ny - 2, nx - 2, 3)) * 0.05
    cores = os.cpu_count() or 1
    t = {}
    t0 = time.perf_counter()
    w, gi = Q.warp(P, u, True)
    t["promote"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    w0, _ = Q.warp(P, u)
    Q.energy(P, u, w0)
    t["evaluate"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    Q.differences(P, np.zeros_like(u), w0, u, w0)
    t["compare"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    Q.gradient(P, u, w, gi)
    t["gradient"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    Q.ggn_diagonal(P, u, gi)
    Q.node_min_jd(P, u)
    t["metric"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    oc.certify_map(u, (1., 1., 1.), 0.0)
    t["certificate"] = time.perf_counter() - t0
    # DST-I apply at the full free-node size (a whole-volume transform cannot be sliced)
    full = Q.make_grid((nz, ny, nx), (1., 1., 1.))
    rhs = rng.normal(size=3 * (nx - 2) * (ny - 2) * (nz - 2))
    t0 = time.perf_counter()
    Q.poisson_apply(full, 0.01, 0.03, rhs)
    t["direction"] = time.perf_counter() - t0
    scale = nz / zs
    per_outer = ((t["evaluate"] + t["compare"] + t["promote"] + t["certificate"]) * PER_OUTER["trials"]
                 + t["gradient"] * (PER_OUTER["gradients"] + PER_OUTER["outer_triples"])
                 + t["metric"] * PER_OUTER["metric_builds"]) * scale + t["direction"] * PER_OUTER["directions"]
    seconds = per_outer * outer
    sample = (f"oracle per component on a {nx}x{ny}x{zs} slab (x{scale:.1f} to the volume) + one full-size DST-I; "
              f"per outer step {PER_OUTER['trials']} trials (certificate, value sampling, energy, stable difference, "
              f"promotion), {PER_OUTER['gradients']}+1 gradients, 1 metric build, {PER_OUTER['directions']} "
              f"directions; x{outer} outer steps = {seconds:.1f} s per pair")
    return 3600. / seconds, cores, sample, sum(t.values())


# ------------------------------------------------------------------------------------------ serving form
def serving_bench(args, grid, weights, shape, config, world, rank, Clocks, local):
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
    config = {"workload": f"head phantom pair {nx}x{ny}x{nz} (x fastest), 1 mm, float64, certified proximal loop "
                          f"{start} {args.outer} outer steps x 5 PG steps (T73 metric)",
              "grid_nodes": nx * ny * nz, "outer_steps": args.outer, "inner_steps": 5,
              "form": "plain FP64" if args.form == "plain" else "mixed (float32 direction, float64 decisions)",
              "l2_policy": "inputs larger than L2 (6.9M-node fields, 55-165 MB each)"}
    if args.impl == "reference":
        if rank != 0:
            return 0
        fixed, moving, _ = head_pair((nz, ny, nx), (1., 1., 1.), seed=args.seed)
        for _ in range(args.warmup):
            pass
        vals, samples = [], None
        t_all = time.perf_counter()
        for _ in range(max(1, args.steps)):
            v, cores, samples, _ = cpu_baseline(shape, fixed, moving, weights, args.cpu_slab, args.outer)
            vals.append(v)
        value = float(np.mean(vals))
        line = dict(metric=METRIC.format(args.form), value=value, unit="pairs/hour", n_gpus=args.gpus, steps=args.steps,
                    warmup=args.warmup, ms_per_step=3.6e6 / value, higher_is_better=True, scaling="weak",
                    vs_baseline=None, dtype="f64", data="synthetic", config=config, impl="reference",
                    cpu_baseline=dict(value=value, unit="pairs/hour", cores=cores, kind="port", sample=samples),
                    e2e=dict(value=value, unit="pairs/hour", h2d_bytes_per_step=0, d2h_bytes_per_step=0),
                    wall_seconds=time.perf_counter() - t_all)
        print(json.dumps(line))
        return 0

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    from seq_vp_3d_b200 import _lib
    from seq_vp_3d_b200.grid import make_grid_3d
    from seq_vp_3d_b200.solver import PGConfig3D, Registration, SequentialConfig3D, solve_sequential
    import ctypes

    fixed, moving, _ = head_pair((nz, ny, nx), (1., 1., 1.), seed=args.seed + rank)
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=1., hy=1., hz=1., unit="mm")
    f_dev = torch.from_numpy(fixed).cuda()
    m_dev = torch.from_numpy(moving).cuda()
    outer_cfg, inner_cfg = SequentialConfig3D(max_iterations=args.outer), PGConfig3D()
    stream = torch.cuda.current_stream()

    phases = []

    def step(f, m):
        if args.preopt:
            from seq_vp_3d_b200.preopt import register_pair
            res, record = register_pair(f, m, grid, weights, outer=args.outer, inner_config=inner_cfg,
                                        precision=args.form)
            reg = None
        else:
            reg = Registration(grid, f, m, **weights, precision=args.form)
            res, record = solve_sequential(reg, config=outer_cfg, inner_config=inner_cfg), {}
        if not res.certified:
            raise RuntimeError(f"registration ended without a certified state: {res.status}")
        # host-clock phases of the pair (the certified loop's figure includes its host control)
        phases.append(dict(preopt_s=record.get("preopt", {}).get("seconds"),
                           transfer_s=record.get("transfer", {}).get("elapsed_seconds"),
                           certified_loop_s=res.elapsed_seconds))
        return reg, res

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if args.concurrency > 1:
        return serving_bench(args, grid, weights, shape, config, world, rank, Clocks, local)

    for _ in range(args.warmup):
        step(f_dev, m_dev)
    phases.clear()
    # ---------------------------------------------------------------- timed: device-resident inputs
    launches0 = ctypes.c_int64()
    _lib.call("svp_counters", ctypes.byref(launches0))
    _lib.call("svp_timers_enable", 1)
    barrier()
    results = []
    with Clocks(local) as clocks:
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(args.steps):
            results.append(step(f_dev, m_dev)[1])
        end.record(stream)
        barrier()
    seconds = max_over_ranks(start.elapsed_time(end) / 1e3)
    launches1 = ctypes.c_int64()
    _lib.call("svp_counters", ctypes.byref(launches1))
    timers = {}
    for name in (*kernel_counts(shape), *STATE_DEPENDENT_KERNELS):
        cnt, ms = ctypes.c_int64(), ctypes.c_double()
        _lib.call("svp_timer_read", name.encode(), ctypes.byref(cnt), ctypes.byref(ms))
        if cnt.value:
            timers[name] = (cnt.value, ms.value)
    _lib.call("svp_timers_enable", 0)
    value = world * args.steps / seconds * 3600.
    timed_phases = phases[:args.steps]
    # ---------------------------------------------------------------- e2e: public API from pinned host buffers
    f_host = torch.from_numpy(fixed).pin_memory()
    m_host = torch.from_numpy(moving).pin_memory()
    u_out = torch.empty(grid.shape + (3,), dtype=torch.float64).pin_memory()
    w_out = torch.empty(grid.shape, dtype=torch.float64).pin_memory()
    barrier()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(args.steps):
        f = f_host.to("cuda", non_blocking=True)
        m = m_host.to("cuda", non_blocking=True)
        reg, res = step(f, m)
        u_out.copy_(res.final_state.u, non_blocking=True)
        w_out.copy_(res.final_state.warped, non_blocking=True)
    e_end.record(stream)
    barrier()
    e2e_seconds = max_over_ranks(e_start.elapsed_time(e_end) / 1e3)
    e2e_value = world * args.steps / e2e_seconds * 3600.
    h2d = 2 * fixed.nbytes
    d2h = u_out.numel() * 8 + w_out.numel() * 8

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
                            share_of_timed=ms / 1e3 / (seconds * world) if seconds else None)
            if flop:
                # the cell kernels are FP64-pipe bound: their FLOP rate against the nominal FP64 peak
                roofline["fp64"] = dict(flop_per_launch=flop, achieved_tflops=flop / per_launch_s / 1e12,
                                        peak_tflops=FP64_PEAK_TFLOPS, frac=flop / per_launch_s / 1e12 / FP64_PEAK_TFLOPS,
                                        peak_source="nominal (148 SMs x 64 FP64 FMA/clk x 2 x 1965 MHz)")
        if args.profile:
            total = sum(v[1] for v in timers.values())
            for k, (c, ms) in sorted(timers.items(), key=lambda kv: -kv[1][1]):
                print(f"[profile] {k:24s} launches={c:7d} total={ms:10.1f} ms avg={ms / c:8.3f} ms "
                      f"share={ms / total:6.3f}", file=sys.stderr)
            r = results[-1]
            print(f"[profile] pair: status={r.status} outer={r.counts['outer_accepted']} trials={r.counts['trials']} "
                  f"mse {r.native_mse:.6g} -> {r.final_mse:.6g} GF {r.GF_initial:.4g} -> {r.GF_final:.4g}",
                  file=sys.stderr)
        cpu = None
        if world == 1 and not args.no_cpu:
            v, cores, sample, _ = cpu_baseline(shape, fixed, moving, weights, args.cpu_slab, args.outer)
            cpu = dict(value=v, unit="pairs/hour", cores=cores, kind="port", sample=sample)
        r = results[-1]
        line = dict(metric=METRIC.format(args.form), value=value, unit="pairs/hour", n_gpus=world, steps=args.steps,
                    warmup=args.warmup, ms_per_step=seconds * 1e3 / args.steps, higher_is_better=True,
                    scaling="weak", vs_baseline=None, dtype="f64", data="synthetic", config=config,
                    e2e=dict(value=e2e_value, unit="pairs/hour", h2d_bytes_per_step=h2d, d2h_bytes_per_step=d2h),
                    gpu_launches=int(launches1.value - launches0.value), roofline=roofline, cpu_baseline=cpu,
                    clocks=clocks.summary(),
                    result=dict(status=r.status, certified=bool(r.certified), outer_accepted=r.counts["outer_accepted"],
                                trials=r.counts["trials"], native_mse=r.native_mse, final_mse=r.final_mse,
                                GF_initial=r.GF_initial, GF_final=r.GF_final),
                    phases=phase_summary(timed_phases, timers, args.steps))
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
