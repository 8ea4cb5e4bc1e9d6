"""Second half of make_golden.py: the Q1 energy/gradient/metric/DST fixture (q1.npz), generated by running the
reference's CPU path on a small seeded problem with an active localized barrier.  Imported by make_golden.py after
the reference is on sys.path."""
import os

import numpy as np


def seeded_images(shape, seed):
    """Fixed/moving pair: Gaussian blobs + noise, moving = fixed shifted smoothly (only needs to be smooth)."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    fixed = np.zeros(shape)
    moving = np.zeros(shape)
    for _ in range(10):
        c = rng.uniform([1, 1, 1], [nz - 2, ny - 2, nx - 2])
        s = rng.uniform(1.5, 3.0)
        a = rng.uniform(0.2, 1.0)
        d = rng.normal(size=3) * 0.6
        fixed += a * np.exp(-((zz - c[0]) ** 2 + (yy - c[1]) ** 2 + (xx - c[2]) ** 2) / (2 * s * s))
        moving += a * np.exp(-((zz - c[0] - d[0]) ** 2 + (yy - c[1] - d[1]) ** 2 + (xx - c[2] - d[2]) ** 2)
                             / (2 * s * s))
    fixed = fixed / fixed.max() + rng.normal(size=shape) * 0.01
    moving = moving / moving.max() + rng.normal(size=shape) * 0.01
    return fixed, moving


def compressed_field(grid, strength, centre, seed, amp=0.15):
    """Zero-boundary smooth field with a local compression along x (J ~ 1 - strength at the centre)."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = grid.shape
    hx, hy, hz = grid.spacing
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cz, cy, cx = centre
    s = 1.6
    g = np.exp(-((zz - cz) ** 2 + (yy - cy) ** 2) / (2 * s * s))
    u = np.zeros(grid.shape + (3,))
    u[..., 0] = -strength * np.clip(xx - cx, -1, 1) * hx * g
    taper = (np.sin(np.pi * zz / (nz - 1)) * np.sin(np.pi * yy / (ny - 1)) * np.sin(np.pi * xx / (nx - 1)))
    for r, h in enumerate((hx, hy, hz)):
        u[..., r] += amp * h * taper * np.sin(2 * np.pi * (r + 1) * (xx + 2 * yy + 3 * zz) / 17 + rng.uniform(0, 6))
    u[[0, -1]] = 0.; u[:, [0, -1]] = 0.; u[:, :, [0, -1]] = 0.
    return np.ascontiguousarray(u)


def make_q1(out):
    from jd_curl.three_d.grid import make_grid_3d
    from jd_curl.three_d.problem import Weights3D, make_problem
    from jd_curl.three_d.feasibility import PrescreenCertificateConfig
    from jd_curl.three_d.boundary import restrict_free, inject_free
    from jd_curl.three_d.residuals import evaluate_trial, promote_trial
    from jd_curl.three_d.linearization import (build_linearization, energy_gradient, outer_gradient_vectors,
                                               barrier_ggn_diagonal, barrier_ggn_hvp)
    from jd_curl.three_d.energy_comparison import stable_energy_reduction, stable_energy_reductions
    from jd_curl.three_d.poisson import build_poisson_inverse
    from jd_curl.three_d.solvers.poisson_gradient import (image_curvature_shift, metric_diagonal,
                                                          EquilibratedInverse)
    from jd_curl.three_d.solvers.jd_affine import node_min_jd, affine_factors
    from jd_curl.three_d.solvers.global_jd_step import global_root_cpu
    from jd_curl.three_d.interpolation import sample_points
    from jd_curl.types import InvalidTrial

    data = {}
    grid = make_grid_3d(nx=13, ny=12, nz=11, hx=1.0, hy=1.1, hz=0.9, unit="mm")
    nz, ny, nx = grid.shape
    fixed, moving = seeded_images(grid.shape, 5)
    fov = [n * h for n, h in zip((nx, ny, nz), grid.spacing)]
    lstar = float(np.prod(fov)) ** (1 / 3)
    weights = Weights3D(lam=0.1 / lstar ** 2, mu=0.03, nu=0.03, kappa=0.002)
    config = PrescreenCertificateConfig(delta=0., max_depth=48, max_boxes=255, tile_size=65536, fallback_workers=2)
    u_ref = compressed_field(grid, 0.5, (5, 6, 6), 1, amp=0.1)
    problem = make_problem(grid=grid, fixed_image=fixed, moving_image=moving, u_ref=u_ref, weights=weights,
                           certificate_config=config, barrier_location="closed27_uniform", barrier_activation=.05)
    u1 = compressed_field(grid, 0.965, (5, 6, 6), 2)
    u2 = u1 + 0.02 * compressed_field(grid, 0.3, (4, 5, 7), 3)
    t1, t2 = evaluate_trial(problem, restrict_free(u1, grid)), evaluate_trial(problem, restrict_free(u2, grid))
    assert not isinstance(t1, InvalidTrial) and not isinstance(t2, InvalidTrial), (t1, t2)
    data.update(grid=np.array([nx, ny, nz]), spacing=np.array(grid.spacing), fixed=fixed, moving=moving, u_ref=u_ref,
                u1=u1, u2=u2, weights=np.array([weights.lam, weights.mu, weights.nu, weights.kappa]),
                barrier=np.array([0.05, 0.0]))
    spline = problem.sampler._spline
    data["spline_c"] = np.asarray(spline.c)
    for k, t in enumerate(spline.t):
        data[f"knots{k}"] = np.asarray(t)
    for name, tr in (("t1", t1), ("t2", t2)):
        e = tr.energy
        data[f"{name}/energy"] = np.array([e.image, e.proximity, e.jd, e.curl, e.barrier, e.curvature])
        data[f"{name}/warped"] = tr.warped
    p1 = promote_trial(problem, t1)
    data["t1/image_grad"] = p1.image_grad
    lin = build_linearization(problem, p1)
    for term in ("total", "outer", "image", "proximity", "jd", "curl", "barrier"):
        data[f"grad/{term}"] = energy_gradient(lin, term=term)
    gF, gD, gE = outer_gradient_vectors(lin)
    data["outer_vectors"] = np.stack([gF, gD, gE])
    data["ggn_diag"] = barrier_ggn_diagonal(lin)
    rng = np.random.default_rng(3)
    p = rng.normal(size=3 * grid.n_free_scalar) * 0.01
    data["hvp_p"] = p
    data["ggn_hvp"] = barrier_ggn_hvp(lin, p)
    E = stable_energy_reduction(problem, t1, t2)
    F = stable_energy_reduction(problem, t1, t2, outer_only=True)
    EF = stable_energy_reductions(problem, t1, t2)
    data["reduction"] = np.array([E.actual, E.resolution, F.actual, F.resolution, EF[0].actual, EF[1].actual])
    # spline samples at interior off-node points (value + gradient)
    q = np.stack([rng.uniform(grid.axes[k][0], grid.axes[k][-1], 300) for k in range(3)], -1)
    s = sample_points(problem.sampler, q, with_gradient=True)
    data.update(sample_points=q, sample_value=s.value, sample_grad=s.gradient)
    # metric: shift alpha, diagonal, Poisson apply, equilibrated direction
    alpha = image_curvature_shift(problem, p1, 1.0)
    a, b = weights.lam + alpha, weights.mu / 2 + weights.nu / 2
    inverse = build_poisson_inverse(grid, a=a, b=b, metric="q1")
    rhs = rng.normal(size=3 * grid.n_free_scalar)
    data["poisson_ab"] = np.array([alpha, a, b, metric_diagonal(grid, a, b, "q1")])
    data["poisson_rhs"] = rhs
    data["poisson_apply"] = inverse.apply(rhs)
    data["poisson_denominator"] = inverse.denominator
    data["poisson7_apply"] = build_poisson_inverse(grid, a=a, b=b, metric="seven_point").apply(rhs)
    m = metric_diagonal(grid, a, b, "q1")
    d = data["ggn_diag"]
    scale = np.sqrt(m) / np.sqrt(d)
    node62 = node_min_jd(problem, p1)
    node73 = node_min_jd(problem, p1, extension_activation=0.25, stats={})
    r = affine_factors(node73, grid, 0.25)
    data["node_jd_t62"] = node62
    data["node_jd_t73"] = node73
    data["scale"] = scale * r
    g = data["grad/total"]
    data["direction"] = -EquilibratedInverse(inverse, scale * r).apply(g)
    # global closed27 cubic JD root along the direction (T66)
    for k, limit in enumerate((1.0, 40.0)):
        data[f"jd_root{k}"] = np.array([limit, np.nan if (rr := global_root_cpu(problem, p1, data["direction"],
                                                                                limit)["root"]) is None else rr])
    np.savez_compressed(os.path.join(out, "q1.npz"), **data)
    print("q1.npz: energy", data["t1/energy"], "node73 min", node73[1:-1, 1:-1, 1:-1].min(),
          "roots", data["jd_root0"], data["jd_root1"])


def make_seq(out, policy="image_shift_ggn_equilibrated_jd_affine_v1", name="seq.npz", seed=3, outer_steps=6,
             shape=(14, 13, 12), pair=None, theta0=None):
    """The reference's full certified proximal loop (CPU, default PG route; T62 metric or the native T73) on a small
    pair."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    from seq_vp_3d_b200.synthetic import blob_pair, default_weights
    from jd_curl.three_d.grid import make_grid_3d
    from jd_curl.three_d.problem import Weights3D, make_problem
    from jd_curl.three_d.feasibility import PrescreenCertificateConfig
    from jd_curl.three_d.sequential import solve_sequential, SequentialReuseConfig3D
    from jd_curl.three_d.solvers.poisson_gradient import ConservativePGConfig3D
    spacing = (1.0, 1.0, 1.0)
    fixed, moving, u_gt = blob_pair(shape, spacing, seed=seed) if pair is None else pair
    nz, ny, nx = shape
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=1., hy=1., hz=1., unit="mm")
    w = default_weights(shape, spacing)
    weights = Weights3D(lam=w["lam"], mu=w["mu"], nu=w["nu"], kappa=w["kappa"])
    config = PrescreenCertificateConfig(delta=0., max_depth=48, max_boxes=255, tile_size=65536, fallback_workers=2)
    problem = make_problem(grid=grid, fixed_image=fixed, moving_image=moving, u_ref=np.zeros(grid.shape + (3,)),
                           weights=weights, certificate_config=config, barrier_location="closed27_uniform",
                           barrier_activation=.05)
    inner = ConservativePGConfig3D(max_iterations=5, metric_policy=policy, resolution_exit=True)
    outer = SequentialReuseConfig3D(max_iterations=outer_steps, eta0=.01)
    theta = np.zeros(3 * grid.n_free_scalar) if theta0 is None else theta0(grid)
    res = solve_sequential(problem, theta, solver="pg", inner_config=inner, config=outer)
    rows = []
    attempts = []
    for k, row in enumerate(res.history):
        rows.append([k, row["outer_accepted"], row["inner_accepted_steps"], row["E_start"],
                     np.nan if row["E_candidate"] is None else row["E_candidate"], row["GF_before"],
                     np.nan if row["GF_candidate"] is None else row["GF_candidate"], row["forcing_target"]])
        for a in row["inner_history"]:
            attempts.append([k, a["iteration"], a["attempt"], a["tau"], a["accepted"],
                             np.nan if a["actual_reduction"] is None else a["actual_reduction"],
                             a["energy_base"], a["gradient_norm"]])
    e = res.final_state.energy
    np.savez_compressed(os.path.join(out, name), fixed=fixed, moving=moving, spacing=np.array(spacing),
                        weights=np.array([w["lam"], w["mu"], w["nu"], w["kappa"]]),
                        status=np.array(res.status), reason=np.array(res.reason), theta0=theta,
                        theta=res.final_state.theta, rows=np.array(rows, dtype=np.float64),
                        attempts=np.array(attempts, dtype=np.float64),
                        inner_status=np.array([r["inner_status"] for r in res.history]),
                        attempt_reasons=np.array([a["reason"] for r in res.history for a in r["inner_history"]]),
                        final_energy=np.array([e.image, e.proximity, e.jd, e.curl, e.barrier]),
                        gf=np.array([res.GF_initial, res.GF_final, res.GF_threshold]),
                        counts=np.array([res.counts["outer_accepted"], res.counts["inner_calls"]]))
    print(name + ":", res.status, res.reason, "outer", res.counts["outer_accepted"], "rows", len(rows),
          "attempts", len(attempts), "final E", e.total)


def make_t73(out):
    """Node JD measure with and without the T69/T73 face/interior extension (solvers/jd_affine.py:205) on a seeded
    field with strongly curved J, so that the extension lowers many cells' minima; plus the seeded pair's full
    loop with the native T73 metric policy."""
    from jd_curl.three_d.grid import make_grid_3d
    from jd_curl.three_d.problem import Weights3D, make_problem
    from jd_curl.three_d.feasibility import PrescreenCertificateConfig
    from jd_curl.three_d.solvers.jd_affine import node_min_jd
    shape, spacing = (16, 15, 14), (1.0, 0.9, 1.1)
    AMP = 0.2
    nz, ny, nx = shape
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=spacing[0], hy=spacing[1], hz=spacing[2], unit="mm")
    fixed, moving = seeded_images(shape, 11)
    rng = np.random.default_rng(12)
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    u = np.zeros(shape + (3,))
    for r, h in enumerate(spacing):
        for _ in range(4):
            k = rng.uniform(0.6, 1.6, size=3)
            u[..., r] += AMP * h * np.sin(k[0] * xx + k[1] * yy + k[2] * zz + rng.uniform(0, 6))
    u[[0, -1]] = 0.; u[:, [0, -1]] = 0.; u[:, :, [0, -1]] = 0.
    u = np.ascontiguousarray(u)
    weights = Weights3D(lam=0.1, mu=0.03, nu=0.03, kappa=0.002)
    config = PrescreenCertificateConfig(delta=0., max_depth=48, max_boxes=255, tile_size=65536, fallback_workers=2)
    problem = make_problem(grid=grid, fixed_image=fixed, moving_image=moving, u_ref=np.zeros(grid.shape + (3,)),
                           weights=weights, certificate_config=config, barrier_location="closed27_uniform",
                           barrier_activation=.05)

    class State:
        pass
    st = State()
    st.u = u
    node62 = node_min_jd(problem, st)
    stats = {}
    node73 = node_min_jd(problem, st, extension_activation=0.25, stats=stats)
    inner = node73[1:-1, 1:-1, 1:-1] < node62[1:-1, 1:-1, 1:-1]
    np.savez_compressed(os.path.join(out, "t73.npz"), u=u, spacing=np.array(spacing), node62=node62, node73=node73,
                        candidates=np.array(stats.get("candidates", 0)), lowered=np.array(stats.get("lowered_cells", 0)),
                        lowered_any=np.array(stats.get("lowered_cells_any", 0)))
    print("t73.npz: candidates", stats.get("candidates", 0), "lowered", stats.get("lowered_cells", 0), "lowered nodes",
          int(inner.sum()), "min", float(node62.min()), float(node73.min()))
    # the full loop with the native T73 policy on a pair whose ground truth compresses strongly (min JD >= 0.15),
    # so the face/interior extension meets candidate cells during the solve
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    from seq_vp_3d_b200 import synthetic as syn
    pshape, psp = (16, 15, 14), (1., 1., 1.)
    prng = np.random.default_rng(21)
    fixed2 = syn.blob_pair(pshape, psp, seed=21)[0]
    u_gt = syn._ground_truth(pshape, psp, prng, 3, 2.5, 2.2, 0.15)
    moving2 = syn._resample(fixed2, u_gt, psp)
    def start(grid):       # a certified start with a strong local compression (J ~ 0.12 near the centre)
        from jd_curl.three_d.boundary import restrict_free
        u0 = compressed_field(grid, 0.88, (8, 7, 7), 22, amp=0.05)
        return restrict_free(u0, grid)
    make_seq(out, policy="image_shift_ggn_equilibrated_jd_affine_v3", name="seq_t73.npz", outer_steps=8,
             shape=pshape, pair=(fixed2, moving2, u_gt), theta0=start)
