"""Generate the golden fixtures of the certified-registration hot path by running the reference CPU code.

This script is the only place that imports the reference (Zhaobh0620/seq_vp_3d, package ``jd_curl``).  It runs in a
container where the reference tree is mounted (its path is the required ``--reference`` argument), writes
small ``.npz`` files beside itself and records the library versions used.  Nothing at test or bench time reads the
reference: the fixtures are the frozen evidence.

The reference needs ``nibabel`` only for NIfTI I/O; a stub module is installed before the import.

Fixtures
--------
certificate.npz   per-cell edge-hull margins/flags, float Bernstein prescreen bounds, interval Bernstein fallback
                  arrays and certify_map records on several grids/fields (feasibility.py, compiled_enclosure.py,
                  certificate_prescreen.py, compiled_fallback.py).
cells.npz         standalone cells through fallback_arrays + _classify (subdivision verdicts, witnesses, budgets).
seq.npz           the reference's solve_sequential (default PG route, T62 metric) on a small seeded pair.
q1.npz            spline coefficients/samples, energy terms, gradients, GGN diagonal, GGN HVP, DST-I Poisson apply,
                  stable energy reductions of a small problem (residuals.py, linearization.py, poisson.py,
                  energy_comparison.py).

certificate_configs.npz  certify_map records of each certificate config class (bare, Adaptive, Enclosure,
                  CompiledFallback, Prescreen; the reference's defaults) and depth-first subdivision verdicts.
backend_signatures.json  parameter lists of the reference plug-in methods (backends/accelerated.py,
                  backends/hybrid.py) that the backend= adapter provides.
seq_config1.npz   the reference's solve_sequential on the 32^3 blob pair (seed 0) with the native T73 metric, 40
                  outer steps of 5 PG steps (the reference CPU route of the 32^3 float64 workload).

Run:  python tests/golden/make_golden.py --reference PATH [--only certificate,cells,q1,seq,t73,preopt,configs,signatures,config1]
"""
import argparse
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

STATUS = {"certified_feasible": 0, "infeasible": 1, "uncertain": 2}
REASONS = ["positive_enclosure_cover", "positive_bernstein_cover", "JACOBIAN_VIOLATION", "arithmetic_uncertain",
           "subdivision_budget", "NONFINITE_STATE", "NONZERO_BOUNDARY", "INVALID_DOMAIN", "unsupported_arithmetic",
           "sample_witness", "subdivision_witness", "box_budget", "depth_budget", "positive_edge_hull",
           "not_checked"]


def import_reference(path):
    sys.modules.setdefault("nibabel", types.ModuleType("nibabel"))
    sys.path.insert(0, path)
    import jd_curl  # noqa: F401
    return path


def versions():
    import scipy
    import numba
    return dict(numpy=np.__version__, scipy=scipy.__version__, numba=numba.__version__,
                python=sys.version.split()[0])


def record_array(result):
    """Flatten a FeasibilityResult into (int64[13], float64[6])."""
    nan = float("nan")
    ints = np.array([STATUS[result.status], REASONS.index(result.reason), result.n_cells_checked,
                     result.n_uncertain, result.n_infeasible, result.n_boxes, result.max_depth,
                     -1 if result.witness_cell is None else result.witness_cell,
                     getattr(result, "n_fast_cells", -1), getattr(result, "n_fallback_cells", -1),
                     getattr(result, "n_prescreen_cells", -1),
                     result.min_jd_lower_bound is not None, result.sampled_min_jd is not None], dtype=np.int64)
    point = result.witness_reference_point or (nan, nan, nan)
    flts = np.array([nan if result.min_jd_lower_bound is None else result.min_jd_lower_bound,
                     nan if result.min_margin_lower_bound is None else result.min_margin_lower_bound,
                     nan if result.sampled_min_jd is None else result.sampled_min_jd, *point], dtype=np.float64)
    return ints, flts


def fallback_digest(ok, arrays):
    """SHA-256 over the ok flags and, for ok cells, the five (27,) arrays in cell order (NaN rows skipped)."""
    import hashlib
    h = hashlib.sha256(np.ascontiguousarray(ok, dtype=np.uint8).tobytes())
    for c in np.flatnonzero(ok):
        h.update(np.ascontiguousarray(arrays[:, c], dtype=np.float64).tobytes())
    return h.hexdigest()


def counterexample_shifted(d, c):
    """T05-type cell x -> (x, y + 2(x-c)z, -2(x-c)y + dz): J = d + 4(x-c)^2, minimum at x = c."""
    cube = np.array([(x, y, z) for z in (0., 1.) for y in (0., 1.) for x in (0., 1.)])
    x, y, z = cube.T
    return np.stack((x, y + 2 * (x - c) * z, -2 * (x - c) * y + d * z), axis=-1) - cube


def inside(u, g):
    """Clip each component so that every node stays strictly inside the box: |u_r| <= 0.9 h_r dist_r."""
    nz, ny, nx = g.shape
    out = u.copy()
    for r, n in enumerate((nx, ny, nz)):
        i = np.arange(n)
        dist = np.minimum(i, n - 1 - i) * 0.9 * g.spacing[r]
        shape = [1, 1, 1]
        shape[2 - r] = n
        lim = dist.reshape(shape)
        out[..., r] = np.clip(out[..., r], -lim, lim)
    return np.ascontiguousarray(out)


def certificate_fields():
    """(name, grid kwargs, u) cases: the reference's own folding field plus seeded smooth/rough/hard fields."""
    from jd_curl.three_d.grid import make_grid_3d
    from jd_curl.three_d.backends.edge_hull_gpu import synthetic_folding_field, _counterexample
    from jd_curl.three_d.cell_q1 import cell_node_indices
    cases = []
    ga = dict(nx=9, ny=8, nz=7, hx=1.0, hy=1.25, hz=0.8)
    gb = dict(nx=14, ny=12, nz=11, hx=1.0, hy=1.0, hz=1.0)
    gc = dict(nx=17, ny=13, nz=12, hx=0.9, hy=1.1, hz=1.3)
    for name, kw in (("folding_a", ga), ("folding_b", gb), ("folding_c", gc)):
        g = make_grid_3d(**kw, unit="mm")
        cases.append((name, kw, synthetic_folding_field(g)))
    g = make_grid_3d(**ga, unit="mm")
    cases.append(("zero_a", ga, np.zeros(g.shape + (3,))))
    rng = np.random.default_rng(7)
    for name, kw, amp in (("smooth_b", gb, 0.15), ("rough_b", gb, 0.42), ("rough_c", gc, 0.33)):
        g = make_grid_3d(**kw, unit="mm")
        h = np.array(g.spacing)
        zz, yy, xx = np.meshgrid(*(np.linspace(0., 1., n) for n in g.shape), indexing="ij")
        u = np.stack([np.sin(np.pi * (k + 1) * xx) * np.sin(np.pi * yy) * np.sin(np.pi * (2 - k % 2) * zz)
                      for k in range(3)], axis=-1) * 0.8 * h
        u = u + rng.normal(size=g.shape + (3,)) * amp * h
        u[[0, -1]] = 0.; u[:, [0, -1]] = 0.; u[:, :, [0, -1]] = 0.
        cases.append((name, kw, inside(u, g)))
    # mild: certified through the edge hull and the prescreen (seeded; checked certified when generated)
    g = make_grid_3d(**gb, unit="mm")
    h = np.array(g.spacing)
    zz, yy, xx = np.meshgrid(*(np.linspace(0., 1., n) for n in g.shape), indexing="ij")
    u = np.stack([np.sin(np.pi * (k + 1) * xx) * np.sin(np.pi * yy) * np.sin(np.pi * (2 - k % 2) * zz)
                  for k in range(3)], axis=-1) * 0.5 * h
    u = u + np.random.default_rng(100).normal(size=g.shape + (3,)) * 0.12 * h
    u[[0, -1]] = 0.; u[:, [0, -1]] = 0.; u[:, :, [0, -1]] = 0.
    cases.append(("mild_b", gb, inside(u, g)))
    # hard: smooth field with embedded T05-type cells of small positive/negative interior JD
    g = make_grid_3d(**gc, unit="mm")
    h = np.array(g.spacing)
    u = np.zeros(g.shape + (3,))
    u += rng.normal(size=g.shape + (3,)) * 0.02 * h
    u[[0, -1]] = 0.; u[:, [0, -1]] = 0.; u[:, :, [0, -1]] = 0.
    flat = u.reshape(-1, 3)
    cz, cy, cx = g.cell_shape
    ds = [0.01, 1e-3, 1e-5, 0.2, 0.05, -1e-4, 3e-3, 1e-7]
    k = 0
    for z in range(2, cz - 2, 3):
        for y in range(2, cy - 2, 3):
            for x in range(2, cx - 2, 4):
                c = (z * cy + y) * cx + x
                nodes = cell_node_indices(g, slice(c, c + 1))[0]
                flat[nodes] = _counterexample(ds[k % len(ds)]) * h
                k += 1
    cases.append(("hard_c", gc, inside(u, g)))
    # hardpos: the same with positive interior minima only -> certified through prescreen, fallback, subdivision
    u = np.zeros(g.shape + (3,))
    u += rng.normal(size=g.shape + (3,)) * 0.01 * h
    u[[0, -1]] = 0.; u[:, [0, -1]] = 0.; u[:, :, [0, -1]] = 0.
    flat = u.reshape(-1, 3)
    ds = [0.02, 1e-3, 1e-5, 3e-3, 0.2, 0.05, 0.012, 1e-7]
    k = 0
    for z in range(2, cz - 2, 3):
        for y in range(2, cy - 2, 3):
            for x in range(2, cx - 2, 4):
                c = (z * cy + y) * cx + x
                nodes = cell_node_indices(g, slice(c, c + 1))[0]
                flat[nodes] = counterexample_shifted(ds[k % len(ds)], (0.5, 0.3, 0.77)[k % 3]) * h
                k += 1
    cases.append(("hardpos_c", gc, inside(u, g)))
    # blocks: constant blocks and exactly zero edge differences
    g = make_grid_3d(**ga, unit="mm")
    u = np.zeros(g.shape + (3,))
    u[2:5, 2:6, 1:4] = (0.3, -0.2, 0.1)
    u[1:3, 1:3, 5:8] = (-0.1, 0.25, 0.05)
    cases.append(("blocks_a", ga, u))
    # nonzero boundary and out-of-domain trial (early returns)
    g = make_grid_3d(**ga, unit="mm")
    u = np.zeros(g.shape + (3,)); u[0, 3, 3, 1] = 1e-3
    cases.append(("boundary_a", ga, u))
    u = np.zeros(g.shape + (3,)); u[3, 3, 3, 0] = 50.0
    cases.append(("domain_a", ga, u))
    u = np.zeros(g.shape + (3,)); u[3, 3, 3, 2] = np.nan
    cases.append(("nonfinite_a", ga, u))
    return cases


def make_certificate(out):
    from jd_curl.three_d.grid import make_grid_3d
    from jd_curl.three_d.feasibility import (PrescreenCertificateConfig, certify_map, _classify,
                                             _node_indices_for)
    from jd_curl.three_d.compiled_enclosure import parallel_margins
    from jd_curl.three_d.certificate_prescreen import prescreen_lower_bounds
    from jd_curl.three_d.compiled_fallback import fallback_arrays
    from jd_curl.three_d.cell_q1 import CellQ1Operators3D
    data = {}
    names = []
    for name, kw, u in certificate_fields():
        g = make_grid_3d(**kw, unit="mm")
        names.append(name)
        data[f"{name}/grid"] = np.array([kw["nx"], kw["ny"], kw["nz"]], dtype=np.int64)
        data[f"{name}/spacing"] = np.array([kw["hx"], kw["hy"], kw["hz"]])
        data[f"{name}/u"] = u
        finite = bool(np.all(np.isfinite(u)))
        for delta in (0.0, 0.01):
            tag = f"{name}/d{delta}"
            if finite:
                margin, flag = parallel_margins(u, g, delta)
                data[f"{tag}/margin"] = margin
                data[f"{tag}/flag"] = flag.astype(np.uint8)
            for tile in (64, 65536):
                cfg = PrescreenCertificateConfig(delta=delta, max_depth=48, max_boxes=255, tile_size=tile,
                                                 fallback_workers=2)
                ints, flts = record_array(certify_map(u, g, config=cfg))
                data[f"{tag}/t{tile}/record_i"] = ints
                data[f"{tag}/t{tile}/record_f"] = flts
            if not finite:
                continue
            # per-cell fallback arrays and subdivision verdicts (cell by cell, so one bad cell flags only itself)
            cells = np.arange(g.n_cells)
            verts = u.reshape(-1, 3)[_node_indices_for(g, cells)]
            n = g.n_cells
            ok = np.zeros(n, np.uint8)
            arrays = np.full((5, n, 27), np.nan)
            cls_i = np.full((n, 5), -1, np.int64)      # status, reason, boxes, depth, has_margin
            cls_f = np.full((n, 4), np.nan)            # margin, witness point xyz
            cfg = PrescreenCertificateConfig(delta=delta, max_depth=48, max_boxes=255, tile_size=65536,
                                             fallback_workers=1)
            for c in range(n):
                res = fallback_arrays(verts[c:c + 1], g.spacing, delta, np.geterr())
                if res is None:
                    continue
                ok[c] = 1
                p, coeff, samples = res
                arrays[0, c] = p.lo.ravel(); arrays[1, c] = p.hi.ravel()
                arrays[2, c] = coeff.lo.ravel(); arrays[3, c] = coeff.hi.ravel()
                arrays[4, c] = samples.ravel()
                if coeff.lo.min() > 0:
                    continue
                r = _classify(coeff[0], p[0], delta, float(samples[0].min()), cfg)
                cls_i[c] = (STATUS[r.status], REASONS.index(r.reason), r.n_boxes, r.max_depth,
                            r.min_margin_lower_bound is not None)
                cls_f[c, 0] = np.nan if r.min_margin_lower_bound is None else r.min_margin_lower_bound
                if r.witness_reference_point is not None:
                    cls_f[c, 1:] = r.witness_reference_point
            data[f"{tag}/fallback_ok"] = ok
            # full arrays for the classified cells and every 11th cell; a digest pins all of them
            classified = np.flatnonzero(cls_i[:, 0] >= 0)
            if len(classified) > 48:
                classified = np.random.default_rng(n).choice(classified, 48, replace=False)
            keep = np.union1d(classified, np.arange(0, n, 17))
            data[f"{tag}/fallback_keep"] = keep
            data[f"{tag}/fallback"] = arrays[:, keep]
            data[f"{tag}/fallback_sha256"] = np.array(fallback_digest(ok, arrays))
            data[f"{tag}/classify_i"] = cls_i
            data[f"{tag}/classify_f"] = cls_f
        if finite:
            table = CellQ1Operators3D(g, location="closed27_uniform").coefficients
            data[f"{name}/prescreen"] = prescreen_lower_bounds(u, g, table, np.arange(g.n_cells))
            data[f"{name}/closed27_D"] = np.asarray(table)
    data["names"] = np.array(names)
    data["reasons"] = np.array(REASONS)
    np.savez_compressed(os.path.join(out, "certificate.npz"), **data, versions=np.array(repr(versions())))
    print("certificate.npz:", len(names), "fields")


def make_configs(out):
    """certify_map records of the reference's certificate config family (bare, Adaptive, Enclosure, CompiledFallback,
    Prescreen, each with its own defaults) on every certificate field, plus the bare config's depth-first _classify
    verdicts on the standalone cells of cells.npz."""
    from jd_curl.three_d.grid import make_grid_3d
    from jd_curl.three_d import feasibility as F
    from jd_curl.three_d.compiled_fallback import fallback_arrays
    data = {}
    classes = ("CertificateConfig", "AdaptiveCertificateConfig", "EnclosureCertificateConfig",
               "CompiledFallbackCertificateConfig", "PrescreenCertificateConfig")
    names = []
    for name, kw, u in certificate_fields():
        g = make_grid_3d(**kw, unit="mm")
        names.append(name)
        for cls in classes:
            for delta in (0.0, 0.01):
                cfg = getattr(F, cls)(delta=delta)
                res = F.certify_map(u, g, config=cfg)
                ints, flts = record_array(res)
                tag = f"{name}/{cls}/d{delta}"
                data[f"{tag}/record_i"] = ints
                data[f"{tag}/record_f"] = flts
                data[f"{tag}/version"] = np.array(res.certificate_version)
    data["names"] = np.array(names)
    data["classes"] = np.array(classes)
    cells = np.load(os.path.join(out, "cells.npz"))
    verts, h = cells["vertices"], cells["spacing"]
    for delta in (0.0, 0.01):
        for depth, boxes in ((12, 255), (6, 40)):
            cfg = F.CertificateConfig(delta=delta, max_depth=depth, max_boxes=boxes)
            n = len(verts)
            cls_i = np.full((n, 5), -1, np.int64)
            cls_f = np.full((n, 4), np.nan)
            for c in range(n):
                res = fallback_arrays(verts[c:c + 1], h, delta, np.geterr())
                if res is None:
                    continue
                p, coeff, samples = res
                r = F._classify(coeff[0], p[0], delta, float(samples[0].min()), cfg)
                cls_i[c] = (STATUS[r.status], REASONS.index(r.reason), r.n_boxes, r.max_depth,
                            r.min_margin_lower_bound is not None)
                cls_f[c, 0] = np.nan if r.min_margin_lower_bound is None else r.min_margin_lower_bound
                if r.witness_reference_point is not None:
                    cls_f[c, 1:] = r.witness_reference_point
            tag = f"dfs/d{delta}/m{depth}_{boxes}"
            data[f"{tag}/classify_i"] = cls_i
            data[f"{tag}/classify_f"] = cls_f
            hist = np.bincount(cls_i[:, 1][cls_i[:, 1] >= 0], minlength=len(REASONS))
            print(tag, {REASONS[i]: int(c) for i, c in enumerate(hist) if c})
    np.savez_compressed(os.path.join(out, "certificate_configs.npz"), **data, versions=np.array(repr(versions())))
    print("certificate_configs.npz:", len(names), "fields x", len(classes), "config classes")


# the adapter methods of seq_vp_3d_b200.backend.B200Backend and the reference plug-in class each one mirrors
BACKEND_METHODS = {
    "evaluate_trial": "AcceleratedHybridBackend", "promote_trial": "AcceleratedHybridBackend",
    "gradient": "AcceleratedHybridBackend", "poisson": "AcceleratedHybridBackend",
    "diagonal": "HybridBackend", "diagonal_launch": "AcceleratedHybridBackend",
    "node_min_jd": "HybridBackend", "global_jd_root": "HybridBackend", "linearize": "AcceleratedHybridBackend",
    "stable_energy_reduction": "AcceleratedHybridBackend", "stable_energy_reductions": "AcceleratedHybridBackend",
    "outer_gradient_vectors": "AcceleratedHybridBackend", "outer_norms": "AcceleratedHybridBackend",
    "cpu_state": "AcceleratedHybridBackend",
}
POISSON_METHODS = ("apply", "prepare_equilibrated", "apply_equilibrated")


def make_signatures(out):
    """backend_signatures.json: the parameter lists (name, kind, default) of the reference plug-in's methods that
    the B200 backend adapter provides, read with inspect from the reference classes."""
    import inspect
    import json
    from jd_curl.three_d.backends import accelerated, hybrid

    def params(fn):
        fn = inspect.unwrap(fn)
        return [[p.name, str(p.kind), None if p.default is inspect.Parameter.empty else repr(p.default)]
                for p in inspect.signature(fn).parameters.values()]

    classes = dict(AcceleratedHybridBackend=accelerated.AcceleratedHybridBackend, HybridBackend=hybrid.HybridBackend)
    data = dict(backend={name: params(getattr(classes[cls], name)) for name, cls in BACKEND_METHODS.items()},
                poisson={name: params(getattr(hybrid._HostPoisson, name)) for name in POISSON_METHODS},
                source={name: cls for name, cls in BACKEND_METHODS.items()})
    with open(os.path.join(out, "backend_signatures.json"), "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    print("backend_signatures.json:", len(data["backend"]), "backend methods,", len(data["poisson"]), "Poisson methods")


def make_cells(out):
    """Standalone cells with tiny/negative interior JD, exercising every subdivision outcome."""
    from jd_curl.three_d.feasibility import PrescreenCertificateConfig, _classify
    from jd_curl.three_d.compiled_fallback import fallback_arrays
    from jd_curl.three_d.backends.edge_hull_gpu import _counterexample
    rng = np.random.default_rng(11)
    h = np.array([1.1, 0.9, 1.3])
    verts = []
    for k in range(420):
        kind = k % 7
        shift = 0.01 if (k // 7) % 2 else 0.0          # half of the cells sit just above delta = 0.01
        if kind == 0:
            d = shift + 10. ** rng.uniform(-9, -0.5) * (1 if rng.random() < .8 else -1)
            v = _counterexample(d)
        elif kind == 5:                       # minimum between the closed27 points: subdivision witnesses
            d = shift + 10. ** rng.uniform(-6, -2) * (1 if rng.random() < .6 else -1)
            v = counterexample_shifted(d, rng.uniform(0.05, 0.45))
        elif kind == 6:                       # very small positive minimum off the sample points: budgets
            v = counterexample_shifted(shift + 10. ** rng.uniform(-12, -7), rng.uniform(0.05, 0.95))
        elif kind == 1:                       # axis-permuted counterexample: psi(w) = Q phi(Q^T w)
            d = shift + 10. ** rng.uniform(-7, -1)
            cube = np.array([(x, y, z) for z in (0., 1.) for y in (0., 1.) for x in (0., 1.)])
            phi = _counterexample(d) + cube
            perm = rng.permutation(3)
            v = np.empty((8, 3))
            for a, w in enumerate(cube):
                src = np.empty(3)
                src[perm] = w                  # Q^T w
                b = int(src[0] + 2 * src[1] + 4 * src[2])
                v[a] = phi[b][perm] - w        # Q phi(Q^T w) - w
        elif kind == 2:                       # random near-degenerate affine+bilinear map
            v = rng.normal(size=(8, 3)) * 0.45
        elif kind == 3:                       # counterexample plus small noise
            v = (_counterexample(shift + 10. ** rng.uniform(-6, -1))
                 + rng.normal(size=(8, 3)) * 10. ** rng.uniform(-6, -2))
        else:                                 # strongly folded
            v = rng.normal(size=(8, 3)) * 0.8
        verts.append(v * h)
    verts = np.ascontiguousarray(np.array(verts))
    data = dict(vertices=verts, spacing=h)
    for delta in (0.0, 0.01):
        for depth, boxes in ((48, 255), (6, 40)):
            cfg = PrescreenCertificateConfig(delta=delta, max_depth=depth, max_boxes=boxes, tile_size=65536,
                                             fallback_workers=1)
            n = len(verts)
            ok = np.zeros(n, np.uint8)
            arrays = np.full((5, n, 27), np.nan)
            cls_i = np.full((n, 5), -1, np.int64)
            cls_f = np.full((n, 4), np.nan)
            for c in range(n):
                res = fallback_arrays(verts[c:c + 1], h, delta, np.geterr())
                if res is None:
                    continue
                ok[c] = 1
                p, coeff, samples = res
                arrays[:, c] = (p.lo.ravel(), p.hi.ravel(), coeff.lo.ravel(), coeff.hi.ravel(), samples.ravel())
                r = _classify(coeff[0], p[0], delta, float(samples[0].min()), cfg)
                cls_i[c] = (STATUS[r.status], REASONS.index(r.reason), r.n_boxes, r.max_depth,
                            r.min_margin_lower_bound is not None)
                cls_f[c, 0] = np.nan if r.min_margin_lower_bound is None else r.min_margin_lower_bound
                if r.witness_reference_point is not None:
                    cls_f[c, 1:] = r.witness_reference_point
            tag = f"d{delta}/m{depth}_{boxes}"
            data[f"{tag}/ok"] = ok
            data[f"{tag}/arrays"] = arrays
            data[f"{tag}/classify_i"] = cls_i
            data[f"{tag}/classify_f"] = cls_f
            hist = np.bincount(cls_i[:, 1][cls_i[:, 1] >= 0], minlength=len(REASONS))
            print(tag, {REASONS[i]: int(c) for i, c in enumerate(hist) if c})
    np.savez_compressed(os.path.join(out, "cells.npz"), **data, versions=np.array(repr(versions())))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference tree (the directory holding jd_curl)")
    ap.add_argument("--only", default="certificate,cells,q1,seq,t73,preopt")
    args = ap.parse_args()
    import_reference(args.reference)
    only = set(args.only.split(","))
    if "certificate" in only:
        make_certificate(HERE)
    if "cells" in only:
        make_cells(HERE)
    if "q1" in only:
        from q1_golden import make_q1      # second half of this generator (energy, gradient, DST)
        make_q1(HERE)
    if "seq" in only:
        from q1_golden import make_seq     # the full certified proximal loop on a small pair
        make_seq(HERE)
    if "t73" in only:
        from q1_golden import make_t73     # node JD measure with the T69/T73 face/interior extension
        make_t73(HERE)
    if "preopt" in only:
        from preopt_golden import make_preopt   # the float32 pyramid pre-optimizer and its pieces
        make_preopt(HERE)
    if "signatures" in only:
        make_signatures(HERE)
    if "configs" in only:
        make_configs(HERE)
    if "config1" in only:
        from q1_golden import make_seq     # the 32^3 blob pair, native T73 metric, 40 outer steps
        make_seq(HERE, policy="image_shift_ggn_equilibrated_jd_affine_v3", name="seq_config1.npz", seed=0,
                 outer_steps=40, shape=(32, 32, 32))


if __name__ == "__main__":
    main()
