"""GPU certificate parity: every margin, flag, bound, interval array and verdict bit-identical to the reference
(golden fixtures) and to the C oracle on larger seeded fields."""
import hashlib

import numpy as np
import pytest
import torch

from conftest import all_vertices, same_bits, same_bits_nan
from oracle import cert as oc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def svp():
    from seq_vp_3d_b200 import certificate
    assert torch.cuda.is_available()
    return certificate


def grid_of(g, name):
    from seq_vp_3d_b200.grid import make_grid_3d
    nx, ny, nz = (int(v) for v in g[f"{name}/grid"])
    hx, hy, hz = (float(v) for v in g[f"{name}/spacing"])
    return make_grid_3d(nx=nx, ny=ny, nz=nz, hx=hx, hy=hy, hz=hz, unit="mm")


def names(g):
    return [str(n) for n in g["names"]]


def test_margins_bitwise(svp, cert_golden):
    g = cert_golden
    for name in names(g):
        u = g[f"{name}/u"]
        if not np.all(np.isfinite(u)):
            continue
        grid = grid_of(g, name)
        for d in (0.0, 0.01):
            m, f = svp.parallel_margins(u, grid, d)
            gm, gf = g[f"{name}/d{d}/margin"], g[f"{name}/d{d}/flag"].astype(bool)
            assert np.array_equal(f, gf), (name, d)
            assert same_bits(m[~gf], gm[~gf]), (name, d)


def test_prescreen_bitwise(svp, cert_golden):
    g = cert_golden
    for name in names(g):
        u = g[f"{name}/u"]
        if not np.all(np.isfinite(u)):
            continue
        grid = grid_of(g, name)
        low = svp.prescreen_lower_bounds(u, grid, g[f"{name}/closed27_D"], np.arange(grid.n_cells))
        assert same_bits_nan(low, g[f"{name}/prescreen"]), name


def test_fallback_arrays_bitwise(svp, cert_golden):
    g = cert_golden
    for name in names(g):
        u = g[f"{name}/u"]
        if not np.all(np.isfinite(u)):
            continue
        verts = all_vertices(u)
        for d in (0.0, 0.01):
            tag = f"{name}/d{d}"
            ok, *arrs = (t.cpu().numpy() for t in svp.fallback_arrays_device(verts, g[f"{name}/spacing"], d))
            assert np.array_equal(ok, g[f"{tag}/fallback_ok"]), tag
            full = np.stack(arrs)
            digest = hashlib.sha256(ok.astype(np.uint8).tobytes())
            for c in np.flatnonzero(ok):
                digest.update(np.ascontiguousarray(full[:, c]).tobytes())
            assert digest.hexdigest() == str(g[f"{tag}/fallback_sha256"]), tag


@pytest.mark.parametrize("delta", [0.0, 0.01])
@pytest.mark.parametrize("budget", [(48, 255), (6, 40)])
def test_classify_standalone_cells(svp, cells_golden, delta, budget):
    g = cells_golden
    V, h = g["vertices"], g["spacing"]
    tag = f"d{delta}/m{budget[0]}_{budget[1]}"
    ok, plo, phi, clo, chi, smp = (t.cpu().numpy() for t in svp.fallback_arrays_device(V, h, delta))
    assert np.array_equal(ok, g[f"{tag}/ok"])
    sel = np.flatnonzero(ok)
    assert same_bits(np.stack([plo, phi, clo, chi, smp])[:, sel], g[f"{tag}/arrays"][:, sel])
    verdicts = svp.classify_cells(clo[sel], chi[sel], plo[sel], phi[sel], delta, *budget)
    gi, gf = g[f"{tag}/classify_i"], g[f"{tag}/classify_f"]
    for k, r in zip(sel, verdicts):
        assert (r["status"], r["reason"], r["boxes"], r["depth"], r["margin"] is not None) == tuple(gi[k]), k
        if r["margin"] is not None:
            assert same_bits(r["margin"], gf[k, 0]), k
        if r["witness"] is not None:
            assert same_bits(r["witness"], gf[k, 1:]), k


def record_of(res):
    from seq_vp_3d_b200.certificate import REASONS, STATUS
    ints = np.array([STATUS.index(res.status), REASONS.index(res.reason), res.n_cells_checked, res.n_uncertain,
                     res.n_infeasible, res.n_boxes, res.max_depth,
                     -1 if res.witness_cell is None else res.witness_cell, res.n_fast_cells,
                     res.n_fallback_cells, res.n_prescreen_cells, res.min_jd_lower_bound is not None,
                     res.sampled_min_jd is not None], dtype=np.int64)
    nan = float("nan")
    pt = res.witness_reference_point or (nan, nan, nan)
    flts = np.array([nan if res.min_jd_lower_bound is None else res.min_jd_lower_bound,
                     nan if res.min_margin_lower_bound is None else res.min_margin_lower_bound,
                     nan if res.sampled_min_jd is None else res.sampled_min_jd, *pt])
    return ints, flts


def test_certify_map_records(svp, cert_golden):
    g = cert_golden
    for name in names(g):
        u, grid = g[f"{name}/u"], grid_of(g, name)
        for d in (0.0, 0.01):
            for tile in (64, 65536):
                cfg = svp.PrescreenCertificateConfig(delta=d, max_depth=48, max_boxes=255, tile_size=tile)
                ri, rf = record_of(svp.certify_map(u, grid, config=cfg))
                if ri[0] == 0 or ri[2] == 0:      # early returns report n_uncertain = n_cells as the reference does
                    pass
                assert np.array_equal(ri, g[f"{name}/d{d}/t{tile}/record_i"]), (name, d, tile, ri)
                assert same_bits_nan(rf, g[f"{name}/d{d}/t{tile}/record_f"]), (name, d, tile, rf)


def seeded_field(shape, spacing, amp, seed):
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    h = np.array(spacing)
    zz, yy, xx = np.meshgrid(*(np.linspace(0., 1., n) for n in shape), indexing="ij")
    u = np.stack([np.sin(np.pi * (k + 1) * xx) * np.sin(np.pi * yy) * np.sin(np.pi * zz) for k in range(3)], -1)
    u = u * 0.6 * h + rng.normal(size=shape + (3,)) * amp * h
    u[[0, -1]] = 0.; u[:, [0, -1]] = 0.; u[:, :, [0, -1]] = 0.
    for r, n in enumerate((nx, ny, nz)):
        i = np.arange(n)
        lim = (np.minimum(i, n - 1 - i) * 0.9 * h[r]).reshape([n if k == 2 - r else 1 for k in range(3)])
        u[..., r] = np.clip(u[..., r], -lim, lim)
    return np.ascontiguousarray(u)


@pytest.mark.parametrize("amp,seed", [(0.05, 1), (0.14, 2), (0.22, 3), (0.3, 4)])
def test_certify_map_matches_oracle_larger(svp, amp, seed):
    from seq_vp_3d_b200.grid import make_grid_3d
    shape, h = (36, 41, 47), (0.9, 1.0, 1.2)
    grid = make_grid_3d(nx=shape[2], ny=shape[1], nz=shape[0], hx=h[0], hy=h[1], hz=h[2], unit="mm")
    u = seeded_field(shape, h, amp, seed)
    for d in (0.0, 0.01):
        for tile in (4096, 65536):
            cfg = svp.PrescreenCertificateConfig(delta=d, max_depth=48, tile_size=tile)
            ri, rf = record_of(svp.certify_map(u, grid, config=cfg))
            oi, of = oc.certify_map(u, h, d, tile_size=tile)
            assert np.array_equal(ri, oi), (amp, d, tile, ri, oi)
            assert same_bits_nan(rf, of), (amp, d, tile, rf, of)
        m, f = svp.parallel_margins(u, grid, d)
        om, of_ = oc.edge_hull(u, h, d, threads=8)
        assert np.array_equal(f, of_) and same_bits(m, om)


def test_margins_full_size_tile_rule(svp):
    """Margins at 96^3 against the oracle, plus the flag rule on a field with one overflowing node."""
    from seq_vp_3d_b200.grid import make_grid_3d
    shape, h = (96, 96, 96), (1.0, 1.0, 1.0)
    grid = make_grid_3d(nx=96, ny=96, nz=96, hx=1., hy=1., hz=1., unit="mm")
    u = seeded_field(shape, h, 0.2, 9)
    u[40, 50, 60] = (1e300, -1e300, 1e300)
    m, f = svp.parallel_margins(u, grid, 0.0)
    om, of_ = oc.edge_hull(u, h, 0.0, threads=8)
    assert np.array_equal(f, of_) and f.sum() == 8
    assert same_bits(m[~f], om[~f])


def test_config_family_records(svp, cert_golden, configs_golden):
    """certify_map under each certificate config class at the reference's own defaults: the bare class (whole-cell
    Bernstein, depth-first subdivision), Adaptive (lowest bound first), Enclosure, CompiledFallback and Prescreen;
    every record field and the certificate version equal the reference's."""
    from conftest import CONFIG_EXECUTIONS
    from seq_vp_3d_b200.grid import make_grid_3d
    from test_oracle_certificate import expected_record
    c = configs_golden
    for name in names(c):
        u = cert_golden[f"{name}/u"]
        grid = grid_of(cert_golden, name)
        for cls in c["classes"]:
            hull, pre, _, _, _ = CONFIG_EXECUTIONS[str(cls)]
            for d in (0.0, 0.01):
                tag = f"{name}/{cls}/d{d}"
                res = svp.certify_map(u, grid, config=getattr(svp, str(cls))(delta=d))
                ri, rf = record_of(res)
                assert np.array_equal(ri, expected_record(c[f"{tag}/record_i"], hull, pre)), (tag, ri)
                assert same_bits_nan(rf, c[f"{tag}/record_f"]), (tag, rf)
                assert res.certificate_version == str(c[f"{tag}/version"]), tag


def test_depth_first_classify(svp, cells_golden, configs_golden):
    """The bare CertificateConfig's depth-first subdivision (svp_classify_cells_policy) on the standalone cells."""
    verts, h = cells_golden["vertices"], cells_golden["spacing"]
    for d in (0.0, 0.01):
        ok, plo, phi, clo, chi, _ = (t.cpu().numpy() for t in svp.fallback_arrays_device(verts, h, d))
        sel = np.flatnonzero(ok)
        for depth, boxes in ((12, 255), (6, 40)):
            tag = f"dfs/d{d}/m{depth}_{boxes}"
            ci, cf = configs_golden[f"{tag}/classify_i"], configs_golden[f"{tag}/classify_f"]
            got = svp.classify_cells(clo[sel], chi[sel], plo[sel], phi[sel], d, depth, boxes, depth_first=True)
            for k, r in zip(sel, got):
                assert (r["status"], r["reason"], r["boxes"], r["depth"], r["margin"] is not None) == tuple(ci[k]), \
                    (tag, k)
                if r["margin"] is not None:
                    assert same_bits(r["margin"], cf[k, 0])
                if r["witness"] is not None:
                    assert same_bits(r["witness"], cf[k, 1:])


# ---------------------------------------------------------------------------------------------- directed rounding
def test_directed_margins_are_valid_and_tighter(svp, cert_golden):
    """The directed-rounding edge hull: wherever neither arithmetic flags a cell, its margin is at least the
    reference's (every directed end lies inside the nearest-plus-one-ulp end), and it flags no cell the reference
    does not."""
    g = cert_golden
    tighter = 0
    for name in names(g):
        u, grid = g[f"{name}/u"], grid_of(g, name)
        if not np.all(np.isfinite(u)):
            continue
        for d in (0.0, 0.01):
            m, f = svp.parallel_margins(u, grid, d)
            md, fd = svp.parallel_margins(u, grid, d, directed=True)
            assert not np.any(fd & ~f), (name, d)
            both = ~f & ~fd
            assert np.all(md[both] >= m[both]), (name, d)
            tighter += int(np.sum(md[both] > m[both]))
    assert tighter > 0


def test_directed_verdicts_cell_by_cell(svp, cells_golden):
    """Verdict by verdict on the 420 standalone cells (every subdivision outcome of the reference), both deltas, both
    budgets: every cell the reference decides (certified or infeasible) gets the same verdict in the directed
    arithmetic; an undecided directed verdict where the reference decided counts as a failure.  Cells the reference
    leaves uncertain may be decided."""
    verts, h = cells_golden["vertices"], cells_golden["spacing"]
    decided_more = 0
    for d in (0.0, 0.01):
        ok, plo, phi, clo, chi, _ = (t.cpu().numpy() for t in svp.fallback_arrays_device(verts, h, d, directed=True))
        for depth, boxes in ((48, 255), (6, 40)):
            tag = f"d{d}/m{depth}_{boxes}"
            ref_ok, ci = cells_golden[f"{tag}/ok"].astype(bool), cells_golden[f"{tag}/classify_i"]
            assert np.all(ok.astype(bool) | ~ref_ok), tag      # finite reference arrays stay finite
            sel = np.flatnonzero(ok)
            got = svp.classify_cells(clo[sel], chi[sel], plo[sel], phi[sel], d, depth, boxes, directed=True)
            for k, r in zip(sel, got):
                if not ref_ok[k]:
                    continue
                ref_status = int(ci[k, 0])
                if ref_status in (0, 1):
                    assert r["status"] == ref_status, (tag, k, r, ci[k])
                elif r["status"] != 2:
                    decided_more += 1
    print("directed decisions where the reference was uncertain:", decided_more)


def test_directed_certify_map_records(svp, cert_golden):
    """Whole-map certificates in the directed arithmetic on the golden fields (PrescreenCertificateConfig, both
    deltas): the reference's decided statuses are reproduced, and a certified map's lower bound is at least the
    reference's."""
    g = cert_golden
    for name in names(g):
        u, grid = g[f"{name}/u"], grid_of(g, name)
        for d in (0.0, 0.01):
            cfg = svp.PrescreenCertificateConfig(delta=d, max_depth=48, max_boxes=255, tile_size=65536)
            res = svp.certify_map(u, grid, config=cfg, directed=True)
            ri, rf = g[f"{name}/d{d}/t65536/record_i"], g[f"{name}/d{d}/t65536/record_f"]
            if ri[0] in (0, 1):
                assert svp.STATUS.index(res.status) == ri[0], (name, d, res.status)
            if ri[0] == 0 and np.isfinite(rf[0]):
                assert res.min_jd_lower_bound >= rf[0], (name, d)
