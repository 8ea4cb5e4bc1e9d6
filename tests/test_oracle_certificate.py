"""The C oracle of the certificate against the golden fixtures generated by the reference (CPU, no GPU)."""
import hashlib

import numpy as np
import pytest

from conftest import all_vertices, same_bits, same_bits_nan
from oracle import cert


def _names(g):
    return [str(n) for n in g["names"]]


def test_oracle_margins_prescreen(cert_golden):
    g = cert_golden
    for name in _names(g):
        u, h = g[f"{name}/u"], g[f"{name}/spacing"]
        if not np.all(np.isfinite(u)):
            continue
        n = (u.shape[0] - 1) * (u.shape[1] - 1) * (u.shape[2] - 1)
        assert same_bits_nan(cert.prescreen(u, h, np.arange(n), threads=4), g[f"{name}/prescreen"]), name
        assert same_bits(cert.closed27_table(h), g[f"{name}/closed27_D"]), name
        for d in (0.0, 0.01):
            m, f = cert.edge_hull(u, h, d, threads=4)
            gm, gf = g[f"{name}/d{d}/margin"], g[f"{name}/d{d}/flag"].astype(bool)
            assert np.array_equal(f, gf), (name, d)
            assert same_bits(m[~gf], gm[~gf]), (name, d)


def test_oracle_fallback_and_classify(cert_golden):
    g = cert_golden
    for name in _names(g):
        u, h = g[f"{name}/u"], g[f"{name}/spacing"]
        if not np.all(np.isfinite(u)):
            continue
        verts = all_vertices(u)
        for d in (0.0, 0.01):
            tag = f"{name}/d{d}"
            ok = np.zeros(len(verts), np.uint8)
            full = np.full((5, len(verts), 27), np.nan)
            ci, cf = g[f"{tag}/classify_i"], g[f"{tag}/classify_f"]
            for c, v in enumerate(verts):
                res = cert.fallback_cell(v, h, d)
                ok[c] = res[0]
                if not res[0]:
                    continue
                full[:, c] = res[1:]
                if ci[c, 0] >= 0:
                    r = cert.classify(res[3], res[4], res[1], res[2], d)
                    assert (r["status"], r["reason"], r["boxes"], r["depth"], r["margin"] is not None) == tuple(ci[c])
                    if r["margin"] is not None:
                        assert same_bits(r["margin"], cf[c, 0])
                    if r["witness"] is not None:
                        assert same_bits(r["witness"], cf[c, 1:])
            assert np.array_equal(ok, g[f"{tag}/fallback_ok"]), tag
            digest = hashlib.sha256(ok.tobytes())
            for c in np.flatnonzero(ok):
                digest.update(np.ascontiguousarray(full[:, c]).tobytes())
            assert digest.hexdigest() == str(g[f"{tag}/fallback_sha256"]), tag
            keep = g[f"{tag}/fallback_keep"]
            assert same_bits_nan(full[:, keep], g[f"{tag}/fallback"]), tag


def test_oracle_certify_map_records(cert_golden):
    g = cert_golden
    for name in _names(g):
        u, h = g[f"{name}/u"], g[f"{name}/spacing"]
        for d in (0.0, 0.01):
            for tile in (64, 65536):
                ri, rf = cert.certify_map(u, h, d, tile_size=tile)
                assert np.array_equal(ri, g[f"{name}/d{d}/t{tile}/record_i"]), (name, d, tile)
                assert same_bits_nan(rf, g[f"{name}/d{d}/t{tile}/record_f"]), (name, d, tile)


@pytest.mark.parametrize("delta", [0.0, 0.01])
@pytest.mark.parametrize("budget", [(48, 255), (6, 40)])
def test_oracle_standalone_cells(cells_golden, delta, budget):
    g = cells_golden
    V, h = g["vertices"], g["spacing"]
    tag = f"d{delta}/m{budget[0]}_{budget[1]}"
    for k in range(len(V)):
        res = cert.fallback_cell(V[k], h, delta)
        assert res[0] == bool(g[f"{tag}/ok"][k])
        if not res[0]:
            continue
        assert same_bits(np.array(res[1:]), g[f"{tag}/arrays"][:, k])
        r = cert.classify(res[3], res[4], res[1], res[2], delta, *budget)
        assert (r["status"], r["reason"], r["boxes"], r["depth"], r["margin"] is not None) == \
            tuple(g[f"{tag}/classify_i"][k])
        if r["margin"] is not None:
            assert same_bits(r["margin"], g[f"{tag}/classify_f"][k, 0])
        if r["witness"] is not None:
            assert same_bits(r["witness"], g[f"{tag}/classify_f"][k, 1:])


def expected_record(ints, hull, prescreen):
    """The reference's plain FeasibilityResult (bare and Adaptive configs) has no stage counts and its
    EnclosureFeasibilityResult no prescreen count; the golden writes -1 there, the record structure here 0."""
    ints = np.array(ints)
    absent = slice(8, 11) if not hull else slice(10, 11) if not prescreen else slice(0, 0)
    assert np.all(ints[absent] == -1)
    ints[absent] = 0
    return ints


def test_oracle_config_family_records(cert_golden, configs_golden):
    """The C oracle reproduces certify_map's record for every config class of the reference (bare: whole-cell
    Bernstein with depth-first subdivision; Adaptive: lowest bound first; the Enclosure family with the hull)."""
    from conftest import CONFIG_EXECUTIONS
    g, c = cert_golden, configs_golden
    for name in _names(c):
        u, h = g[f"{name}/u"], g[f"{name}/spacing"]
        for cls in c["classes"]:
            hull, pre, dfs, depth, tile = CONFIG_EXECUTIONS[str(cls)]
            for d in (0.0, 0.01):
                tag = f"{name}/{cls}/d{d}"
                ri, rf = cert.certify_map(u, h, d, max_depth=depth, tile_size=tile, hull=hull, prescreen=pre,
                                          depth_first=dfs)
                assert np.array_equal(ri, expected_record(c[f"{tag}/record_i"], hull, pre)), (tag, ri)
                assert same_bits_nan(rf, c[f"{tag}/record_f"]), (tag, rf)


def test_oracle_depth_first_classify(cells_golden, configs_golden):
    """Depth-first subdivision verdicts of the bare CertificateConfig on the standalone cells."""
    verts, h = cells_golden["vertices"], cells_golden["spacing"]
    for d in (0.0, 0.01):
        for depth, boxes in ((12, 255), (6, 40)):
            tag = f"dfs/d{d}/m{depth}_{boxes}"
            ci, cf = configs_golden[f"{tag}/classify_i"], configs_golden[f"{tag}/classify_f"]
            for k, v in enumerate(verts):
                res = cert.fallback_cell(v, h, d)
                if not res[0]:
                    assert ci[k, 0] < 0
                    continue
                r = cert.classify(res[3], res[4], res[1], res[2], d, depth, boxes, depth_first=True)
                assert (r["status"], r["reason"], r["boxes"], r["depth"], r["margin"] is not None) == tuple(ci[k]), \
                    (tag, k)
                if r["margin"] is not None:
                    assert same_bits(r["margin"], cf[k, 0])
                if r["witness"] is not None:
                    assert same_bits(r["witness"], cf[k, 1:])
