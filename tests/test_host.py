"""Host-side pieces that need no GPU: the per-grid weight total, the boundary taper's host form, and the bench's
phase split."""
import numpy as np

from seq_vp_3d_b200.grid import make_grid_3d
from seq_vp_3d_b200.preopt import boundary_taper


def test_node_weight_total_cached_and_exact():
    grid = make_grid_3d(nx=23, ny=19, nz=17, hx=1.0, hy=1.1, hz=0.9, unit="mm")
    direct = float(np.sum(grid.node_weights(), dtype=np.longdouble))
    assert grid.node_weight_total() == direct
    assert grid.node_weight_total() == direct          # second call: the cached value
    # the total of the trapezoid weights is the box volume
    extent = np.prod([a[-1] - a[0] for a in grid.axes])
    assert abs(direct - extent) <= 1e-12 * extent


def test_boundary_taper_host_form():
    """preopt.py:617: weights min(min(k, n-1-k) / L, 1) per axis, multiplied; faces go to zero, the interior beyond L
    keeps the field."""
    grid = make_grid_3d(nx=14, ny=12, nz=11, hx=1., hy=1., hz=1., unit="mm")
    rng = np.random.default_rng(3)
    u = rng.normal(size=grid.shape + (3,))
    out, w = boundary_taper(u, grid, L=4)
    assert w.shape == grid.shape and np.all(w[[0, -1]] == 0) and np.all(w[:, [0, -1]] == 0)
    assert np.all(w[:, :, [0, -1]] == 0) and w[5, 5, 6] == 1.
    k = np.arange(grid.shape[2])
    assert np.array_equal(w[5, 5], np.minimum(np.minimum(k, grid.shape[2] - 1 - k) / 4., 1.))
    assert np.array_equal(out, w[..., None] * u)


def test_bench_phase_split():
    """One timed pair's host-clock phases: the loop's remainder after its kernels' device time (the pre-optimizer's
    kernels are not the loop's)."""
    import bench
    phase = dict(preopt_s=.2, transfer_s=.01, certified_loop_s=10.)
    timers = {"cell_trial_kernel": (10, 4000.), "prescreen_kernel": (5, 1000.), "pre_data_kernel": (3, 500.)}
    out = bench.phase_summary(phase, timers)
    assert abs(out["preopt_s"] - .2) < 1e-12 and abs(out["certified_loop_s"] - 10.) < 1e-12
    assert abs(out["loop_kernels_s"] - 5.) < 1e-12
    assert abs(out["loop_host_gap_s"] - 5.) < 1e-12
    assert bench.phase_summary(None, timers) is None


def test_cpu_extrapolation_formula():
    """The CPU baseline's seconds per pair: outer x (sum of count x slab seconds x cell-plane scale, the DST-I apply
    counted at full size)."""
    import bench
    t = bench.CpuTable.__new__(bench.CpuTable)
    t.outer, t.scale = 10, 4.
    t.t = {k: 1. for k in bench.PER_OUTER}
    per_outer = sum(bench.PER_OUTER[k] * (1. if k == "direction" else 4.) for k in bench.PER_OUTER)
    assert abs(t.seconds_per_pair() - 10 * per_outer) < 1e-9


def test_grid_ids_equal_the_reference():
    """Grid ids are the reference's (grid.py:49 make_grid_3d) for the same arguments: the ids below were produced by
    the reference's own factory, so certificates and states carry interchangeable grid ids."""
    import pytest
    from seq_vp_3d_b200.grid import InputValidationError, make_grid_3d
    cases = [(dict(nx=9, ny=8, nz=7, hx=1.0, hy=1.25, hz=0.8, unit="mm"),
              "620fe16f0e74b7f6179f254a2fc6cd63b404c299d6ab8b81ecbfca3b1ccc1f1d"),
             (dict(nx=160, ny=192, nz=224, hx=1., hy=1., hz=1., unit="mm"),
              "51c2d3c616b2f6ffbc725eedf59a1547299d87150f2970fb670369a24d85b675"),
             (dict(nx=17, ny=13, nz=12, hx=.9, hy=1.1, hz=1.3, x0=-3.5, y0=2, z0=1e-3, unit="um"),
              "c71764ed3546beb1bd2539b5da42ac304856beefc164a178ee07f16cdb77c3a7")]
    for kw, gid in cases:
        g = make_grid_3d(**kw)
        assert g.grid_id == gid
        assert g.shape == (kw["nz"], kw["ny"], kw["nx"]) and g.omega == kw["hx"] * kw["hy"] * kw["hz"]
    for bad in (dict(nx=4), dict(hx=0.), dict(hx=float("inf")), dict(unit=" "), dict(nx=True)):
        kw = dict(nx=9, ny=8, nz=7, hx=1., hy=1., hz=1., unit="mm")
        kw.update(bad)
        with pytest.raises(InputValidationError):
            make_grid_3d(**kw)
