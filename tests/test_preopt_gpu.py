"""The float32 pyramid pre-optimizer (an uncertified initializer) against the reference's own float32 run on the CPU
(golden preopt.npz): the pyramid images, the Q1 transfer, the pre-objective and its gradient, and the whole
four-level run; then the certified hand-over to the native solve.

Tolerances: the pyramid image and transfer are float64 (1e-12); the pre-objective is float32 with a different
summation order (terms 1e-5 relative, gradient 1e-4 relative L2 against the float64 autograd gradient: the bounds
the reference itself puts on its analytic gradient, preopt_grad.py:38-39); the whole run compounds float32 rounding
through 19 Adam steps over four levels (field within 2e-3 of its largest displacement)."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fx():
    from seq_vp_3d_b200.grid import make_grid_3d
    from seq_vp_3d_b200.synthetic import blob_pair
    d = np.load(os.path.join(GOLDEN, "preopt.npz"))
    nz, ny, nx = (int(v) for v in d["shape"])
    hx, hy, hz = (float(v) for v in d["spacing"])
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=hx, hy=hy, hz=hz, unit="mm")
    fixed, moving, _ = blob_pair((nz, ny, nx), (hx, hy, hz), seed=int(d["pair_seed"]))
    return d, grid, fixed, moving


def test_pyramid_images_and_transfer(fx):
    from seq_vp_3d_b200 import preopt as P
    d, grid, fixed, moving = fx
    grids = P.four_level_grids(grid)
    f = torch.from_numpy(fixed).cuda()
    for lv in range(3):
        assert np.allclose(grids[lv].spacing, d[f"down{lv}_spacing"], rtol=0, atol=1e-15)
        got = P.downsample(f, grid, grids[lv]).cpu().numpy()
        ref = d[f"down{lv}"]
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    got = P.prolong_displacement(torch.from_numpy(d["prolong_in"]).cuda(), grids[1], grids[2]).cpu().numpy()
    assert np.array_equal(got, d["prolong_out"])          # the same operations in the same order


def test_pre_objective_and_gradient(fx):
    from seq_vp_3d_b200 import preopt as P
    from seq_vp_3d_b200.grid import grid_from_shape
    d, grid, fixed, moving = fx
    F, M, u = (torch.from_numpy(np.ascontiguousarray(d[k])).cuda() for k in ("pre_F", "pre_M", "pre_u"))
    lg = grid_from_shape(F.shape, tuple(d["pre_spacing"]))
    terms, grad = P.pre_energy_grad(F, M, lg, u, .3, 1e-3, 10., .2)
    ref = d["pre_terms_f64"]
    got = np.array([terms[k] for k in P.TERMS])
    assert np.all(np.abs(got - ref) <= 1e-5 * np.maximum(np.abs(ref), 1e-3)), (got, ref)
    g = grad.double().cpu().numpy()
    gr = d["pre_grad_f64"]
    assert np.linalg.norm(g - gr) <= 1e-4 * np.linalg.norm(gr)


def test_whole_pyramid_run(fx):
    from seq_vp_3d_b200 import preopt as P
    d, grid, fixed, moving = fx
    config = P.PreoptConfig(iterations=(6, 6, 4, 3), lr=.5, cap=.5, sigma_grad=1., sigma_field=1.,
                            mu=(1., 1., .01, .003), alpha=(1e-3, 1e-3, 1e-3, 0.), kappa_pre=10., j0=.2, seconds=1e9)
    u, record = P.preoptimize(fixed, moving, grid, config)
    got = u.cpu().numpy()
    ref = d["preopt_u"].astype(np.float64)
    scale = np.abs(ref).max()
    assert scale > .3
    assert np.abs(got - ref).max() <= 2e-3 * scale, np.abs(got - ref).max() / scale
    for lv, rec in enumerate(record["levels"]):
        first = np.array([rec["first"][k] for k in ("data", "geometry", "floor", "curvature", "min_det")])
        assert np.allclose(first, d["preopt_first"][lv], rtol=1e-3, atol=1e-4), (lv, first, d["preopt_first"][lv])
    assert np.all(got[[0, -1]] == 0) and np.all(got[:, [0, -1]] == 0) and np.all(got[:, :, [0, -1]] == 0)


def test_certified_handover_and_native_solve(fx):
    """Taper + transfer give a certified field; the native solve starts from it and ends certified."""
    from seq_vp_3d_b200 import preopt as P
    from seq_vp_3d_b200.synthetic import default_weights
    d, grid, fixed, moving = fx
    config = P.PreoptConfig(iterations=(6, 6, 4, 3), lr=.5, cap=.5, sigma_grad=1., sigma_field=1.,
                            mu=(1., 1., .01, .003), alpha=(1e-3, 1e-3, 1e-3, 0.), kappa_pre=10., j0=.2, seconds=1e9)
    w = default_weights(grid.shape, grid.spacing)
    res, record = P.register_pair(fixed, moving, grid, w, preopt=config, outer=2)
    assert record["transfer"]["status"] == "ready"
    assert res.certified
    # the native solve starts at the transferred field and only accepts certified decreases from there
    assert record["transfer"]["accepted_alpha"] in P.TRANSFER_ALPHAS
    assert res.final_mse <= res.native_mse
