"""Pre-optimizer fixture (preopt.npz): the reference's float32 pyramid pre-optimizer run on the CPU (torch) for a small
seeded pair, plus its pieces: the pre-objective terms and autograd gradient at a seeded state (float32 and float64),
downsample_array and prolong_displacement outputs.  Imported by make_golden.py after the reference is on sys.path."""
import os

import numpy as np


def make_preopt(out):
    import sys
    import torch
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    from seq_vp_3d_b200.synthetic import blob_pair
    from jd_curl.three_d.grid import make_grid_3d
    from jd_curl.three_d.preopt import PreoptConfig, preoptimize, _pre_energy_tensors
    from jd_curl.three_d.multiresolution import four_level_grids, prolong_displacement
    from jd_curl.three_d.nifti import downsample_array
    torch.set_num_threads(4)
    shape = (38, 36, 34)                 # (nz, ny, nx): every level keeps >= 5 nodes per axis
    spacing = (1.0, 1.1, 0.9)
    fixed, moving, _ = blob_pair(shape, spacing, seed=7)
    nz, ny, nx = shape
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=spacing[0], hy=spacing[1], hz=spacing[2], unit="mm")
    data = dict(spacing=np.array(spacing), shape=np.array(shape), pair_seed=np.array(7))   # the pair: blob_pair(seed=7)
    grids = four_level_grids(grid)
    for lv in range(3):
        f, g, _ = downsample_array(fixed, grid, grids[lv].shape)
        data[f"down{lv}"] = f
        data[f"down{lv}_spacing"] = np.array(g.spacing)
    # pre-objective at a seeded interior state on level 2 (float32 and float64 autograd)
    lg = grids[2]
    F = data["down2"].astype(np.float32).astype(np.float64)      # the float32 images both precisions then see
    M = downsample_array(moving, grid, lg.shape)[0].astype(np.float32).astype(np.float64)
    rng = np.random.default_rng(8)
    u_int = (rng.normal(size=(3,) + lg.interior_shape) * 0.3).astype(np.float32)
    h = tuple(float(s) for s in lg.spacing)
    for dt, tag in ((torch.float32, "f32"), (torch.float64, "f64")):
        u = torch.tensor(u_int, dtype=dt, requires_grad=True)
        total, det, dterm, geo, flo, cur = _pre_energy_tensors(u, torch.tensor(F, dtype=dt), torch.tensor(M, dtype=dt), h,
                                                              .3, 1e-3, 10., .2)
        grad, = torch.autograd.grad(total, u)
        data[f"pre_terms_{tag}"] = np.array([float(dterm), float(geo), float(flo), float(cur), float(det.min()),
                                             float(total)])
        if tag == "f64":
            data["pre_grad_f64"] = grad.detach().numpy()
    data.update(pre_F=F.astype(np.float32), pre_M=M.astype(np.float32), pre_u=u_int, pre_spacing=np.array(h))
    # Q1 transfer of a seeded zero-face field from level 1 to level 2
    src, dst = grids[1], grids[2]
    w = np.zeros(src.shape + (3,))
    w[1:-1, 1:-1, 1:-1] = rng.normal(size=tuple(n - 2 for n in src.shape) + (3,)) * 0.4
    data["prolong_in"] = w
    data["prolong_out"] = prolong_displacement(w, src, dst)
    # the whole pre-optimizer (CPU), a few iterations per level, field smoothing on, no time cap
    config = PreoptConfig(iterations=(6, 6, 4, 3), lr=.5, cap=.5, sigma_grad=1., sigma_field=1.,
                          mu=(1., 1., .01, .003), alpha=(1e-3, 1e-3, 1e-3, 0.), kappa_pre=10., j0=.2, seconds=1e9)
    u_mm, record = preoptimize(fixed, moving, grid, config=config, device="cpu")
    data["preopt_u"] = u_mm.astype(np.float32)      # float32 precision is the comparison's scale anyway
    data["preopt_first"] = np.array([[lv["first"][k] for k in ("data", "geometry", "floor", "curvature", "min_det")]
                                     for lv in record["levels"]])
    data["preopt_last"] = np.array([[lv["last"][k] for k in ("data", "geometry", "floor", "curvature", "min_det")]
                                    for lv in record["levels"]])
    data["preopt_cap_hits"] = np.array(record["cap_hits"])
    np.savez_compressed(os.path.join(out, "preopt.npz"), **data)
    print("preopt.npz: levels", [lv["shape_zyx"] for lv in record["levels"]], "cap hits", record["cap_hits"],
          "max |u|", float(np.abs(u_mm).max()), "last total", [lv["last"]["total"] for lv in record["levels"]])
