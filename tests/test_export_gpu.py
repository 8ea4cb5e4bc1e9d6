"""Final-state export (final_native.npz / final_native.json / summary.json, the reference's output formats) and the
independent CPU re-certification of the exported field: the C restatement of the reference's certifier (oracle/)
proves the exported u with the same record the device certificate gave."""
import json

import numpy as np
import pytest

from conftest import same_bits_nan

pytestmark = pytest.mark.gpu


def test_export_and_cpu_recertification(tmp_path):
    from oracle import cert as oc
    from seq_vp_3d_b200.export import export_final
    from seq_vp_3d_b200.grid import make_grid_3d
    from seq_vp_3d_b200.solver import PGConfig3D, Registration, SequentialConfig3D, solve_sequential
    from seq_vp_3d_b200.synthetic import blob_pair, default_weights
    from test_certificate_gpu import record_of
    shape, h = (20, 18, 16), (1., 1., 1.)
    fixed, moving, _ = blob_pair(shape, h, seed=5)
    nz, ny, nx = shape
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=1., hy=1., hz=1., unit="mm")
    reg = Registration(grid, fixed, moving, **default_weights(shape, h))
    res = solve_sequential(reg, config=SequentialConfig3D(max_iterations=3), inner_config=PGConfig3D())
    assert res.certified
    rec = export_final(res, str(tmp_path))
    data = np.load(tmp_path / "final_native.npz")
    u = data["u"]
    assert u.shape == shape + (3,) and data["warped"].shape == shape
    assert np.array_equal(u, res.final_state.u.cpu().numpy())
    meta = json.load(open(tmp_path / "final_native.json"))
    assert meta["sha256"] == rec["sha256"] and meta["certificate"]["status"] == "certified_feasible"
    summary = json.load(open(tmp_path / "summary.json"))
    assert summary["status"] == res.status and summary["final_mse"] == res.final_mse
    # independent CPU proof of the exported bytes (the reference's certifier restated in C)
    oi, of = oc.certify_map(u, h, 0.0)
    gi, gf = record_of(res.final_state.certificate)
    assert np.array_equal(oi, gi) and same_bits_nan(of, gf)
