"""The reference's own certified loop with this library plugged in as its backend= (B200Backend).

jd_curl.three_d.sequential.solve_sequential (installed under baseline/_ref) runs unchanged; every trial evaluation,
promotion, gradient, Poisson apply, GGN diagonal, node JD measure, comparison and outer norm goes through
seq_vp_3d_b200.backend.B200Backend.  Its decisions must be those of the reference's CPU run of the same problem
(goldens seq.npz: T62 metric, 6 outer steps from u = 0; seq_t73.npz: native T73 metric, 8 outer steps from a
certified compressed start; seq_config1.npz: the 32^3 blob pair, T73, 40 outer steps): identical statuses, accepted flags, attempt counts and reasons; step sizes within 1e-6.
Skipped where the reference package is not installed."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, installed_reference

pytestmark = pytest.mark.gpu

CASES = [("seq.npz", "image_shift_ggn_equilibrated_jd_affine_v1", 6),
         ("seq_t73.npz", "image_shift_ggn_equilibrated_jd_affine_v3", 8),
         ("seq_config1.npz", "image_shift_ggn_equilibrated_jd_affine_v3", 40)]


@pytest.fixture(scope="module", params=CASES, ids=["t62", "t73", "blob32_40outer"])
def run(request):
    if installed_reference() is None:
        pytest.skip("reference package not installed under baseline/_ref")
    from jd_curl.three_d.grid import make_grid_3d
    from jd_curl.three_d.problem import Weights3D, make_problem
    from jd_curl.three_d.feasibility import PrescreenCertificateConfig
    from jd_curl.three_d.sequential import solve_sequential, SequentialReuseConfig3D
    from jd_curl.three_d.solvers.poisson_gradient import ConservativePGConfig3D
    from seq_vp_3d_b200.backend import B200Backend
    name, policy, outer = request.param
    d = np.load(os.path.join(GOLDEN, name))
    nz, ny, nx = d["fixed"].shape
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=1., hy=1., hz=1., unit="mm")
    lam, mu, nu, kappa = (float(v) for v in d["weights"])
    config = PrescreenCertificateConfig(delta=0., max_depth=48, max_boxes=255, tile_size=65536, fallback_workers=2)
    problem = make_problem(grid=grid, fixed_image=d["fixed"], moving_image=d["moving"],
                           u_ref=np.zeros(grid.shape + (3,)), weights=Weights3D(lam=lam, mu=mu, nu=nu, kappa=kappa),
                           certificate_config=config, barrier_location="closed27_uniform", barrier_activation=.05)
    backend = B200Backend()
    theta0 = np.array(d["theta0"]) if "theta0" in d.files else np.zeros(3 * grid.n_free_scalar)
    res = solve_sequential(problem, theta0, solver="pg",
                           inner_config=ConservativePGConfig3D(max_iterations=5, metric_policy=policy,
                                                               resolution_exit=True),
                           config=SequentialReuseConfig3D(max_iterations=outer, eta0=.01), backend=backend)
    return d, res, backend


def test_reference_loop_decisions_through_backend(run):
    d, res, backend = run
    assert res.status == str(d["status"])
    rows = d["rows"]
    assert len(res.history) == len(rows)
    for row, ref in zip(res.history, rows):
        assert bool(row["outer_accepted"]) == bool(ref[1])
        assert row["inner_accepted_steps"] == int(ref[2])
    assert [r["inner_status"] for r in res.history] == [str(s) for s in d["inner_status"]]
    assert res.counts["outer_accepted"] == int(d["counts"][0])
    assert backend.comparison_counts["gpu"] > 0          # the comparisons ran on the device


def test_reference_loop_attempts_through_backend(run):
    d, res, _ = run
    att = d["attempts"]
    mine = [(k, a["iteration"], a["attempt"], a["tau"], a["accepted"], a["energy_base"], a["gradient_norm"])
            for k, r in enumerate(res.history) for a in r["inner_history"]]
    assert len(mine) == len(att)
    assert [a["reason"] for r in res.history for a in r["inner_history"]] == [str(x) for x in d["attempt_reasons"]]
    for m, ref in zip(mine, att):
        assert m[:3] == tuple(int(v) for v in ref[:3])
        assert bool(m[4]) == bool(ref[4])
        assert abs(m[3] - ref[3]) <= 1e-6 * abs(ref[3])
        assert abs(m[5] - ref[6]) <= 1e-9 * abs(ref[6])
        assert abs(m[6] - ref[7]) <= 1e-6 * abs(ref[7])


def test_reference_loop_final_state_through_backend(run):
    d, res, _ = run
    ref = d["theta"]
    assert np.linalg.norm(res.final_state.theta - ref) <= 1e-6 * np.linalg.norm(ref)
    assert res.final_state.certificate.status == "certified_feasible"
