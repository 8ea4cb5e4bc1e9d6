"""End-to-end: the device-resident certified proximal loop against the reference's own solve_sequential on the same
seeded pairs (golden seq.npz: conservative PG route with the T62 metric, 6 outer steps from u = 0; seq_t73.npz: the
native T73 metric, 8 outer steps from a certified start with a strong local compression).

Discrete decisions (statuses, accepted flags, attempt counts) must be identical; the continuous trajectory agrees
to the precision that the 1e-12 kernel parity propagates through 30 BB2 steps."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


# (fixture, metric policy, outer steps): the T62 metric from u = 0, and the native T73 metric from a certified start
# with a strong local compression
CASES = [("seq.npz", "image_shift_ggn_equilibrated_jd_affine_v1", 6),
         ("seq_t73.npz", "image_shift_ggn_equilibrated_jd_affine_v3", 8),
         # the 32^3 blob pair (seed 0) with the native T73 metric and 40 outer steps: the reference's CPU route of
         # the 32^3 float64 workload
         ("seq_config1.npz", "image_shift_ggn_equilibrated_jd_affine_v3", 40)]


@pytest.fixture(scope="module", params=CASES, ids=["t62", "t73", "blob32_40outer"])
def run(request):
    from seq_vp_3d_b200.grid import make_grid_3d
    from seq_vp_3d_b200.solver import PGConfig3D, Registration, SequentialConfig3D, solve_sequential
    name, policy, outer = request.param
    d = np.load(os.path.join(GOLDEN, name))
    nz, ny, nx = d["fixed"].shape
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=1., hy=1., hz=1., unit="mm")
    lam, mu, nu, kappa = (float(v) for v in d["weights"])
    reg = Registration(grid, d["fixed"], d["moving"], lam=lam, mu=mu, nu=nu, kappa=kappa)
    theta0 = torch.from_numpy(np.ascontiguousarray(d["theta0"])).cuda() if "theta0" in d.files else None
    res = solve_sequential(reg, theta0, config=SequentialConfig3D(max_iterations=outer),
                           inner_config=PGConfig3D(metric_policy=policy))
    return d, res


def test_outer_decisions_match_reference(run):
    d, res = run
    assert res.status == str(d["status"])
    rows = d["rows"]
    assert len(res.history) == len(rows)
    for row, ref in zip(res.history, rows):
        assert row["accepted"] == bool(ref[1])
        assert row["inner_accepted_steps"] == int(ref[2])
    assert [r["inner_status"] for r in res.history] == [str(s) for s in d["inner_status"]]
    assert res.counts["outer_accepted"] == int(d["counts"][0])
    assert res.certified


def test_inner_attempts_match_reference(run):
    d, res = run
    att = d["attempts"]
    mine = [(k, a["iteration"], a["attempt"], a["tau"], a["accepted"], a["actual"], a["energy_base"],
             a["gradient_norm"]) for k, r in enumerate(res.history) for a in r["inner_history"]]
    assert len(mine) == len(att)
    reasons = [a["reason"] for r in res.history for a in r["inner_history"]]
    assert reasons == [str(x) for x in d["attempt_reasons"]]
    for m, ref in zip(mine, att):
        assert m[:3] == tuple(int(v) for v in ref[:3])
        assert bool(m[4]) == bool(ref[4])
        assert abs(m[3] - ref[3]) <= 1e-6 * abs(ref[3])            # step sizes
        assert abs(m[6] - ref[6]) <= 1e-9 * abs(ref[6])            # base energies
        assert abs(m[7] - ref[7]) <= 1e-6 * abs(ref[7])            # gradient norms


def test_final_state_matches_reference(run):
    d, res = run
    theta = res.final_state.theta.cpu().numpy()
    ref = d["theta"]
    assert np.linalg.norm(theta - ref) <= 1e-6 * np.linalg.norm(ref)
    e = res.final_state.energy
    assert abs(e[0] + e[4] - (d["final_energy"][0] + d["final_energy"][4])) <= 1e-8 * d["final_energy"][0]
    gf = d["gf"]
    assert abs(res.GF_initial - gf[0]) <= 1e-10 * gf[0]
    assert abs(res.GF_final - gf[1]) <= 1e-6 * gf[1]
