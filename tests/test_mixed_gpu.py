"""The mixed form (float32 search direction, float64 energies, decisions and certificate) against the plain float64
form on the same inputs: the errors of the gradient terms, the GGN diagonal, the Poisson apply and the
preconditioned direction are stated here as tested bounds, and a whole certified solve in the mixed form ends
certified with the plain form's final MSE within 1% (the north star's equal-MSE condition).

Stated bounds (relative, normwise): gradients 1e-5, GGN diagonal 1e-5, DST-I Poisson apply and direction 1e-5.
float32 carries 6e-8 relative per operation; the Q1 sums over 27 points and the 3 x 2 DST passes stay well inside.
"""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
BOUND = 1e-5


def rel(a, b):
    a, b = a.detach().double().cpu().numpy().ravel(), b.detach().double().cpu().numpy().ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def pairs():
    from seq_vp_3d_b200.grid import make_grid_3d
    from seq_vp_3d_b200.pair import DevicePair
    d = np.load(os.path.join(GOLDEN, "q1.npz"))
    nx, ny, nz = (int(v) for v in d["grid"])
    hx, hy, hz = (float(v) for v in d["spacing"])
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=hx, hy=hy, hz=hz, unit="mm")
    lam, mu, nu, kappa = (float(v) for v in d["weights"])
    kw = dict(lam=lam, mu=mu, nu=nu, kappa=kappa)
    plain = DevicePair(grid, d["fixed"], d["moving"], d["u_ref"], **kw)
    mixed = DevicePair(grid, d["fixed"], d["moving"], d["u_ref"], **kw, precision="mixed")
    u1 = torch.from_numpy(d["u1"]).cuda()
    w1, g1 = plain.warp(u1, with_gradient=True)
    return d, plain, mixed, u1, w1, g1


@pytest.mark.parametrize("term", ["total", "outer", "jd", "curl", "barrier"])
def test_gradient_terms(pairs, term):
    d, plain, mixed, u1, w1, g1 = pairs
    ref = plain.gradient(u1, w1, g1, term)
    got = mixed.gradient(u1, w1, g1, term)
    assert rel(got, ref) <= BOUND, (term, rel(got, ref))


def test_outer_triple_and_ggn(pairs):
    d, plain, mixed, u1, w1, g1 = pairs
    for got, ref in zip(mixed.outer_gradients(u1, w1, g1), plain.outer_gradients(u1, w1, g1)):
        assert rel(got, ref) <= BOUND
    assert rel(mixed.ggn_diagonal(u1, g1), plain.ggn_diagonal(u1, g1)) <= BOUND


def test_poisson_and_direction(pairs):
    d, plain, mixed, u1, w1, g1 = pairs
    alpha, a, b, m = d["poisson_ab"]
    rhs = torch.from_numpy(d["poisson_rhs"]).cuda()
    assert rel(mixed.poisson_apply(a, b, rhs), plain.poisson_apply(a, b, rhs)) <= BOUND
    s = torch.from_numpy(d["scale"]).cuda()
    g = torch.from_numpy(d["grad/total"]).cuda()
    ref = plain.poisson_apply(a, b, g, scale=s, sign=-1.)
    got = mixed.poisson_apply(a, b, g, scale=s, sign=-1.)
    assert rel(got, ref) <= BOUND


def test_energies_stay_float64(pairs):
    d, plain, mixed, u1, w1, g1 = pairs
    tp, bp = plain.energy(u1, w1)
    tm, bm = mixed.energy(u1, w1)
    assert np.array_equal(tp, tm) and bp == bm


def test_mixed_solve_matches_plain_mse():
    from seq_vp_3d_b200.grid import make_grid_3d
    from seq_vp_3d_b200.solver import PGConfig3D, Registration, SequentialConfig3D, solve_sequential
    from seq_vp_3d_b200.synthetic import blob_pair, default_weights
    shape, h = (24, 22, 20), (1., 1., 1.)
    fixed, moving, _ = blob_pair(shape, h, seed=11)
    nz, ny, nx = shape
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=1., hy=1., hz=1., unit="mm")
    out = {}
    for form in ("plain", "mixed"):
        reg = Registration(grid, fixed, moving, **default_weights(shape, h), precision=form)
        res = solve_sequential(reg, config=SequentialConfig3D(max_iterations=8), inner_config=PGConfig3D())
        assert res.certified
        out[form] = res.final_mse
    assert abs(out["mixed"] - out["plain"]) <= .01 * out["plain"], out


def test_screened_trial(pairs):
    """The mixed form's float32 energy screen (svp_trial_energy_screened) against the float64 one-pass trial on the
    same base and trial (the fixture's barrier is active): warped image, image gradient, the image, proximity and
    barrier terms, the violation count, the activity mask and the F difference are bitwise the float64 call's; the
    JD and curl terms carry float32 rounding within 1e-5 relative, and the screened E difference lies within the
    returned band of the float64 one (both directions: u1 -> u2 and u2 -> u1).  The barrier term and F difference
    come from a float64 closed27 sweep in a different kernel: equal within 1e-12 relative (contraction order)."""
    d, plain, mixed, u1, w1, g1 = pairs
    u2 = torch.from_numpy(d["u2"]).cuda()
    w2, _ = plain.warp(u2)
    for (ua, wa, ub) in ((u1, w1, u2), (u2, w2, u1)):
        ref = plain.trial_energy(ua, wa, ub)
        got = plain.trial_energy_screened(ua, wa, ub)
        assert torch.equal(got[0], ref[0]) and torch.equal(got[1], ref[1]) and torch.equal(got[5], ref[5])
        rt, gt = ref[2], got[2]
        assert got[3] == ref[3]
        assert rt[0] == gt[0] and rt[1] == gt[1]                            # image, proximity
        assert abs(rt[4] - gt[4]) <= 1e-12 * abs(rt[4])                     # barrier
        for k in (2, 3):                                                    # JD, curl
            assert abs(gt[k] - rt[k]) <= 1e-5 * abs(rt[k]), (k, gt[k], rt[k])
        assert abs(got[4][1] - ref[4][1]) <= 1e-12 * (abs(rt[0]) + abs(rt[4]))   # F = image + barrier
        band = got[6]
        assert band > 0 and abs(got[4][0] - ref[4][0]) <= band, (got[4][0], ref[4][0], band)


def test_screened_difference(pairs):
    """svp_energy_difference_screened (the outer commit's screened comparison of two evaluated states) against the
    float64 svp_energy_difference_masked, both directions: dF (image + barrier, float64 in both; the barrier sums run
    in a different kernel) within 1e-12 relative, dE within the returned band, and the band is the screened trial's
    for the same pair of states (the same float32 sums)."""
    d, plain, mixed, u1, w1, g1 = pairs
    u2 = torch.from_numpy(d["u2"]).cuda()
    w2, _ = plain.warp(u2)
    for (ua, wa, ub, wb) in ((u1, w1, u2, w2), (u2, w2, u1, w1)):
        ref = plain.energy_difference(ua, wa, ub, wb)
        dE, dF, band = plain.energy_difference_screened(ua, wa, ub, wb)
        scale = abs(ref[1]) + abs(plain.energy(ub, wb)[0][4])
        assert abs(dF - ref[1]) <= 1e-12 * scale, (dF, ref[1])
        assert band > 0 and abs(dE - ref[0]) <= band, (dE, ref[0], band)
        assert band == plain.trial_energy_screened(ua, wa, ub)[6]
