"""The numpy Q1 oracle against the golden fixture generated by the reference (CPU)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import q1 as Q

TOL = 1e-13   # oracle vs reference: different BLAS/op order, same binary64 algorithm


def rel(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def fx():
    d = np.load(os.path.join(GOLDEN, "q1.npz"))
    nx, ny, nz = d["grid"]
    g = Q.make_grid((nz, ny, nx), tuple(d["spacing"]))
    lam, mu, nu, kappa = d["weights"]
    P = Q.make_problem(g, d["fixed"], d["moving"], d["u_ref"], lam, mu, nu, kappa)
    w1, ig1 = Q.warp(P, d["u1"], True)
    return d, g, P, w1, ig1


def test_spline(fx):
    d, g, P, w1, ig1 = fx
    assert rel(P.coeff, d["spline_c"]) < TOL
    for k in range(3):
        assert np.array_equal(Q.not_a_knot_knots(g.axes[::-1][k]), d[f"knots{k}"])
    v, gr = Q.spline_sample(P.coeff, g, d["sample_points"])
    assert rel(v, d["sample_value"]) < TOL and rel(gr, d["sample_grad"]) < TOL
    assert rel(w1, d["t1/warped"]) < TOL and rel(ig1, d["t1/image_grad"]) < TOL


def test_energy_terms(fx):
    d, g, P, w1, ig1 = fx
    e = Q.energy(P, d["u1"])
    ref = d["t1/energy"][:5]
    assert np.all(np.abs(e - ref) <= 1e-13 * np.abs(ref)), (e, ref)
    assert ref[4] > 0      # the localized barrier is active in this fixture


@pytest.mark.parametrize("term", ["total", "outer", "image", "proximity", "jd", "curl", "barrier"])
def test_gradients(fx, term):
    d, g, P, w1, ig1 = fx
    assert rel(Q.gradient(P, d["u1"], w1, ig1, term), d[f"grad/{term}"]) < TOL


def test_ggn(fx):
    d, g, P, w1, ig1 = fx
    assert rel(Q.ggn_diagonal(P, d["u1"], ig1), d["ggn_diag"]) < TOL
    assert rel(Q.ggn_hvp(P, d["u1"], ig1, d["hvp_p"]), d["ggn_hvp"]) < TOL


def test_stable_reduction(fx):
    d, g, P, w1, ig1 = fx
    w2, _ = Q.warp(P, d["u2"])
    dE, dF = Q.differences(P, d["u1"], w1, d["u2"], w2)
    red = d["reduction"]
    assert abs(float(-dE) - red[0]) < 0.1 * red[1] and abs(float(-dF) - red[2]) < 0.1 * red[3]


def test_poisson_and_metric(fx):
    d, g, P, w1, ig1 = fx
    lam, mu, nu, _ = d["weights"]
    alpha = Q.image_curvature_shift(P, ig1)
    a, b = lam + alpha, mu / 2 + nu / 2
    assert abs(alpha - d["poisson_ab"][0]) <= 1e-14 * alpha
    assert Q.metric_diagonal(g, a, b) == pytest.approx(d["poisson_ab"][3], rel=1e-15)
    assert rel(Q.poisson_apply(g, a, b, d["poisson_rhs"]), d["poisson_apply"]) < TOL
    assert rel(Q.poisson_apply(g, a, b, d["poisson_rhs"], "seven_point"), d["poisson7_apply"]) < TOL
    m = Q.metric_diagonal(g, a, b)
    scale = np.sqrt(m) / np.sqrt(d["ggn_diag"]) * Q.affine_factors(d["node_jd_t73"])
    assert rel(scale, d["scale"]) < TOL
    assert rel(-scale * Q.poisson_apply(g, a, b, scale * d["grad/total"]), d["direction"]) < TOL


def test_node_measure_face_interior_extension():
    """The oracle's T69/T73 estimator against the reference's node_min_jd(extension_activation=.25) (t73.npz)."""
    d = np.load(os.path.join(GOLDEN, "t73.npz"))
    u = d["u"]
    nz, ny, nx = u.shape[:3]
    g = Q.make_grid((nz, ny, nx), tuple(d["spacing"]))
    z = np.zeros((nz, ny, nx))
    P = Q.make_problem(g, z, z, np.zeros_like(u), .1, .03, .03, .002)
    inner = (slice(1, -1),) * 3
    n62 = Q.node_min_jd(P, u)
    n73, ncand = Q.node_min_jd(P, u, .25)
    assert rel(n62[inner], d["node62"][inner]) < TOL
    assert ncand == int(d["candidates"]) and np.sum(n73[inner] < n62[inner]) > 0
    err = np.abs(n73[inner] - d["node73"][inner]) / np.abs(d["node73"][inner])
    assert err.max() < 1e-12, err.max()


def test_node_measure_and_root(fx):
    d, g, P, w1, ig1 = fx
    n62 = Q.node_min_jd(P, d["u1"])
    assert rel(n62[1:-1, 1:-1, 1:-1], d["node_jd_t62"][1:-1, 1:-1, 1:-1]) < TOL
    for k in range(2):
        lim, root = d[f"jd_root{k}"]
        r = Q.global_jd_root(P, d["u1"], d["direction"], lim)
        assert (r is None and np.isnan(root)) or r == pytest.approx(root, rel=1e-12)
