"""GPU parity of the Q1 energy path: spline, energy terms, gradients, GGN, stable differences, DST-I Poisson,
node JD measure and JD root against the reference (golden q1.npz) and the numpy oracle on larger seeded problems.

Tolerance (the plain FP64 form's contract): 1e-12 relative, normwise for vectors and per term for energies.
The vector kernels that the solver's decisions depend on (axpy, step bound) are checked bit for bit."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, same_bits
from oracle import q1 as Q

pytestmark = pytest.mark.gpu
TOL = 1e-12


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    a, b = np.ravel(a), np.ravel(b)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def gold():
    from seq_vp_3d_b200.grid import make_grid_3d
    from seq_vp_3d_b200.pair import DevicePair
    d = np.load(os.path.join(GOLDEN, "q1.npz"))
    nx, ny, nz = (int(v) for v in d["grid"])
    hx, hy, hz = (float(v) for v in d["spacing"])
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=hx, hy=hy, hz=hz, unit="mm")
    lam, mu, nu, kappa = (float(v) for v in d["weights"])
    P = DevicePair(grid, d["fixed"], d["moving"], d["u_ref"], lam=lam, mu=mu, nu=nu, kappa=kappa)
    u1 = dev(d["u1"])
    w1, g1 = P.warp(u1, with_gradient=True)
    return d, grid, P, u1, w1, g1


def test_spline(gold):
    d, grid, P, u1, w1, g1 = gold
    assert rel(P.spline_coefficients(), d["spline_c"]) < TOL
    v, g = P.sample_points(d["sample_points"])
    assert rel(v, d["sample_value"]) < TOL and rel(g, d["sample_grad"]) < TOL
    assert rel(w1, d["t1/warped"]) < TOL and rel(g1, d["t1/image_grad"]) < TOL
    w, none = P.warp(u1)
    assert none is None and torch.equal(w, w1)      # value-only sampling gives the same values


def test_energy_terms(gold):
    d, grid, P, u1, w1, g1 = gold
    terms, bad = P.energy(u1, w1)
    ref = d["t1/energy"][:5]
    assert bad == 0 and ref[4] > 0
    assert np.all(np.abs(terms - ref) <= TOL * np.abs(ref)), (terms, ref)


@pytest.mark.parametrize("term", ["total", "outer", "image", "proximity", "jd", "curl", "barrier"])
def test_gradients(gold, term):
    d, grid, P, u1, w1, g1 = gold
    assert rel(P.gradient(u1, w1, g1, term), d[f"grad/{term}"]) < TOL


def test_outer_vectors_and_ggn(gold):
    d, grid, P, u1, w1, g1 = gold
    for got, ref in zip(P.outer_gradients(u1, w1, g1), d["outer_vectors"]):
        assert rel(got, ref) < TOL
    assert rel(P.ggn_diagonal(u1, g1), d["ggn_diag"]) < TOL
    assert rel(P.ggn_hvp(u1, g1, dev(d["hvp_p"])), d["ggn_hvp"]) < TOL


def test_stable_difference(gold):
    d, grid, P, u1, w1, g1 = gold
    u2 = dev(d["u2"])
    w2, _ = P.warp(u2)
    dE, dF = P.energy_difference(u1, w1, u2, w2)
    red = d["reduction"]            # actual = -(trial - base), resolution = 16 eps max(E)
    # within 1e-12 relative and within 1/8 of the reference's own comparison resolution
    for got, ref, res in ((-dE, red[0], red[1]), (-dF, red[2], red[3])):
        assert abs(got - ref) <= min(TOL * abs(ref), res / 8), (dE, dF, red)


def test_one_pass_trial_matches_separate_passes(gold):
    """svp_trial_energy: warped image, image gradient, energy terms, violations and base -> trial differences are
    bitwise those of svp_warp, svp_energy and svp_energy_difference."""
    d, grid, P, u1, w1, g1 = gold
    u2 = dev(d["u2"])
    w2, g2 = P.warp(u2, with_gradient=True)
    terms, bad = P.energy(u2, w2)
    diff = P.energy_difference(u1, w1, u2, w2)
    tw, tg, tterms, tbad, tdiff, act2 = P.trial_energy(u1, w1, u2)
    assert torch.equal(tw, w2) and torch.equal(tg, g2)
    assert same_bits(tterms, terms) and tbad == bad
    assert same_bits(np.array(tdiff), np.array(diff))
    tw, none, tterms, tbad, tdiff, _ = P.trial_energy(u1, w1, u2, with_gradient=False)
    assert none is None and torch.equal(tw, w2) and same_bits(tterms, terms)
    # barrier activity masks only skip work: with the states' masks (from their own evaluations as trials) the
    # values are bitwise the same; u1 has active cells (the fixture's barrier is active) and inactive ones
    act1 = P.trial_energy(u2, w2, u1)[5]
    assert 0 < int(act1.sum()) < act1.numel()
    assert same_bits(np.array(P.energy_difference(u1, w1, u2, w2, act1, act2)), np.array(diff))
    # with the base's own mask the trial evaluation sweeps the base only where it can contribute: same bits
    hw, hg, hterms, hbad, hdiff, hact = P.trial_energy(u1, w1, u2, base_active=act1)
    assert torch.equal(hw, w2) and torch.equal(hg, g2) and torch.equal(hact, act2)
    assert same_bits(hterms, terms) and hbad == bad and same_bits(np.array(hdiff), np.array(diff))
    rw, rg, rterms, rbad, rdiff, ract = P.trial_energy(u2, w2, u1, base_active=act2)
    assert torch.equal(ract, act1) and same_bits(np.array(rdiff), np.array(P.energy_difference(u2, w2, u1, w1)))
    # the gradient, the outer triple and the GGN diagonal with u1's mask: bitwise the unmasked values
    for term in ("total", "barrier"):
        assert torch.equal(P.gradient(u1, w1, g1, term, active=act1), P.gradient(u1, w1, g1, term))
    for a, b in zip(P.outer_gradients(u1, w1, g1, act1), P.outer_gradients(u1, w1, g1)):
        assert torch.equal(a, b)
    assert torch.equal(P.ggn_diagonal(u1, g1, act1), P.ggn_diagonal(u1, g1))


def test_poisson_metric_direction(gold):
    d, grid, P, u1, w1, g1 = gold
    alpha, a, b, m = d["poisson_ab"]
    rhs = dev(d["poisson_rhs"])
    assert rel(P.poisson_apply(a, b, rhs), d["poisson_apply"]) < TOL
    assert rel(P.poisson_apply(a, b, rhs, metric="seven_point"), d["poisson7_apply"]) < TOL
    s = dev(d["scale"])
    g = dev(d["grad/total"])
    assert rel(P.poisson_apply(a, b, g, scale=s, sign=-1.), d["direction"]) < TOL


def test_node_measure_and_root(gold):
    d, grid, P, u1, w1, g1 = gold
    node = P.node_min_jd(u1).cpu().numpy()
    assert rel(node[1:-1, 1:-1, 1:-1], d["node_jd_t62"][1:-1, 1:-1, 1:-1]) < TOL
    direction = dev(d["direction"])
    for k in range(2):
        lim, root = d[f"jd_root{k}"]
        r, bad = P.jd_root(u1, direction, lim)
        assert bad == 0
        assert (r is None and np.isnan(root)) or abs(r - root) <= 1e-12 * root, (r, root)


def test_node_measure_face_interior_extension():
    """T69/T73 (solvers/jd_affine.py:173 extend_minima): the same candidate cells as the reference and its node
    measure within 1e-12 on a field whose extension lowers several cells' minima (metric estimate, not a bound)."""
    from seq_vp_3d_b200.grid import make_grid_3d
    from seq_vp_3d_b200.pair import DevicePair
    d = np.load(os.path.join(GOLDEN, "t73.npz"))
    u = d["u"]
    nz, ny, nx = u.shape[:3]
    hx, hy, hz = (float(v) for v in d["spacing"])
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=hx, hy=hy, hz=hz, unit="mm")
    z = np.zeros((nz, ny, nx))
    P = DevicePair(grid, z, z, np.zeros_like(u), lam=.1, mu=.03, nu=.03, kappa=.002)
    ud = dev(u)
    ref62, ref73 = d["node62"], d["node73"]
    inner = (slice(1, -1),) * 3
    assert np.sum(ref73[inner] < ref62[inner]) > 0          # the extension matters on this field
    got62 = P.node_min_jd(ud).cpu().numpy()
    assert rel(got62[inner], ref62[inner]) < TOL
    stats = {}
    got73 = P.node_min_jd(ud, 0.25, stats).cpu().numpy()
    assert stats["candidates"] == int(d["candidates"])
    err = np.abs(got73[inner] - ref73[inner]) / np.maximum(np.abs(ref73[inner]), 1e-300)
    assert err.max() <= 1e-12, err.max()


# ------------------------------------------------------------------------------------------ larger, vs the oracle
def seeded_problem(shape, spacing, seed):
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    fixed = np.zeros(shape)
    moving = np.zeros(shape)
    for _ in range(12):
        c = rng.uniform([2, 2, 2], [nz - 3, ny - 3, nx - 3])
        s = rng.uniform(2, 5)
        a = rng.uniform(.2, 1.)
        d = rng.normal(size=3)
        fixed += a * np.exp(-((zz - c[0]) ** 2 + (yy - c[1]) ** 2 + (xx - c[2]) ** 2) / (2 * s * s))
        moving += a * np.exp(-((zz - c[0] - d[0]) ** 2 + (yy - c[1] - d[1]) ** 2 + (xx - c[2] - d[2]) ** 2) / (2 * s * s))
    h = np.array(spacing)
    taper = (np.sin(np.pi * zz / (nz - 1)) * np.sin(np.pi * yy / (ny - 1)) * np.sin(np.pi * xx / (nx - 1)))
    u = np.stack([taper * np.sin(2 * np.pi * (k + 1) * (xx + yy + zz) / 23 + k) for k in range(3)], -1) * 0.15 * h
    # a local compression that activates the barrier
    g = np.exp(-((zz - nz // 2) ** 2 + (yy - ny // 2) ** 2) / 4.)
    u[..., 0] += -0.94 * np.clip(xx - nx // 2, -1, 1) * h[0] * g
    u[[0, -1]] = 0.; u[:, [0, -1]] = 0.; u[:, :, [0, -1]] = 0.
    u_ref = 0.5 * u
    return fixed, moving, np.ascontiguousarray(u), np.ascontiguousarray(u_ref)


@pytest.fixture(scope="module")
def big():
    from seq_vp_3d_b200.grid import make_grid_3d
    from seq_vp_3d_b200.pair import DevicePair
    shape, spacing = (34, 30, 38), (1.0, 0.9, 1.2)
    fixed, moving, u, u_ref = seeded_problem(shape, spacing, 4)
    w = dict(lam=0.1 / 35. ** 2, mu=0.03, nu=0.03, kappa=0.002)
    grid = make_grid_3d(nx=shape[2], ny=shape[1], nz=shape[0], hx=spacing[0], hy=spacing[1], hz=spacing[2],
                        unit="mm")
    P = DevicePair(grid, fixed, moving, u_ref, **w)
    og = Q.make_grid(shape, spacing)
    OP = Q.make_problem(og, fixed, moving, u_ref, w["lam"], w["mu"], w["nu"], w["kappa"])
    return P, OP, dev(u), u


def test_larger_energy_gradient_vs_oracle(big):
    P, OP, ud, u = big
    w, g = P.warp(ud, with_gradient=True)
    ow, og = Q.warp(OP, u, True)
    assert rel(P.spline_coefficients(), OP.coeff) < TOL
    assert rel(w, ow) < TOL and rel(g, og) < TOL
    terms, bad = P.energy(ud, w)
    ref = Q.energy(OP, u, ow)
    assert bad == 0 and ref[4] > 0
    assert np.all(np.abs(terms - ref) <= TOL * np.abs(ref)), (terms, ref)
    assert rel(P.gradient(ud, w, g), Q.gradient(OP, u, ow, og)) < TOL
    assert rel(P.ggn_diagonal(ud, g), Q.ggn_diagonal(OP, u, og)) < TOL
    a, b = 0.01, 0.03
    rhs = np.random.default_rng(1).normal(size=3 * int(np.prod(OP.grid.interior_shape)))
    assert rel(P.poisson_apply(a, b, dev(rhs)), Q.poisson_apply(OP.grid, a, b, rhs)) < TOL


def test_vector_kernels_bitwise(big):
    from seq_vp_3d_b200 import pair as pm
    P, OP, ud, u = big
    rng = np.random.default_rng(5)
    theta = Q.restrict(np.moveaxis(u, -1, 0))
    p = rng.normal(size=theta.shape) * 0.3
    for tau in (0.37, 1e-3, 2.5):
        got = pm.axpy(dev(theta), tau, dev(p)).cpu().numpy()
        assert same_bits(got, theta + tau * p)
    assert torch.equal(P.inject(dev(theta)), dev(Q.inject(theta, OP.grid)))
    assert torch.equal(P.restrict(ud), dev(theta))
    # the fused trial point: axpy's candidate, inject's field and max_abs_diff's maxima, bit for bit
    S = pm.Scalars(4)
    for tau in (0.37, 1e-3):
        cand, uc = P.trial_point(dev(theta), tau, dev(p), S.slot(0))
        S.max_abs_diff(2, pm.axpy(dev(theta), tau, dev(p)), dev(theta))
        v = S.fetch()
        assert same_bits(cand.cpu().numpy(), theta + tau * p)
        assert torch.equal(uc, P.inject(cand))
        assert same_bits(v[:2], v[2:4]) and v[0] == np.max(np.abs((theta + tau * p) - theta))
    assert abs(pm.dot(dev(theta), dev(p)) - float(np.dot(theta, p))) <= 1e-13 * np.abs(theta * p).sum()
    # the fused step scalars: bitwise the separate dot and BB2 reductions, with and without the previous step
    g, pp, th0, g0, p0 = (dev(rng.normal(size=theta.shape)) for _ in range(5))
    T = pm.Scalars(16)
    T.step_dots(0, g, pp)
    T.step_dots(2, g, pp, (dev(theta), th0, g0, p0))
    T.dot(8, g, g)
    T.dot(9, g, pp)
    T.bb2(10, dev(theta), th0, g, g0, p0, pp)
    v = T.fetch()
    assert same_bits(v[0:2], v[8:10]) and same_bits(v[2:4], v[8:10]) and same_bits(v[4:8], v[10:14])
    # step bound: exact min of the reference quotients
    v = p.reshape((3,) + OP.grid.interior_shape)
    pts = (OP.grid.identity() + u)[1:-1, 1:-1, 1:-1]
    best = np.inf
    for r, axis in enumerate(OP.grid.axes):
        pos, neg = v[r] > 0, v[r] < 0
        best = min(best, np.min((axis[-1] - pts[..., r][pos]) / v[r][pos]), np.min((axis[0] - pts[..., r][neg]) / v[r][neg]))
    assert P.step_bound(ud, dev(p)) == best


@pytest.mark.parametrize("shape", [(9, 10, 263), (10, 261, 9), (260, 9, 10), (7, 8, 11)])
def test_poisson_apply_tile_edges(shape):
    """The folded DST-I passes where a half axis spans more than one 128-wide tile (x: 261 free nodes, k0 = 131;
    y: 259, odd, with the middle row; z: 258) and on a grid of short odd and even axes, in both forms, against the
    oracle's dense float64 DST-I (oracle/q1.py poisson_apply, scipy's dstn type 1 'ortho' restated), with and without
    the scale and sign epilogue.  Plain within 1e-12, mixed (3xTF32) within the mixed form's 1e-5."""
    from seq_vp_3d_b200.grid import make_grid_3d
    from seq_vp_3d_b200.pair import DevicePair
    nz, ny, nx = shape
    spacing = (1.0, 0.9, 1.1)
    rng = np.random.default_rng(11)
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=spacing[0], hy=spacing[1], hz=spacing[2], unit="mm")
    og = Q.make_grid(shape, spacing)
    img = rng.random(shape)
    nf = 3 * int(np.prod(og.interior_shape))
    rhs = rng.normal(size=nf)
    scale = rng.random(nf) + .5
    a, b = 0.02, 0.03
    ref = Q.poisson_apply(og, a, b, rhs)
    ref_scaled = -scale * Q.poisson_apply(og, a, b, scale * rhs)
    for form, tol in (("plain", TOL), ("mixed", 1e-5)):
        P = DevicePair(grid, img, img, np.zeros(shape + (3,)), lam=a, mu=.03, nu=.03, kappa=.002, precision=form)
        assert rel(P.poisson_apply(a, b, dev(rhs)), ref) < tol, form
        assert rel(P.poisson_apply(a, b, dev(rhs), scale=dev(scale), sign=-1.), ref_scaled) < tol, form
