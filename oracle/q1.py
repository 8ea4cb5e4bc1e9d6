"""ORACLE -- test infrastructure only: numpy restatement of the reference's Q1 energy path.

Covers (reference paths inside jd_curl/three_d/):
  cell_q1.py:101     CellQ1Operators3D tables (gauss27 / closed27_uniform points, weights, derivative tables)
  geometry.py:60     _compute_cell_geometry (F = I + grad u, cofactor rows, J, curl)
  barrier.py:7-36    barrier_terms, localized C2 branch
  interpolation.py:29 build_image_sampler: not-a-knot tensor cubic spline (SciPy make_interp_spline per axis);
                     restated here as the collocation solve on the not-a-knot knot vector
  backends/spline.py:12 cubic_basis (Cox-de Boor basis and derivative on the knot span)
  residuals.py:189   _energy (longdouble sums), linearization.py:180 energy_gradient, :217 outer_gradient_vectors,
                     :327 barrier_ggn_hvp, :357 barrier_ggn_diagonal
  energy_comparison.py:14 _barrier_difference, :65 _squared_change, :92 _differences
  poisson.py:16      poisson_spectrum, :99 PoissonInverse3D.apply (DST-I, orthonormal) -- restated by the DST-I
                     definition as a dense sine matrix per axis
  solvers/poisson_gradient.py:269 image_curvature_shift, :281 metric_diagonal
  solvers/jd_affine.py:24-60, :205, :228 closed27 cell minima, node_min_jd (T62), affine_factors
  solvers/global_jd_step.py:22-130 first_roots / global_root_cpu
Used by tests/ as the checker, by __graft_entry__.smoke() and bench.py's CPU-baseline leg; never by the product.
Parity pinned by tests/golden/q1.npz (tests/golden/q1_golden.py ran the reference).
"""
from dataclasses import dataclass
from itertools import product

import numpy as np

VERTICES = tuple((x, y, z) for z, y, x in product((0, 1), repeat=3))
GAUSS_NODES = (.5 - np.sqrt(15.) / 10, .5, .5 + np.sqrt(15.) / 10)
GAUSS_WEIGHTS = (5 / 18, 4 / 9, 5 / 18)


# ----------------------------------------------------------------------------------------------- grid and tables
@dataclass(frozen=True)
class Grid:
    shape: tuple      # (nz, ny, nx)
    spacing: tuple    # (hx, hy, hz)
    axes: tuple       # x, y, z node coordinates

    @property
    def omega(self):
        return float(np.prod(self.spacing))

    @property
    def cell_shape(self):
        return tuple(n - 1 for n in self.shape)

    @property
    def interior_shape(self):
        return tuple(n - 2 for n in self.shape)

    @property
    def n_cells(self):
        return int(np.prod(self.cell_shape))

    def node_weights(self):
        t = []
        for n in self.shape[::-1]:
            w = np.ones(n)
            w[[0, -1]] = .5
            t.append(w)
        tx, ty, tz = t
        return self.omega * tz[:, None, None] * ty[None, :, None] * tx[None, None, :]

    def identity(self):
        x, y, z = self.axes
        out = np.empty(self.shape + (3,))
        out[..., 0], out[..., 1], out[..., 2] = x, y[:, None], z[:, None, None]
        return out


def make_grid(shape_zyx, spacing_xyz, origin=(0., 0., 0.)):
    axes = tuple(o + h * np.arange(n, dtype=np.float64)
                 for o, h, n in zip(origin, spacing_xyz, shape_zyx[::-1]))
    return Grid(tuple(int(n) for n in shape_zyx), tuple(float(h) for h in spacing_xyz), axes)


@dataclass(frozen=True)
class Ops:
    points: np.ndarray        # (P, 3) xyz in [0,1]
    weights: np.ndarray       # (P,) quadrature weights including omega
    D: np.ndarray             # (3, P, 8) physical derivative table


def ops(grid, location):
    if location == "gauss27":
        nodes, w1 = GAUSS_NODES, GAUSS_WEIGHTS
    elif location == "closed27_uniform":
        nodes, w1 = (0., .5, 1.), (1 / 3, 1 / 3, 1 / 3)
    else:
        raise ValueError(location)
    points = np.array([(x, y, z) for z, y, x in product(nodes, repeat=3)])
    weights = np.array([grid.omega * x * y * z for z, y, x in product(w1, repeat=3)])
    if location == "closed27_uniform":
        weights = np.full(27, grid.omega / 27)
    D = np.empty((3, len(points), 8))
    for a, vertex in enumerate(VERTICES):
        factors = [points[:, j] if vertex[j] else 1 - points[:, j] for j in range(3)]
        for j in range(3):
            o = [k for k in range(3) if k != j]
            D[j, :, a] = (1 if vertex[j] else -1) / grid.spacing[j] * factors[o[0]] * factors[o[1]]
    return Ops(points, weights, D)


def cell_nodes(grid, cells=None):
    """(ncell, 8) flat node indices of each cell's vertices (cell_q1.py:89)."""
    cz, cy, cx = grid.cell_shape
    c = np.arange(grid.n_cells) if cells is None else np.asarray(cells)
    z, y, x = np.unravel_index(c, (cz, cy, cx))
    _, ny, nx = grid.shape
    return np.stack([((z + vz) * ny + y + vy) * nx + x + vx for vx, vy, vz in VERTICES], axis=-1)


def local(u, grid, cells=None):
    return u.reshape(-1, 3)[cell_nodes(grid, cells)]          # (ncell, 8, 3)


TILE = 8192       # cells per tile (the reference's MemoryConfig.cell_tile_size)


def tiles(grid):
    for start in range(0, grid.n_cells, TILE):
        yield np.arange(start, min(start + TILE, grid.n_cells))


# ----------------------------------------------------------------------------------------------- geometry
def cofactor(F):
    out = np.empty(F.shape)
    for r, j, k in ((0, 1, 2), (1, 2, 0), (2, 0, 1)):
        for c, l, m in ((0, 1, 2), (1, 2, 0), (2, 0, 1)):
            out[..., r, c] = F[..., j, l] * F[..., k, m] - F[..., j, m] * F[..., k, l]
    return out


def grad_points(loc, op):
    """V[n, p, r, j] = sum_a loc[n, a, r] D[j, p, a]: per component/axis (cells, 8) @ (8, P) products, as
    geometry.py:11-32 forms them."""
    n, P = loc.shape[0], op.D.shape[1]
    V = np.empty((n, P, 3, 3))
    for r in range(3):
        v = np.ascontiguousarray(loc[:, :, r])
        for j in range(3):
            V[..., r, j] = v @ op.D[j].T
    return V


def geometry(loc, op):
    """F (n,P,3,3), A, J (n,P), curl (n,P,3) from local vertex displacements (n,8,3)."""
    V = grad_points(loc, op)
    F = V + np.eye(3)
    A = cofactor(F)
    J = np.sum(F[..., 0, :] * A[..., 0, :], axis=-1)
    curl = np.stack((F[..., 2, 1] - F[..., 1, 2], F[..., 0, 2] - F[..., 2, 0], F[..., 1, 0] - F[..., 0, 1]), -1)
    return F, A, J, curl


def barrier_terms(J, delta, weight, activation):
    """Localized C2 barrier b = -w r^2 log t, first and second derivative (barrier.py:18-36)."""
    value, first, second = (np.zeros_like(J) for _ in range(3))
    active = J < activation
    scale = activation - delta
    t = (J[active] - delta) / scale
    r = (activation - J[active]) / scale
    logt = np.log(t)
    near = r < .5
    logt[near] = np.log1p(-r[near])
    value[active] = -weight * r * r * logt
    first[active] = weight * (2 * r * logt - r * r / t) / scale
    second[active] = weight * (-2 * logt + 4 * r / t + (r / t) ** 2) / scale ** 2
    return value, first, second


# ----------------------------------------------------------------------------------------------- spline
def not_a_knot_knots(x):
    return np.r_[(x[0],) * 4, x[2:-2], (x[-1],) * 4]


def basis_and_derivative(t, x, n):
    """cubic_basis (backends/spline.py:12): span, 4 basis values, 4 derivative values per query."""
    x = np.asarray(x, dtype=np.float64)
    span = np.clip(np.searchsorted(t, x, side="right") - 1, 3, n - 1)
    basis = np.ones((x.size, 1))
    quad = None
    for degree in range(1, 4):
        values, saved = [], np.zeros_like(x)
        for r in range(degree):
            right = t[span + r + 1] - x
            left = x - t[span + 1 - degree + r]
            temp = basis[:, r] / (right + left)
            values.append(saved + right * temp)
            saved = left * temp
        values.append(saved)
        basis = np.stack(values, -1)
        if degree == 2:
            quad = basis
    idx = span[:, None] + np.arange(-3, 1)
    zero = np.zeros((x.size, 1))
    a, b = t[idx + 3] - t[idx], t[idx + 4] - t[idx + 1]
    deriv = (3 * np.concatenate((zero, quad), -1) / np.where(a != 0, a, 1)
             - 3 * np.concatenate((quad, zero), -1) / np.where(b != 0, b, 1))
    return idx, basis, deriv


def collocation_matrix(x):
    t = not_a_knot_knots(x)
    n = len(x)
    idx, basis, _ = basis_and_derivative(t, x, n)
    B = np.zeros((n, n))
    for i in range(n):
        B[i, idx[i]] = basis[i]
    return B


def spline_coefficients(image, grid):
    """Tensor not-a-knot cubic coefficients (nz, ny, nx): one collocation solve per axis, x first."""
    c = np.asarray(image, dtype=np.float64).copy()
    for axis, coords in enumerate(grid.axes[::-1]):       # z, y, x storage axes 0, 1, 2 ... processed 0, 1, 2
        B = collocation_matrix(coords)
        moved = np.moveaxis(c, axis, 0)
        sol = np.linalg.solve(B, moved.reshape(len(coords), -1))
        c = np.moveaxis(sol.reshape(moved.shape), 0, axis)
    return np.ascontiguousarray(c)


def spline_sample(coeff, grid, points_xyz, with_gradient=True):
    """value (N,), gradient (N,3) xyz at physical points (N,3)."""
    pts = np.asarray(points_xyz, dtype=np.float64).reshape(-1, 3)
    nz, ny, nx = coeff.shape
    bases = []
    for axis, (coords, n) in enumerate(zip(grid.axes[::-1], (nz, ny, nx))):
        bases.append(basis_and_derivative(not_a_knot_knots(coords), pts[:, 2 - axis], n))
    (iz, bz, dz), (iy, by, dy), (ix, bx, dx) = bases
    c = coeff[iz[:, :, None, None], iy[:, None, :, None], ix[:, None, None, :]]

    def contract(z, y, x):
        return (c * z[:, :, None, None] * y[:, None, :, None] * x[:, None, None, :]).sum(axis=(1, 2, 3))
    value = contract(bz, by, bx)
    if not with_gradient:
        return value, None
    return value, np.stack((contract(bz, by, dx), contract(bz, dy, bx), contract(dz, by, bx)), -1)


# ----------------------------------------------------------------------------------------------- problem
@dataclass
class Problem:
    grid: Grid
    fixed: np.ndarray
    coeff: np.ndarray
    u_ref: np.ndarray
    lam: float
    mu: float
    nu: float
    kappa: float
    activation: float = .05
    delta: float = 0.

    @property
    def barrier_weight(self):
        return self.kappa * self.grid.omega / 27


def make_problem(grid, fixed, moving, u_ref, lam, mu, nu, kappa, activation=.05, delta=0.):
    return Problem(grid, np.asarray(fixed, dtype=np.float64), spline_coefficients(moving, grid),
                   np.asarray(u_ref, dtype=np.float64), lam, mu, nu, kappa, activation, delta)


def warp(problem, u, with_gradient=False):
    pts = problem.grid.identity() + u
    v, g = spline_sample(problem.coeff, problem.grid, pts.reshape(-1, 3), with_gradient)
    shape = problem.grid.shape
    return v.reshape(shape), (None if g is None else g.reshape(shape + (3,)))


def cell_terms(problem, u):
    """(jd, curl, barrier) longdouble sums over all cells, tile by tile (residuals.py:166 _cell_energy)."""
    g = problem.grid
    G, C = ops(g, "gauss27"), ops(g, "closed27_uniform")
    jd = cu = bar = np.longdouble(0)
    for t in tiles(g):
        _, _, J, curl = geometry(local(u, g, t), G)
        _, _, Jr, curlr = geometry(local(problem.u_ref, g, t), G)
        jd += .5 * problem.mu * np.sum(G.weights * (J - Jr) ** 2, dtype=np.longdouble)
        cu += .5 * problem.nu * np.sum(G.weights[None, :, None] * (curl - curlr) ** 2, dtype=np.longdouble)
        _, _, Jc, _ = geometry(local(u, g, t), C)
        if np.any(Jc <= problem.delta):
            raise FloatingPointError("barrier point J <= delta")
        b, _, _ = barrier_terms(Jc, problem.delta, problem.barrier_weight, problem.activation)
        bar += np.sum(b, dtype=np.longdouble)
    return jd, cu, bar


def energy(problem, u, warped=None):
    """(image, proximity, jd, curl, barrier) of residuals.py:189 _energy."""
    if warped is None:
        warped, _ = warp(problem, u)
    q = problem.grid.node_weights()
    image = .5 * np.sum(q * (warped - problem.fixed) ** 2, dtype=np.longdouble)
    prox = .5 * problem.lam * np.sum(q[..., None] * (u - problem.u_ref) ** 2, dtype=np.longdouble)
    jd, cu, bar = cell_terms(problem, u)
    return np.array([float(image), float(prox), float(jd), float(cu), float(bar)])


def _scatter(grid, op, flux, out, cells=None):
    """out (3, nz, ny, nx) += D^T flux (flux (n,P,3,3) [r, j]) (cell_q1.py:116 _transpose_add)."""
    nodes = cell_nodes(grid, cells)
    size = out[0].size
    for r in range(3):
        loc = sum(np.ascontiguousarray(flux[..., r, j]) @ op.D[j] for j in range(3))   # (n, 8)
        out[r] += np.bincount(nodes.ravel(), weights=loc.ravel(), minlength=size).reshape(out[r].shape)


def _flux(A, jd, curl):
    flux = A * jd[..., None, None]
    if curl is not None:
        flux[..., 2, 1] += curl[..., 0]
        flux[..., 1, 2] -= curl[..., 0]
        flux[..., 0, 2] += curl[..., 1]
        flux[..., 2, 0] -= curl[..., 1]
        flux[..., 1, 0] += curl[..., 2]
        flux[..., 0, 1] -= curl[..., 2]
    return flux


def restrict(out):
    return np.ascontiguousarray(out[:, 1:-1, 1:-1, 1:-1]).ravel()


def inject(theta, grid):
    u = np.zeros(grid.shape + (3,))
    u[1:-1, 1:-1, 1:-1] = np.moveaxis(theta.reshape((3,) + grid.interior_shape), 0, -1)
    return u


def gradient(problem, u, warped, image_grad, term="total"):
    """linearization.py:180 energy_gradient on free nodes, component-major."""
    g = problem.grid
    q = g.node_weights()
    out = np.zeros((3,) + g.shape)
    if term in ("total", "outer", "image"):
        out += np.moveaxis(q[..., None] * (warped - problem.fixed)[..., None] * image_grad, -1, 0)
    if term in ("total", "proximity"):
        out += np.moveaxis(problem.lam * q[..., None] * (u - problem.u_ref), -1, 0)
    G, C = ops(g, "gauss27"), ops(g, "closed27_uniform")
    for t in tiles(g):
        if term in ("total", "jd", "curl"):
            _, A, J, curl = geometry(local(u, g, t), G)
            _, _, Jr, curlr = geometry(local(problem.u_ref, g, t), G)
            jd = problem.mu * G.weights * (J - Jr) if term != "curl" else np.zeros_like(J)
            cu = problem.nu * G.weights[None, :, None] * (curl - curlr) if term != "jd" else None
            _scatter(g, G, _flux(A, jd, cu), out, t)
        if term in ("total", "outer", "barrier"):
            _, A, J, _ = geometry(local(u, g, t), C)
            _, first, _ = barrier_terms(J, problem.delta, problem.barrier_weight, problem.activation)
            _scatter(g, C, _flux(A, first, None), out, t)
    return restrict(out)


def ggn_diagonal(problem, u, image_grad):
    """linearization.py:357 barrier_ggn_diagonal."""
    g = problem.grid
    q = g.node_weights()
    out = np.moveaxis(q[..., None] * image_grad ** 2 + problem.lam * q[..., None], -1, 0).copy()
    G, C = ops(g, "gauss27"), ops(g, "closed27_uniform")
    D, Dc = G.D, C.D
    for t in tiles(g):
        _, A, _, _ = geometry(local(u, g, t), G)
        _, Ac, Jc, _ = geometry(local(u, g, t), C)
        _, _, curv = barrier_terms(Jc, problem.delta, problem.barrier_weight, problem.activation)
        nodes = cell_nodes(g, t)
        for r in range(3):
            flat = out[r].ravel()
            for a in range(8):
                lj = sum(A[..., r, j] * D[j, :, a] for j in range(3))
                lc = sum(Ac[..., r, j] * Dc[j, :, a] for j in range(3))
                cs = sum(D[j, :, a] ** 2 for j in range(3) if j != r)
                value = np.sum(G.weights * (problem.mu * lj ** 2 + problem.nu * cs), axis=-1)
                value += np.sum(curv * lc ** 2, axis=-1)
                flat += np.bincount(nodes[:, a], weights=value, minlength=flat.size)
    return restrict(out)


def ggn_hvp(problem, u, image_grad, p):
    """linearization.py:327 barrier_ggn_hvp."""
    g = problem.grid
    q = g.node_weights()
    v = inject(p, g)
    node = q[..., None] * image_grad * np.sum(image_grad * v, -1)[..., None] + problem.lam * q[..., None] * v
    out = np.moveaxis(node, -1, 0).copy()
    G, C = ops(g, "gauss27"), ops(g, "closed27_uniform")
    _, A, _, _ = geometry(local(u, g), G)
    V = grad_points(local(v, g), G)
    jd = np.sum(A * V, axis=(-2, -1))
    curl = np.stack((V[..., 2, 1] - V[..., 1, 2], V[..., 0, 2] - V[..., 2, 0], V[..., 1, 0] - V[..., 0, 1]), -1)
    _scatter(g, G, _flux(A, problem.mu * G.weights * jd, problem.nu * G.weights[None, :, None] * curl), out)
    _, Ac, Jc, _ = geometry(local(u, g), C)
    _, _, curv = barrier_terms(Jc, problem.delta, problem.barrier_weight, problem.activation)
    Vc = grad_points(local(v, g), C)
    lj = np.sum(Ac * Vc, axis=(-2, -1))
    _scatter(g, C, _flux(Ac, curv * lj, None), out)
    return restrict(out)


# ----------------------------------------------------------------------------------------------- stable differences
def barrier_difference(a, b, delta, activation):
    """energy_comparison.py:14-62 localized branch, longdouble."""
    a, b, d = a.astype(np.longdouble), b.astype(np.longdouble), np.longdouble(delta)
    act = np.longdouble(activation)
    a, b = np.minimum(a, act), np.minimum(b, act)
    scale = act - d
    ra, rb = (act - a) / scale, (act - b) / scale
    h = (b - a) / scale
    loga = np.log((a - d) / scale)
    near = ra < .5
    loga[near] = np.log1p(-ra[near])
    x = (b - a) / (a - d)
    ratio = np.empty_like(x)
    near = x >= -.5
    ratio[near] = np.log1p(x[near])
    ratio[~near] = np.log((b[~near] - d) / (a[~near] - d))
    return h * (ra + rb) * loga - rb * rb * ratio


def _sq(a, b):
    a, b = a.astype(np.longdouble), b.astype(np.longdouble)
    return np.sum((b - a) * (b + a), dtype=np.longdouble) / 2


def differences(problem, base_u, base_w, trial_u, trial_w):
    """(E difference, F difference) trial - base (energy_comparison.py:92 _differences)."""
    g = problem.grid
    q = g.node_weights()
    img = lambda w: np.sqrt(q) * (w - problem.fixed)
    prox = lambda u: np.sqrt(problem.lam * q)[..., None] * (u - problem.u_ref)
    image = _sq(img(base_w), img(trial_w))
    total = image + _sq(prox(base_u), prox(trial_u))
    G, C = ops(g, "gauss27"), ops(g, "closed27_uniform")
    w = np.longdouble(problem.kappa) * np.longdouble(g.omega) / 27
    bar = np.longdouble(0)
    for t in tiles(g):
        _, _, Jr, curlr = geometry(local(problem.u_ref, g, t), G)
        blocks = []
        for u in (base_u, trial_u):
            _, _, J, curl = geometry(local(u, g, t), G)
            blocks.append((np.sqrt(problem.mu * G.weights) * (J - Jr),
                           np.sqrt(problem.nu * G.weights)[None, :, None] * (curl - curlr)))
        total += _sq(blocks[0][0], blocks[1][0]) + _sq(blocks[0][1], blocks[1][1])
        Ja = geometry(local(base_u, g, t), C)[2]
        Jb = geometry(local(trial_u, g, t), C)[2]
        bar += w * np.sum(barrier_difference(Ja, Jb, problem.delta, problem.activation), dtype=np.longdouble)
    return total + bar, image + bar


# ----------------------------------------------------------------------------------------------- Poisson / DST-I
def poisson_spectrum(grid, metric="q1"):
    ell, mass = [], []
    for n, h in zip(grid.shape[::-1], grid.spacing):
        theta = np.pi * np.arange(1, n - 1) / (n - 1)
        ell.append((2 * np.sin(theta / 2) / h) ** 2)
        mass.append((2 + np.cos(theta)) / 3)
    ex, ey, ez = ell[0][None, None, :], ell[1][None, :, None], ell[2][:, None, None]
    mx, my, mz = mass[0][None, None, :], mass[1][None, :, None], mass[2][:, None, None]
    return ex + ey + ez if metric == "seven_point" else ex * my * mz + mx * ey * mz + mx * my * ez


def dst1_matrix(n):
    """Orthonormal DST-I: S[j,k] = sqrt(2/(n+1)) sin(pi (j+1)(k+1)/(n+1)); symmetric and its own inverse."""
    jk = np.outer(np.arange(1, n + 1), np.arange(1, n + 1)) % (2 * (n + 1))
    return np.sqrt(2. / (n + 1)) * np.sin(np.pi * jk / (n + 1))


def dst3(x):
    """DST-I along the last three axes of (..., nz, ny, nx)."""
    for axis in (-1, -2, -3):
        S = dst1_matrix(x.shape[axis])
        x = np.moveaxis(np.tensordot(np.moveaxis(x, axis, -1), S, axes=([-1], [0])), -1, axis)
    return x


def poisson_apply(grid, a, b, rhs, metric="q1"):
    den = grid.omega * (a + b * poisson_spectrum(grid, metric))
    f = rhs.reshape((3,) + grid.interior_shape)
    return dst3(dst3(f) / den).ravel()


def image_curvature_shift(problem, image_grad, factor=1.):
    g = problem.grid
    b = image_grad[1:-1, 1:-1, 1:-1]
    q = g.node_weights()[1:-1, 1:-1, 1:-1] / g.omega
    return factor * float(np.mean(q * np.sum(b * b, axis=-1))) / 3


def metric_diagonal(grid, a, b, metric="q1"):
    inv_h2 = sum(1 / h ** 2 for h in grid.spacing)
    return grid.omega * (a + b * (8 / 9) * inv_h2 if metric == "q1" else a + 2 * b * inv_h2)


# ----------------------------------------------------------------------------------------------- JD measure / root
EDGE_INDICES = np.array(
    [[9 * iz + 3 * iy + ix for ix in range(3)] for iz in (0, 2) for iy in (0, 2)]
    + [[9 * iz + 3 * iy + ix for iy in range(3)] for iz in (0, 2) for ix in (0, 2)]
    + [[9 * iz + 3 * iy + ix for iz in range(3)] for iy in (0, 2) for ix in (0, 2)])


def closed27_cell_minima(J):
    f = J[:, EDGE_INDICES]
    f0, f1, f2 = f[..., 0], f[..., 1], f[..., 2]
    a = 2 * (f0 - 2 * f1 + f2)
    b = -3 * f0 + 4 * f1 - f2
    inside = (a > 0) & (b < 0) & (-b < 2 * a)
    em = np.full(f0.shape, np.inf)
    em[inside] = f0[inside] - b[inside] ** 2 / (4 * a[inside])
    return np.minimum(J.min(axis=1), em.min(axis=1))


def to_bernstein27(J):
    """bernstein_barrier.py:26: closed27 values -> Bernstein coefficients, per axis x, y, z middle = 2b - (a+c)/2."""
    v = np.array(J, dtype=np.float64).reshape(-1, 3, 3, 3)
    v[..., 1] = 2. * v[..., 1] - .5 * (v[..., 0] + v[..., 2])
    v[..., 1, :] = 2. * v[..., 1, :] - .5 * (v[..., 0, :] + v[..., 2, :])
    v[:, 1] = 2. * v[:, 1] - .5 * (v[:, 0] + v[:, 2])
    return v.reshape(-1, 27)


_LAGRANGE_TO_POWER = np.array([[1., -3., 2.], [0., 4., -4.], [0., -1., 2.]])   # L_a(t) = sum_i M[a, i] t^i


def _lagrange3(t):
    t = np.asarray(t, dtype=np.float64)
    return np.stack([2 * (t - .5) * (t - 1), -4 * t * (t - 1), 2 * t * (t - .5)], axis=-1)


def _tri_eval(C, x, dx=(0, 0, 0)):
    """sum C[k,j,i] d^dz z^k d^dy y^j d^dx x^i at points x (n, 3) (xyz); C (n, 27) monomial coefficients."""
    def pw(t, d):
        one, zero = np.ones_like(t), np.zeros_like(t)
        return [np.stack([one, t, t * t], -1), np.stack([zero, one, 2 * t], -1), np.stack([zero, zero, 2 * one], -1)][d]
    X, Y, Z = pw(x[:, 0], dx[0]), pw(x[:, 1], dx[1]), pw(x[:, 2], dx[2])
    row = (Z[:, :, None, None] * Y[:, None, :, None] * X[:, None, None, :]).reshape(len(x), 27)
    return np.sum(C * row, axis=1)


def face_interior_minima(J27, starts=4, iterations=30):
    """solvers/jd_affine.py:130 (T69): min over the 9^3 grid of the cell's triquadratic J and of a bounded projected
    Newton descent (30 iterations, <= 40 halvings, strict decrease) from the `starts` lowest grid points."""
    J27 = np.asarray(J27, dtype=np.float64).reshape(-1, 27)
    n = len(J27)
    M = _LAGRANGE_TO_POWER
    C = np.einsum("ncba,ck,bj,ai->nkji", J27.reshape(-1, 3, 3, 3), M, M, M).reshape(-1, 27)
    t9 = np.linspace(0., 1., 9)
    L = _lagrange3(t9)
    V9 = np.kron(L, np.kron(L, L))                                  # (729, 27), z-major rows
    G9 = np.array([(x, y, z) for z in t9 for y in t9 for x in t9])
    grid_values = J27 @ V9.T
    order = np.argsort(grid_values, axis=1, kind="stable")[:, :starts]
    best = grid_values.min(axis=1)
    found = np.full(n, np.inf)
    for s in range(order.shape[1]):
        x = G9[order[:, s]].copy()
        f = _tri_eval(C, x)
        live = np.ones(n, dtype=bool)
        for _ in range(iterations):
            idx = np.flatnonzero(live)
            if idx.size == 0:
                break
            xi, Ci = x[idx], C[idx]
            g = np.stack([_tri_eval(Ci, xi, (1, 0, 0)), _tri_eval(Ci, xi, (0, 1, 0)), _tri_eval(Ci, xi, (0, 0, 1))], -1)
            H = np.empty((idx.size, 3, 3))
            for a, b in ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)):
                d = [0, 0, 0]
                d[a] += 1
                d[b] += 1
                H[:, a, b] = H[:, b, a] = _tri_eval(Ci, xi, tuple(d))
            free = ~(((xi <= 0.) & (g > 0)) | ((xi >= 1.) & (g < 0)))
            gf = np.where(free, g, 0.)
            Hf = H * free[:, :, None] * free[:, None, :] + np.eye(3) * (~free)[:, :, None]
            w, Q = np.linalg.eigh(Hf)
            scale = np.maximum(1., np.abs(w).max(axis=1))
            ok = np.all(w > 1e-12 * scale[:, None], axis=1)
            newton = -np.einsum("nij,nj,nkj,nk->ni", Q, 1 / np.where(ok[:, None], w, 1.), Q, gf)
            d = np.where(ok[:, None], newton, -gf / scale[:, None])
            step, done = np.ones(idx.size), np.zeros(idx.size, dtype=bool)
            for _ in range(40):
                xt = np.clip(xi + step[:, None] * d, 0., 1.)
                ft = _tri_eval(Ci, xt)
                take = (~done) & (ft < f[idx])
                x[idx[take]], f[idx[take]] = xt[take], ft[take]
                done |= take
                step = np.where(done, step, .5 * step)
                if done.all():
                    break
            live[idx[~done]] = False
        found = np.minimum(found, f)
    return np.minimum(best, found)


def node_min_jd(problem, u, extension_activation=None):
    """T62 node measure (solvers/jd_affine.py:205); with extension_activation, the T69/T73 face/interior extension
    on candidate cells (jd_affine.py:173 extend_minima).  Returns (node, number of candidate cells)."""
    g = problem.grid
    J = geometry(local(u, g), ops(g, "closed27_uniform"))[2]
    m = closed27_cell_minima(J)
    ncand = 0
    if extension_activation is not None:
        cand = np.flatnonzero(to_bernstein27(J).min(axis=1) < np.minimum(m, extension_activation))
        ncand = cand.size
        if ncand:
            m[cand] = np.minimum(m[cand], face_interior_minima(J[cand]))
    node = np.full(g.shape, np.inf).ravel()
    nodes = cell_nodes(g)
    for a in range(8):
        np.minimum.at(node, nodes[:, a], m)
    node = node.reshape(g.shape)
    return node if extension_activation is None else (node, ncand)


def affine_factors(node, activation=.25, floor=1e-12):
    inner = node[1:-1, 1:-1, 1:-1]
    r = np.minimum(1., np.maximum(inner, floor) / activation)
    return np.broadcast_to(r, (3,) + r.shape).ravel()


def first_roots(b0, b1, b2, b3, bisections=50):
    """solvers/global_jd_step.py:52."""
    out = np.full(b0.shape, np.inf)
    with np.errstate(all="ignore"):
        maybe = ~(b0 > np.abs(b1) + np.abs(b2) + np.abs(b3))
    if not np.any(maybe):
        return out
    b0, b1, b2, b3 = b0[maybe], b1[maybe], b2[maybe], b3[maybe]
    a, bb, c = 3 * b3, 2 * b2, b1
    one = np.ones_like(b1)
    with np.errstate(all="ignore"):
        linear = a == 0
        r_lin = np.where(linear & (bb != 0), -c / np.where(bb != 0, bb, 1.), np.nan)
        disc = bb * bb - 4 * a * c
        sq = np.sqrt(np.where(disc >= 0, disc, 0.))
        qq = -(bb + np.where(bb >= 0, sq, -sq)) / 2
        r1 = np.where(~linear & (disc >= 0) & (a != 0), qq / np.where(a != 0, a, 1.), np.nan)
        r2 = np.where(~linear & (disc >= 0) & (qq != 0), c / np.where(qq != 0, qq, 1.), np.nan)
        r1 = np.where(linear, r_lin, r1)
        r2 = np.where(linear, np.nan, r2)
    r1 = np.where((r1 > 0) & (r1 < 1), r1, one)
    r2 = np.where((r2 > 0) & (r2 < 1), r2, one)
    t1, t2 = np.minimum(r1, r2), np.maximum(r1, r2)
    qv = lambda s: b0 + s * (b1 + s * (b2 + s * b3))
    touch = lambda s: 4 * np.finfo(float).eps * (np.abs(b0) + s * (np.abs(b1) + s * (np.abs(b2) + s * np.abs(b3))))
    q1, q2, q3 = qv(t1) <= touch(t1), qv(t2) <= touch(t2), qv(one) <= 0
    hi = np.where(q1, t1, np.where(q2, t2, np.where(q3, 1., np.nan)))
    lo = np.where(q1, 0., np.where(q2, t1, np.where(q3, t2, np.nan)))
    has = np.isfinite(hi)
    lo, hi = lo[has], hi[has]
    cs = [x[has] for x in (b0, b1, b2, b3)]
    for _ in range(bisections):
        mid = .5 * (lo + hi)
        neg = cs[0] + mid * (cs[1] + mid * (cs[2] + mid * cs[3])) <= 0
        hi = np.where(neg, mid, hi)
        lo = np.where(neg, lo, mid)
    roots = np.full(b0.shape, np.inf)
    roots[has] = lo
    out[maybe] = roots
    return out


def global_jd_root(problem, u, direction, limit):
    """global_root_cpu: tau of the first closed27 root of det(F + tau V) - delta in (0, limit], or None."""
    g = problem.grid
    C = ops(g, "closed27_uniform")
    F = geometry(local(u, g), C)[0]
    V = grad_points(local(inject(direction, g), g), C)
    AF, AV = cofactor(F), cofactor(V)
    c0 = np.sum(F[..., 0, :] * AF[..., 0, :], -1) - problem.delta
    c1 = np.sum(AF * V, axis=(-2, -1))
    c2 = np.sum(F * AV, axis=(-2, -1))
    c3 = np.sum(V[..., 0, :] * AV[..., 0, :], -1)
    valid = c0 > 0
    r = first_roots(c0[valid], c1[valid] * limit, c2[valid] * limit ** 2, c3[valid] * limit ** 3)
    s = float(r.min()) if r.size else np.inf
    return None if not np.isfinite(s) else s * limit
