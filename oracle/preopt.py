"""Test infrastructure only (the checker, never the product): a float64 numpy restatement of the float32
pre-optimizer's objective and its analytic gradient (jd_curl/three_d/preopt.py:157 _pre_energy_tensors;
preopt_grad.py:1-25 for the gradient formula), pinned against the reference's own autograd gradient
(tests/golden/preopt.npz).

u_int: (3, D-2, H-2, W-2) interior displacement in voxel units (components x, y, z); F, M: (D, H, W); h = (hx, hy, hz).
"""
import numpy as np


def _pad(u_int):
    return np.pad(u_int, ((0, 0), (1, 1), (1, 1), (1, 1)))


def _coords(u, D, H, W):
    """Unclamped sample coordinates (x + u) of every node, and the clamped ones with their chi masks."""
    zz, yy, xx = np.meshgrid(np.arange(D, dtype=float), np.arange(H, dtype=float), np.arange(W, dtype=float),
                             indexing="ij")
    raw = [xx + u[0], yy + u[1], zz + u[2]]
    out, chi = [], []
    for c, n in zip(raw, (W, H, D)):
        chi.append(((c > 0) & (c < n - 1)).astype(float))
        out.append(np.clip(c, 0, n - 1))
    return out, chi


def _trilinear(M, ix, iy, iz):
    D, H, W = M.shape
    x0, y0, z0 = np.floor(ix).astype(int), np.floor(iy).astype(int), np.floor(iz).astype(int)
    wx1, wy1, wz1 = ix - x0, iy - y0, iz - z0
    wx0, wy0, wz0 = (x0 + 1) - ix, (y0 + 1) - iy, (z0 + 1) - iz

    def corner(dz, dy, dx):
        z, y, x = z0 + dz, y0 + dy, x0 + dx
        inside = (z <= D - 1) & (y <= H - 1) & (x <= W - 1)
        return np.where(inside, M[np.minimum(z, D - 1), np.minimum(y, H - 1), np.minimum(x, W - 1)], 0.)
    c = {(a, b, e): corner(a, b, e) for a in (0, 1) for b in (0, 1) for e in (0, 1)}
    wx, wy, wz = (wx0, wx1), (wy0, wy1), (wz0, wz1)
    T = sum(c[(a, b, e)] * wx[e] * wy[b] * wz[a] for a in (0, 1) for b in (0, 1) for e in (0, 1))
    dtx = sum((c[(a, b, 1)] - c[(a, b, 0)]) * wy[b] * wz[a] for a in (0, 1) for b in (0, 1))
    dty = sum((c[(a, 1, e)] - c[(a, 0, e)]) * wx[e] * wz[a] for a in (0, 1) for e in (0, 1))
    dtz = sum((c[(1, b, e)] - c[(0, b, e)]) * wx[e] * wy[b] for b in (0, 1) for e in (0, 1))
    return T, (dtx, dty, dtz)


def pre_energy_grad(F, M, h, u_int, mu, alpha, kappa, j0):
    """(terms [data, geometry, floor, curvature, min det, total], gradient like u_int)."""
    F, M = np.asarray(F, float), np.asarray(M, float)
    D, H, W = F.shape
    u = _pad(np.asarray(u_int, float))
    (ix, iy, iz), chi = _coords(u, D, H, W)
    T, dT = _trilinear(M, ix, iy, iz)
    r = T - F
    data = .5 * np.sum(r * r)
    grad = np.stack([r * dT[c] * chi[c] for c in range(3)])[:, 1:-1, 1:-1, 1:-1]
    # cell-centre derivatives: mean of the four edge differences along each axis (voxel units)
    def der(axis):
        g = np.diff(u, axis=1 + axis)
        for ax in range(3):
            if ax != axis:
                sl0 = [slice(None)] * 4
                sl1 = [slice(None)] * 4
                sl0[1 + ax] = slice(0, -1)
                sl1[1 + ax] = slice(1, None)
                g = .5 * (g[tuple(sl0)] + g[tuple(sl1)])
        return g
    dz, dy, dx = der(0), der(1), der(2)
    d = (dx, dy, dz)
    Fm = [[(1. if c == k else 0.) + d[k][c] * (h[c] / h[k]) for k in range(3)] for c in range(3)]
    det = (Fm[0][0] * (Fm[1][1] * Fm[2][2] - Fm[1][2] * Fm[2][1]) - Fm[0][1] * (Fm[1][0] * Fm[2][2] - Fm[1][2] * Fm[2][0])
           + Fm[0][2] * (Fm[1][0] * Fm[2][1] - Fm[1][1] * Fm[2][0]))
    curl = (Fm[2][1] - Fm[1][2], Fm[0][2] - Fm[2][0], Fm[1][0] - Fm[0][1])
    geometry = .5 * mu * (np.sum((det - 1) ** 2) + sum(np.sum(c * c) for c in curl))
    low = np.maximum(j0 - det, 0.)
    floor = kappa * np.sum(low ** 2)
    A = mu * (det - 1) - 2 * kappa * low
    cof = [[Fm[1][1] * Fm[2][2] - Fm[1][2] * Fm[2][1], -(Fm[1][0] * Fm[2][2] - Fm[1][2] * Fm[2][0]),
            Fm[1][0] * Fm[2][1] - Fm[1][1] * Fm[2][0]],
           [-(Fm[0][1] * Fm[2][2] - Fm[0][2] * Fm[2][1]), Fm[0][0] * Fm[2][2] - Fm[0][2] * Fm[2][0],
            -(Fm[0][0] * Fm[2][1] - Fm[0][1] * Fm[2][0])],
           [Fm[0][1] * Fm[1][2] - Fm[0][2] * Fm[1][1], -(Fm[0][0] * Fm[1][2] - Fm[0][2] * Fm[1][0]),
            Fm[0][0] * Fm[1][1] - Fm[0][1] * Fm[1][0]]]
    zero = np.zeros_like(det)
    adj = [[zero, -curl[2], curl[1]], [curl[2], zero, -curl[0]], [-curl[1], curl[0], zero]]
    full = np.zeros((3, D, H, W))
    for c in range(3):
        for k in range(3):
            G = (A * cof[c][k] + mu * adj[c][k]) * (h[c] / h[k])
            # each vertex of the cell: +1/4 at the high end along axis k, -1/4 at the low end
            for bz in (0, 1):
                for by in (0, 1):
                    for bx in (0, 1):
                        bit = (bx, by, bz)[k]
                        full[c, bz:D - 1 + bz, by:H - 1 + by, bx:W - 1 + bx] += G * (.25 if bit else -.25)
    grad = grad + full[:, 1:-1, 1:-1, 1:-1]
    curvature = 0.
    if alpha > 0:
        hx, hy, hz = h
        ui = u[:, 1:-1, 1:-1, 1:-1]
        lap = ((u[:, 2:, 1:-1, 1:-1] - 2 * ui + u[:, :-2, 1:-1, 1:-1]) / (hz * hz)
               + (u[:, 1:-1, 2:, 1:-1] - 2 * ui + u[:, 1:-1, :-2, 1:-1]) / (hy * hy)
               + (u[:, 1:-1, 1:-1, 2:] - 2 * ui + u[:, 1:-1, 1:-1, :-2]) / (hx * hx))
        lap = lap * np.array([hx, hy, hz])[:, None, None, None]
        curvature = .5 * alpha * np.sum(lap ** 2)
        L = _pad(lap)
        li = L[:, 1:-1, 1:-1, 1:-1]
        d2 = ((L[:, 2:, 1:-1, 1:-1] - 2 * li + L[:, :-2, 1:-1, 1:-1]) / (hz * hz)
              + (L[:, 1:-1, 2:, 1:-1] - 2 * li + L[:, 1:-1, :-2, 1:-1]) / (hy * hy)
              + (L[:, 1:-1, 1:-1, 2:] - 2 * li + L[:, 1:-1, 1:-1, :-2]) / (hx * hx))
        grad = grad + alpha * np.array([hx, hy, hz])[:, None, None, None] * d2
    total = data + geometry + floor + curvature
    return np.array([data, geometry, floor, curvature, det.min(), total]), grad
