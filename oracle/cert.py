"""ORACLE -- test infrastructure only: ctypes front of oracle/cert_oracle.c (the CPU restatement of the reference
certificate: jd_curl/three_d/compiled_enclosure.py, certificate_prescreen.py, compiled_fallback.py, feasibility.py).

Used by tests/ as the checker, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg; never by the product.
"""
import ctypes
import os
import subprocess
import threading
from itertools import product

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libcert_oracle.so")

UNIT = 2. ** -53
ETA = 1e-290
SQRT27_UP = 5.196152422706633


def _gamma(n):
    return n * UNIT / (1 - n * UNIT)


G12, G6, G3 = _gamma(12), _gamma(6), _gamma(3)

_lib = None
_lock = threading.Lock()


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB):
                build()
            L = ctypes.CDLL(LIB)
            P, I, D = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double
            L.oc_edge_hull.argtypes = [P, I, I, I, P, D, I, I, P, P]
            L.oc_prescreen.argtypes = [P, I, I, I, P, P, I, I, D, D, D, D, D, P]
            L.oc_fallback_cell.argtypes = [P, P, D, P, P, P, P, P]
            L.oc_fallback_cell.restype = ctypes.c_int
            L.oc_classify.argtypes = [P, P, P, P, D, I, I, ctypes.c_int, P]
            L.oc_certify_map.argtypes = [P, I, I, I, P, P, P, P, D, I, I, I, P, ctypes.c_int, D, D, D, D, D,
                                         ctypes.c_int, ctypes.c_int, P, P]
            _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _split(n, threads):
    threads = max(1, min(threads, n))
    edges = np.linspace(0, n, threads + 1).astype(np.int64)
    return [(int(a), int(b)) for a, b in zip(edges[:-1], edges[1:]) if b > a]


def _run(fn, n, threads):
    parts = _split(n, threads)
    if len(parts) <= 1:
        for a, b in parts:
            fn(a, b)
        return
    ts = [threading.Thread(target=fn, args=p) for p in parts]
    for t in ts:
        t.start()
    for t in ts:
        t.join()


def closed27_table(spacing):
    """CellQ1Operators3D(grid, location='closed27_uniform').coefficients (cell_q1.py:101-129), same expressions."""
    nodes = (0., .5, 1.)
    points = np.array([(x, y, z) for z, y, x in product(nodes, repeat=3)])
    vertices = [(x, y, z) for z, y, x in product((0, 1), repeat=3)]
    D = np.empty((3, 27, 8))
    for a, vertex in enumerate(vertices):
        factors = [points[:, j] if vertex[j] else 1 - points[:, j] for j in range(3)]
        for j in range(3):
            others = [k for k in range(3) if k != j]
            D[j, :, a] = (1 if vertex[j] else -1) / spacing[j] * factors[others[0]] * factors[others[1]]
    return D


def edge_hull(u, spacing, delta, threads=1):
    u = np.ascontiguousarray(u, dtype=np.float64)
    nz, ny, nx = u.shape[:3]
    n = (nz - 1) * (ny - 1) * (nx - 1)
    margin, flag = np.empty(n), np.empty(n, np.uint8)
    h = np.ascontiguousarray(spacing, dtype=np.float64)
    L = lib()
    _run(lambda a, b: L.oc_edge_hull(_ptr(u), nz, ny, nx, _ptr(h), float(delta), a, b, _ptr(margin), _ptr(flag)),
         n, threads)
    return margin, flag.astype(bool)


def prescreen(u, spacing, cells, threads=1):
    u = np.ascontiguousarray(u, dtype=np.float64)
    nz, ny, nx = u.shape[:3]
    D = np.ascontiguousarray(closed27_table(spacing))
    cells = np.ascontiguousarray(cells, dtype=np.int64)
    out = np.full(len(cells), np.nan)
    nonzero = np.abs(D[D != 0])
    if not np.all(np.isfinite(D)) or (nonzero.size and nonzero.min() < np.finfo(np.float64).tiny):
        return out
    L = lib()
    _run(lambda a, b: L.oc_prescreen(_ptr(u), nz, ny, nx, _ptr(D), _ptr(cells), a, b, G12, G6, G3, SQRT27_UP, ETA,
                                     _ptr(out)), len(cells), threads)
    return out


def fallback_cell(v, spacing, delta):
    """(ok, plo, phi, clo, chi, samples) of one cell, v = (8,3) vertex displacements."""
    v = np.ascontiguousarray(v, dtype=np.float64).reshape(8, 3)
    h = np.ascontiguousarray(spacing, dtype=np.float64)
    out = [np.empty(27) for _ in range(5)]
    ok = lib().oc_fallback_cell(_ptr(v), _ptr(h), float(delta), *[_ptr(a) for a in out])
    return (bool(ok), *out)


class _Cls(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("reason", ctypes.c_int32), ("has_margin", ctypes.c_int32),
                ("has_witness", ctypes.c_int32), ("boxes", ctypes.c_int64), ("depth", ctypes.c_int64),
                ("margin", ctypes.c_double), ("witness", ctypes.c_double * 3)]


def classify(clo, chi, plo, phi, delta, max_depth=48, max_boxes=255, depth_first=False):
    r = _Cls()
    arrs = [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (clo, chi, plo, phi)]
    lib().oc_classify(*[_ptr(a) for a in arrs], float(delta), int(max_depth), int(max_boxes), int(depth_first),
                      ctypes.byref(r))
    return dict(status=r.status, reason=r.reason, boxes=r.boxes, depth=r.depth,
                margin=r.margin if r.has_margin else None,
                witness=tuple(r.witness) if r.has_witness else None)


def certify_map(u, spacing, delta, *, max_depth=48, max_boxes=255, tile_size=65536, origin=(0., 0., 0.),
                hull=True, prescreen=True, depth_first=False):
    """(rec_i int64[13], rec_f float64[6]) of feasibility.certify_map: PrescreenCertificateConfig by default;
    prescreen=False the CompiledFallback execution, hull=False the whole-cell Bernstein execution of the bare /
    Adaptive configs (depth_first=True for the bare CertificateConfig)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    nz, ny, nx = u.shape[:3]
    h = np.ascontiguousarray(spacing, dtype=np.float64)
    axes = [np.ascontiguousarray(o + s * np.arange(n, dtype=np.float64)) for o, s, n in zip(origin, h, (nx, ny, nz))]
    D = np.ascontiguousarray(closed27_table(h))
    nonzero = np.abs(D[D != 0])
    use = int(np.all(np.isfinite(D)) and not (nonzero.size and nonzero.min() < np.finfo(np.float64).tiny))
    rec_i, rec_f = np.zeros(13, np.int64), np.zeros(6)
    lib().oc_certify_map(_ptr(u), nz, ny, nx, _ptr(h), *[_ptr(a) for a in axes], float(delta), int(max_depth),
                         int(max_boxes), int(tile_size), _ptr(D), use and prescreen, G12, G6, G3, SQRT27_UP, ETA,
                         int(hull), int(depth_first), _ptr(rec_i), _ptr(rec_f))
    return rec_i, rec_f
