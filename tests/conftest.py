import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a); run with -m gpu")


def same_bits(a, b):
    """Bitwise equality of float64 arrays (NaN payloads included)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def same_bits_nan(a, b):
    """Bitwise equality where both are not NaN, and NaN in the same places."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    na, nb = np.isnan(a), np.isnan(b)
    return a.shape == b.shape and np.array_equal(na, nb) and same_bits(np.where(na, 0., a), np.where(nb, 0., b))


@pytest.fixture(scope="session")
def cert_golden():
    return np.load(os.path.join(GOLDEN, "certificate.npz"))


@pytest.fixture(scope="session")
def cells_golden():
    return np.load(os.path.join(GOLDEN, "cells.npz"))


def cell_vertices(u, c):
    nz, ny, nx = u.shape[:3]
    cx, cy = nx - 1, ny - 1
    x0, y0, z0 = c % cx, (c // cx) % cy, c // (cx * cy)
    return np.array([u[z0 + (a >> 2), y0 + ((a >> 1) & 1), x0 + (a & 1)] for a in range(8)])


def all_vertices(u):
    nz, ny, nx = u.shape[:3]
    n = (nz - 1) * (ny - 1) * (nx - 1)
    c = np.arange(n)
    cx, cy = nx - 1, ny - 1
    x0, y0, z0 = c % cx, (c // cx) % cy, c // (cx * cy)
    return np.stack([u[z0 + (a >> 2), y0 + ((a >> 1) & 1), x0 + (a & 1)] for a in range(8)], axis=1)


@pytest.fixture(scope="session")
def configs_golden():
    return np.load(os.path.join(GOLDEN, "certificate_configs.npz"))


# (hull, prescreen, depth_first, max_depth, tile_size) of each certificate config class at its own defaults
CONFIG_EXECUTIONS = {
    "CertificateConfig": (False, False, True, 12, 8192),
    "AdaptiveCertificateConfig": (False, False, False, 48, 8192),
    "EnclosureCertificateConfig": (True, False, False, 48, 8192),
    "CompiledFallbackCertificateConfig": (True, False, False, 48, 8192),
    "PrescreenCertificateConfig": (True, True, False, 48, 8192),
}


def installed_reference():
    """The reference package (jd_curl) installed under baseline/_ref, or None.  Only the backend= adapter's GPU test
    uses it: the reference's own solve_sequential then drives this library through the adapter.  The package needs
    nibabel only for NIfTI I/O, so a stub module stands in for it."""
    import types
    path = os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(path, "jd_curl")):
        return None
    sys.modules.setdefault("nibabel", types.ModuleType("nibabel"))
    if path not in sys.path:
        sys.path.append(path)
    import jd_curl
    return jd_curl
