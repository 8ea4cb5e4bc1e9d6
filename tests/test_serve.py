"""Admission logic of the serving form (no GPU: the registration callable is a host fake).  Requests wait for a slot
and for HBM budget, run in arrival order among those that fit, and failures keep the slot open."""
import threading
import time

import pytest

from seq_vp_3d_b200.grid import make_grid_3d
from seq_vp_3d_b200.serve import RegistrationServer, footprint_bytes


class Fake:
    def __init__(self, delay=.05):
        self.delay = delay
        self.lock = threading.Lock()
        self.active = 0
        self.peak = 0
        self.order = []

    def __call__(self, fixed, moving, grid, weights):
        with self.lock:
            self.active += 1
            self.peak = max(self.peak, self.active)
            self.order.append(weights["id"])
        time.sleep(self.delay)
        with self.lock:
            self.active -= 1
        if weights.get("fail"):
            raise FloatingPointError("nonfinite")
        return type("R", (), {"certified": True, "status": "ok", "id": weights["id"]})()


def grid(n):
    return make_grid_3d(nx=n, ny=n, nz=n, hx=1., hy=1., hz=1., unit="mm")


def test_slots_bound_concurrency_and_all_finish():
    fake = Fake()
    with RegistrationServer(slots=3, hbm_budget=None, run=fake) as srv:
        futs = [srv.submit(None, None, grid(8), dict(id=k)) for k in range(9)]
        ids = [f.result(timeout=10).id for f in futs]
    assert ids == list(range(9))
    assert fake.peak == 3
    assert len(srv.latencies) == 9 and set(srv.percentiles()) == {"p50", "p95", "p99"}


def test_budget_admits_by_footprint():
    fake = Fake()
    g = grid(16)
    one = footprint_bytes(g.shape)
    with RegistrationServer(slots=4, hbm_budget=int(2.5 * one), run=fake) as srv:
        futs = [srv.submit(None, None, g, dict(id=k)) for k in range(6)]
        [f.result(timeout=10) for f in futs]
    assert fake.peak == 2            # four slots, but only two fit the budget at a time


def test_too_large_request_is_refused_and_failures_keep_slots():
    fake = Fake(delay=.01)
    g = grid(16)
    with RegistrationServer(slots=1, hbm_budget=footprint_bytes(g.shape) // 2, run=fake) as srv:
        with pytest.raises(MemoryError):
            srv.submit(None, None, g, dict(id=0)).result(timeout=5)
    with RegistrationServer(slots=1, hbm_budget=None, run=fake) as srv:
        bad = srv.submit(None, None, g, dict(id=1, fail=True))
        good = srv.submit(None, None, g, dict(id=2))
        with pytest.raises(FloatingPointError):
            bad.result(timeout=5)
        assert good.result(timeout=5).id == 2
