"""Continuous batching of certified registrations on one GPU (the serving form).

Requests arrive while others run.  Each admitted request gets a slot: a host worker thread and its own CUDA stream,
its own device state (pair constants, displacement, BB history, certificate workspace), so the device work of the
requests in flight overlaps and fills the gaps that one registration's host control leaves.  Admission is by slot and
by HBM footprint: a request waits until a slot is free and its estimated device footprint fits the remaining budget.
Only certified results are returned (a registration that ends uncertified raises in its future).

Every request's result is the one it gets alone: no state is shared between slots (the kernels are deterministic and
per-pair; the certificate workspace is per thread), which tests/test_serve_gpu.py checks bit for bit.
"""
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np


def footprint_bytes(shape, preopt=True):
    """Estimated device bytes of one registration at grid `shape` (nz, ny, nx): node fields (u, u_ref, warped,
    image gradient, images, spline) of the base, trial and reference states, free vectors (gradients, direction,
    theta, scale, BB history), the two cell-local gradient buffers (24 doubles per cell each), the DST scratch and
    the certificate workspace (about 70 B per cell)."""
    nz, ny, nx = shape
    nn, nc, nf = nx * ny * nz, (nx - 1) * (ny - 1) * (nz - 1), (nx - 2) * (ny - 2) * (nz - 2)
    node = 8 * nn * (3 * 3 + 3 * 3 + 3 + 3)           # u / image gradient of base, trial, previous; images, spline
    free = 8 * 3 * nf * 12                              # gradients, direction, theta, scale, BB history, DST scratch
    cells = 8 * 24 * nc * 2 + 70 * nc
    pre = 4 * nn * 12 if preopt else 0
    return int(1.15 * (node + free + cells + pre))


@dataclass
class Request:
    fixed: object
    moving: object
    grid: object
    weights: dict
    tag: object = None
    submitted: float = 0.
    started: float = 0.
    finished: float = 0.
    footprint: int = 0
    future: Future = field(default_factory=Future)


class RegistrationServer:
    """slots: registrations in flight; hbm_budget: bytes the requests in flight may hold (None: 80% of the free
    device memory at start); run: the registration callable (default: preopt.register_pair with the given outer
    steps, precision and pre-optimizer), called as run(fixed, moving, grid, weights) on the worker's stream."""

    def __init__(self, slots=4, hbm_budget=None, run=None, outer=200, precision="plain", preopt="native",
                 device="cuda"):
        import torch
        self.slots = int(slots)
        if self.slots < 1:
            raise ValueError("slots >= 1")
        if hbm_budget is None and torch.cuda.is_available():
            free, _ = torch.cuda.mem_get_info()
            hbm_budget = int(.8 * free)
        self.hbm_budget = hbm_budget
        self.device = device
        if run is None:
            from .preopt import NATIVE_PREOPT, register_pair
            cfg = NATIVE_PREOPT if preopt == "native" else preopt

            def run(fixed, moving, grid, weights):
                res, _ = register_pair(fixed, moving, grid, weights, preopt=cfg, outer=outer, precision=precision)
                return res
        self._run = run
        self._cv = threading.Condition()
        self._queue = []
        self._in_use = 0
        self._closed = False
        self.latencies = []
        self._workers = [threading.Thread(target=self._worker, name=f"svp-slot-{k}", daemon=True)
                         for k in range(self.slots)]
        for t in self._workers:
            t.start()

    def submit(self, fixed, moving, grid, weights, tag=None):
        req = Request(fixed, moving, grid, weights, tag, submitted=time.perf_counter(),
                      footprint=footprint_bytes(grid.shape))
        if self.hbm_budget is not None and req.footprint > self.hbm_budget:
            req.future.set_exception(MemoryError(f"request needs ~{req.footprint / 1e9:.1f} GB, budget "
                                                 f"{self.hbm_budget / 1e9:.1f} GB"))
            return req.future
        with self._cv:
            if self._closed:
                raise RuntimeError("server closed")
            self._queue.append(req)
            self._cv.notify_all()
        return req.future

    def _next(self):
        """First queued request (arrival order) whose footprint fits; blocks until one does or the server closes."""
        with self._cv:
            while True:
                for i, req in enumerate(self._queue):
                    if self.hbm_budget is None or self._in_use + req.footprint <= self.hbm_budget:
                        self._in_use += req.footprint
                        return self._queue.pop(i)
                if self._closed and not self._queue:
                    return None
                self._cv.wait()

    def _worker(self):
        stream = None
        try:
            import torch
            if torch.cuda.is_available():
                stream = torch.cuda.Stream(device=self.device)
        except Exception:
            stream = None
        while True:
            req = self._next()
            if req is None:
                return
            req.started = time.perf_counter()
            try:
                if stream is not None:
                    import torch
                    with torch.cuda.stream(stream):
                        res = self._run(req.fixed, req.moving, req.grid, req.weights)
                        stream.synchronize()
                else:
                    res = self._run(req.fixed, req.moving, req.grid, req.weights)
                if not getattr(res, "certified", True):
                    raise RuntimeError(f"registration ended without a certified state: {res.status}")
                req.finished = time.perf_counter()
                with self._cv:
                    self.latencies.append(req.finished - req.submitted)
                req.future.set_result(res)
            except BaseException as exc:          # the request fails, the slot stays open
                req.future.set_exception(exc)
            finally:
                with self._cv:
                    self._in_use -= req.footprint
                    self._cv.notify_all()

    def close(self, wait=True):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        if wait:
            for t in self._workers:
                t.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def percentiles(self, qs=(50, 95, 99)):
        with self._cv:
            lat = list(self.latencies)
        return {f"p{q}": float(np.percentile(lat, q)) for q in qs} if lat else {}
