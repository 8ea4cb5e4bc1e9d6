"""Serving form on the GPU: three registrations admitted together (their own streams and threads) give bit for bit
the results each gets alone, and every returned result is certified."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_results_alone_equal_results_in_the_mix():
    from seq_vp_3d_b200.grid import make_grid_3d
    from seq_vp_3d_b200.preopt import register_pair
    from seq_vp_3d_b200.serve import RegistrationServer
    from seq_vp_3d_b200.synthetic import blob_pair, default_weights
    shape, h = (20, 18, 16), (1., 1., 1.)
    nz, ny, nx = shape
    grid = make_grid_3d(nx=nx, ny=ny, nz=nz, hx=1., hy=1., hz=1., unit="mm")
    w = default_weights(shape, h)
    pairs = [blob_pair(shape, h, seed=s)[:2] for s in (21, 22, 23)]

    def run(fixed, moving, g, weights):
        res, _ = register_pair(fixed, moving, g, weights, preopt=None, outer=4)
        return res
    alone = [run(f, m, grid, w) for f, m in pairs]
    with RegistrationServer(slots=3, run=run) as srv:
        futs = [srv.submit(f, m, grid, w) for f, m in pairs]
        mixed = [fu.result(timeout=600) for fu in futs]
    for a, b in zip(alone, mixed):
        assert a.certified and b.certified
        assert a.status == b.status and a.counts == b.counts
        assert torch.equal(a.final_state.theta, b.final_state.theta)
        assert np.array_equal(a.final_state.energy, b.final_state.energy)
    assert len(srv.latencies) == 3
