"""Final-state export in the reference's output formats (docs/usage.md section 4; scripts/run_stage_3d_e19_mri.py:2048
save('final_native.npz', u=..., warped=...) and :2054 final_native.json).

final_native.npz   u: (nz, ny, nx, 3) float64 displacement in mm, components (x, y, z); warped: the warped moving image
final_native.json  {path, sha256, role, certificate: the FeasibilityResult record of the final state}
summary.json       status, reason, energies, GF and threshold, MSE (native and final) and their ratio, counts, timings

The exported u is the certified state's u (its bytes, copied once from the device); any certifier can re-prove it
(the reference's certify_map, or this package's certify_map on the same array).
"""
import hashlib
import json
import os
from dataclasses import asdict

import numpy as np

ROLE = "certified_native_final_state"


def _sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


def _plain(v):
    if isinstance(v, (np.floating, np.integer)):
        return v.item()
    if isinstance(v, np.ndarray):
        return v.tolist()
    if isinstance(v, dict):
        return {k: _plain(x) for k, x in v.items()}
    if isinstance(v, (list, tuple)):
        return [_plain(x) for x in v]
    return v


def export_final(result, out_dir, extra=None):
    """Write final_native.npz, final_native.json and summary.json for a SequentialResult; returns the json record."""
    state = result.final_state
    if state is None:
        raise ValueError("no final state to export")
    if state.certificate.status != "certified_feasible":
        raise ValueError("only certified states are exported")
    os.makedirs(out_dir, exist_ok=True)
    u = state.u.detach().cpu().numpy() if hasattr(state.u, "detach") else np.asarray(state.u)
    warped = state.warped.detach().cpu().numpy() if hasattr(state.warped, "detach") else np.asarray(state.warped)
    path = os.path.join(out_dir, "final_native.npz")
    np.savez(path, u=u, warped=warped)
    cert = asdict(state.certificate)
    cert.pop("config", None)
    record = dict(path="final_native.npz", sha256=_sha256(path), role=ROLE, certificate=_plain(cert))
    with open(os.path.join(out_dir, "final_native.json"), "w") as f:
        json.dump(record, f, indent=1)
    e = [float(x) for x in state.energy]
    summary = dict(status=result.status, reason=result.reason,
                   energy=dict(image=e[0], proximity=e[1], jd=e[2], curl=e[3], barrier=e[4], total=state.total,
                               outer=state.outer),
                   GF_initial=result.GF_initial, GF_final=result.GF_final, GF_threshold=result.GF_threshold,
                   native_mse=result.native_mse, final_mse=result.final_mse,
                   mse_ratio=None if not result.native_mse else result.final_mse / result.native_mse,
                   counts=_plain(result.counts), elapsed_seconds=result.elapsed_seconds,
                   timings=_plain(result.timings), **_plain(extra or {}))
    with open(os.path.join(out_dir, "summary.json"), "w") as f:
        json.dump(summary, f, indent=1)
    return record
