"""The backend= adapter's call surface against the reference plug-in's (CPU; no GPU needed).

tests/golden/backend_signatures.json holds the parameter lists of the reference's AcceleratedHybridBackend /
HybridBackend methods and its Poisson object (backends/accelerated.py, backends/hybrid.py), read with inspect by
tests/golden/make_golden.py --only signatures.  A loop written against the reference plug-in calls these methods
with these names, kinds and defaults."""
import inspect
import json
import os

from conftest import GOLDEN


def _params(fn):
    return [[p.name, str(p.kind), None if p.default is inspect.Parameter.empty else repr(p.default)]
            for p in inspect.signature(fn).parameters.values()]


def _golden():
    with open(os.path.join(GOLDEN, "backend_signatures.json")) as f:
        return json.load(f)


def test_backend_methods_match_reference_signatures():
    from seq_vp_3d_b200.backend import B200Backend
    g = _golden()
    for name, params in g["backend"].items():
        assert hasattr(B200Backend, name), name
        assert _params(getattr(B200Backend, name)) == params, name


def test_poisson_object_matches_reference_signatures():
    from seq_vp_3d_b200.backend import _Poisson
    for name, params in _golden()["poisson"].items():
        assert _params(getattr(_Poisson, name)) == params, name


def test_backend_identity_attributes():
    """The reference loops switch to the plug-in's evaluation path when evaluation_backend_id is set
    (sequential.py:203, poisson_gradient.py:1100) and record backend_id; both are class-level facts here."""
    import seq_vp_3d_b200.backend as b
    assert b.BACKEND_ID and "sm100a" in b.BACKEND_ID
    src = inspect.getsource(b.B200Backend.__init__)
    assert "self.evaluation_backend_id" in src and "self.backend_id" in src and "self.device" in src
