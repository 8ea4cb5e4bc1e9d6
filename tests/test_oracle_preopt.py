"""The float64 restatement of the pre-objective and its analytic gradient (oracle/preopt.py) against the reference's
own autograd values (golden preopt.npz, generated with the reference's float64 pre-objective)."""
import os

import numpy as np

from conftest import GOLDEN
from oracle import preopt as O


def test_pre_objective_and_gradient_match_reference_autograd():
    d = np.load(os.path.join(GOLDEN, "preopt.npz"))
    terms, grad = O.pre_energy_grad(d["pre_F"], d["pre_M"], tuple(d["pre_spacing"]), d["pre_u"], .3, 1e-3, 10., .2)
    ref = d["pre_terms_f64"]
    assert np.all(np.abs(terms - ref) <= 1e-12 * np.maximum(np.abs(ref), 1e-3)), (terms, ref)
    gr = d["pre_grad_f64"]
    assert np.linalg.norm(grad - gr) <= 1e-12 * np.linalg.norm(gr)
