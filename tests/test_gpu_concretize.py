"""gear_constrained_lower (device dual sweep) against the reference fixtures, the oracle
(same algorithm in numpy) and the reference test's known answer. Tolerance 1e-9 relative;
infeasible boxes must match exactly."""
import os
import warnings

import numpy as np
import pytest
import torch

from gear_b200.concretize import constraints_solving
from oracle.concretize import constrained_lower

pytestmark = pytest.mark.gpu
RTOL = 1e-9
GOLD = os.path.join(os.path.dirname(__file__), "golden", "concretize.npz")
CASES = sorted({k.rsplit("_", 1)[0] for k in np.load(GOLD).files})


def rel_err(a, b):
    both_inf = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
    return float(np.max(np.where(both_inf, 0.0, np.abs(a - b) / np.maximum(1.0, np.abs(b)))))


def _gpu(xl, xu, obj, A, b, cap=0, sign=-1.0):
    t = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")
    out, inf = constraints_solving(t(xl), t(xu), t(obj), (t(A), t(b)), sign=sign, max_rows=cap,
                                   return_infeasible=True)
    torch.cuda.synchronize()
    return out[..., 0].cpu().numpy(), inf.cpu().numpy()


@pytest.mark.parametrize("case", CASES)
def test_matches_reference_fixtures(case):
    d = np.load(GOLD)
    cap = int(case.split("cap")[1])
    lb, inf = _gpu(*(d[case + s] for s in ("_xl", "_xu", "_obj", "_A", "_b")), cap=cap)
    ref = d[case + "_lb"]
    assert np.array_equal(np.isposinf(lb), np.isposinf(ref))
    assert rel_err(lb, ref) < RTOL


def test_known_answer_both_sides():
    xl, xu = np.array([[-1.0, -2.0]]), np.array([[2.0, 1.0]])
    A, b = np.array([[[1.0, 1.0]]]), np.array([[2.0]])
    lo, _ = _gpu(xl, xu, np.eye(2)[None], A, b, sign=-1.0)
    hi, _ = _gpu(xl, xu, np.eye(2)[None], A, b, sign=1.0)
    assert np.allclose(lo, [[-1.0, -2.0]], atol=1e-12)
    assert np.allclose(hi, [[0.0, -1.0]], atol=1e-12)


@pytest.mark.parametrize("B,H,X,K,cap", [(256, 2, 30, 10, 0), (128, 1, 200, 16, 0), (96, 3, 17, 24, 5)])
def test_matches_oracle_random(B, H, X, K, cap):
    g = np.random.default_rng(B + X)
    c = g.uniform(-2, 2, (B, X))
    w = g.uniform(0.05, 0.95, (B, X))
    xl, xu = c - w, c + w
    obj = g.normal(size=(B, H, X))
    A = g.normal(size=(B, K, X))
    t = g.uniform(-1.3, 1.05, (B, K))
    b = -(A * ((xl + xu) / 2)[:, None]).sum(-1) + t * (np.abs(A) * ((xu - xl) / 2)[:, None]).sum(-1)
    lb, inf = _gpu(xl, xu, obj, A, b, cap=cap)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        ref = constrained_lower(xl, xu, obj, A, b, max_rows=cap)
    assert np.array_equal(np.isposinf(lb), np.isposinf(ref))
    assert np.array_equal(inf.astype(bool), np.isposinf(ref).any(1))
    assert rel_err(lb, ref) < RTOL


def test_no_rows_is_the_box_bound():
    g = np.random.default_rng(3)
    xl = g.uniform(-1, 0, (10, 7)); xu = xl + g.uniform(0, 1, (10, 7))
    obj = g.normal(size=(10, 2, 7))
    t = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")
    out = constraints_solving(t(xl), t(xu), t(obj), None)[..., 0].cpu().numpy()
    ref = constrained_lower(xl, xu, obj, None, None)
    assert rel_err(out, ref) < RTOL
