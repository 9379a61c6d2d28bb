"""The constrained-concretisation oracle against the reference's own sort_out_constr_batches +
constraints_solving (fixtures recorded by tests/golden/make_concretize_golden.py) and against
the reference test's known answer (test_constrained_concretize.py: box [-1,2]x[-2,1] with
x0 + x1 + 2 <= 0 gives lower bounds (-1, -2))."""
import os
import warnings

import numpy as np
import pytest

from oracle.concretize import constrained_lower

GOLD = os.path.join(os.path.dirname(__file__), "golden", "concretize.npz")
CASES = sorted({k.rsplit("_", 1)[0] for k in np.load(GOLD).files})


def rel_err(a, b):
    both_inf = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
    return float(np.max(np.where(both_inf, 0.0, np.abs(a - b) / np.maximum(1.0, np.abs(b)))))


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference(case):
    d = np.load(GOLD)
    cap = int(case.split("cap")[1])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        lb = constrained_lower(d[case + "_xl"], d[case + "_xu"], d[case + "_obj"], d[case + "_A"], d[case + "_b"],
                               max_rows=cap)
    ref = d[case + "_lb"]
    assert np.array_equal(np.isposinf(lb), np.isposinf(ref))       # infeasible boxes
    assert rel_err(lb, ref) < 1e-12


def test_known_answer():
    lb = constrained_lower(np.array([[-1.0, -2.0]]), np.array([[2.0, 1.0]]), np.eye(2)[None],
                           np.array([[[1.0, 1.0]]]), np.array([[2.0]]))
    assert np.allclose(lb, [[-1.0, -2.0]], rtol=0, atol=1e-12)


def test_rows_only_tighten_and_stay_sound():
    """Every lower bound is at most the true minimum over sampled feasible points."""
    d = np.load(GOLD)
    case = "small_cap0"
    xl, xu, obj, A, b = (d[case + s] for s in ("_xl", "_xu", "_obj", "_A", "_b"))
    lb = d[case + "_lb"]
    rng = np.random.default_rng(0)
    for bi in range(xl.shape[0]):
        x = xl[bi] + (xu[bi] - xl[bi]) * rng.random((4000, xl.shape[1]))
        feas = (x @ A[bi].T + b[bi] <= 0).all(1)
        if not feas.any():
            continue
        vals = x[feas] @ obj[bi].T
        assert np.all(lb[bi] <= vals.min(0) + 1e-9)
