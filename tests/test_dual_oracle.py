"""The rigorous dual-bound oracle against the reference's dual_lower_bound and
certify_infeasible (fixtures recorded by tests/golden/make_dual_golden.py): the same
infinite bounds, the same double-double decisions, finite bounds within 1e-14 relative (the
reference's torch reductions and numpy sum in different orders; every order is covered by
the error term), and identical infeasibility verdicts."""
import os
import warnings

import numpy as np
import pytest

from oracle.rigorous_dual import certify_infeasible, dual_lower_bound

GOLD = os.path.join(os.path.dirname(__file__), "golden", "dual.npz")
CASES = ["plain", "infsides", "cancel", "shared", "dense"]


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference(case):
    d = np.load(GOLD)
    g = lambda k: d[f"{case}_{k}"]
    m, n = g("mn")
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        lb, E, dd = dual_lower_bound(g("row"), g("col"), g("val"), m, n, g("c"), g("c0"), g("h"), g("l"), g("u"),
                                     g("y"))
    ref = g("lb")
    assert np.array_equal(np.isinf(lb), np.isinf(ref))
    fin = np.isfinite(ref)
    assert np.all(np.abs(lb - ref)[fin] <= 1e-14 * np.maximum(1.0, np.abs(ref[fin])))
    assert np.array_equal(dd, g("dd"))


def test_farkas_verdicts():
    d = np.load(GOLD)
    g = lambda k: d[f"farkas_{k}"]
    m, n = g("mn")
    v = certify_infeasible(g("row"), g("col"), g("val"), m, n, g("h"), g("l"), g("u"), g("y"))
    assert np.array_equal(v, g("inf")) and v.sum() > 0


def test_bound_below_lp_optimum():
    """lb <= the LP optimum, found by scipy's linprog on a few of the plain-case domains."""
    from scipy.optimize import linprog
    d = np.load(GOLD)
    g = lambda k: d[f"plain_{k}"]
    m, n = g("mn")
    lb = g("lb")
    for b in range(6):
        G = np.zeros((m, n))
        G[g("row"), g("col")] = g("val")[b]
        res = linprog(g("c")[b], A_ub=G, b_ub=g("h")[b], bounds=list(zip(g("l")[b], g("u")[b])), method="highs")
        if res.status == 0:
            assert lb[b] <= res.fun + g("c0")[b] + 1e-9
