"""gear_dual_lower_bound (one CTA per domain) against the reference's rigorous_dual fixtures:
the same infinite bounds and double-double decisions, finite bounds within 1e-14 relative
(block reductions sum in another order; the error term covers every order), the same
infeasibility verdicts, and every bound below the LP optimum."""
import os

import numpy as np
import pytest
import torch

from gear_b200.dual import Rows, certify_infeasible, dual_lower_bound

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "dual.npz")
CASES = ["plain", "infsides", "cancel", "shared", "dense"]


def _t(a):
    return torch.tensor(a, dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("case", CASES)
def test_matches_reference(case):
    d = np.load(GOLD)
    g = lambda k: d[f"{case}_{k}"]
    m, n = g("mn")
    rows = Rows(torch.tensor(g("row")), torch.tensor(g("col")), _t(g("val")), m, n)
    lb, E, dd = dual_lower_bound(rows, _t(g("c")), _t(g("c0")), _t(g("h")), _t(g("l")), _t(g("u")), _t(g("y")))
    lb = lb.cpu().numpy()
    ref = g("lb")
    assert np.array_equal(np.isinf(lb), np.isinf(ref))
    fin = np.isfinite(ref)
    assert np.all(np.abs(lb - ref)[fin] <= 1e-14 * np.maximum(1.0, np.abs(ref[fin])))
    assert np.array_equal(dd.cpu().numpy(), g("dd"))


def test_farkas_verdicts():
    d = np.load(GOLD)
    g = lambda k: d[f"farkas_{k}"]
    m, n = g("mn")
    rows = Rows(torch.tensor(g("row")), torch.tensor(g("col")), _t(g("val")), m, n)
    v = certify_infeasible(rows, _t(g("h")), _t(g("l")), _t(g("u")), _t(g("y")))
    assert np.array_equal(v.cpu().numpy(), g("inf"))


def test_below_lp_optimum_random():
    from scipy.optimize import linprog
    g = np.random.default_rng(7)
    B, m, n = 64, 9, 14
    G = g.normal(size=(B, m, n)) * (g.random((m, n)) < 0.5)
    h = g.random((B, m)) + 0.5
    l, u = -g.random((B, n)) - 0.1, g.random((B, n)) + 0.1
    c = g.normal(size=(B, n))
    c0 = g.normal(size=B)
    y = g.random((B, m)) * 0.5
    rows = Rows.from_dense(_t(G))
    lb, _, _ = dual_lower_bound(rows, _t(c), _t(c0), _t(h), _t(l), _t(u), _t(y))
    lb = lb.cpu().numpy()
    for b in range(0, B, 8):
        res = linprog(c[b], A_ub=G[b], b_ub=h[b], bounds=list(zip(l[b], u[b])), method="highs")
        assert res.status == 0 and lb[b] <= res.fun + c0[b]
