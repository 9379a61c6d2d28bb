"""The oracle under cut rows (CrownOracle.compute_bounds(constraints=(A, b))) against the
reference's compute_bounds with PerturbationLpNorm(constraints=...): every concretisation,
intermediate passes included, over box ∩ rows (tests/golden/cuts_*.npz, recorded by
make_cuts_golden.py). Exact-arithmetic McCormick ties against the reference's exact-tie run on
every row; the default rule with the reference's intermediate bounds injected on every row; and
the bounds are sound on sampled feasible points. (They need not be above the bounds without the
rows: the rows change intermediate bounds and so the relaxations.)"""
import numpy as np
import pytest

from golden_cuts import cut_cases, load_cuts
from oracle.crown import EXACT_TIE_TOL, CrownOracle

TOL = 1e-9


def _rel(a, b):
    same = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
    with np.errstate(invalid="ignore"):
        return np.where(same, 0.0, np.abs(a - b) / np.maximum(1.0, np.abs(b)))


@pytest.mark.parametrize("case", cut_cases())
def test_exact_ties_match_reference(case):
    m, g, d, _ = load_cuts(case)
    lb, _, lA, lbias = CrownOracle(g, tie_tol=EXACT_TIE_TOL).compute_bounds(
        d["x_L"], d["x_U"], d["C"], constraints=(d["A"], d["b"]))
    assert _rel(lb, d["lb_exact"]).max() < TOL
    assert _rel(lbias, d["lbias_exact"]).max() < TOL
    assert np.abs(lA - d["lA_exact"]).max() <= TOL * max(1.0, np.abs(d["lA_exact"]).max())


@pytest.mark.parametrize("case", cut_cases())
def test_default_rule_with_reference_intermediates(case):
    m, g, d, inject = load_cuts(case)
    lb, _, lA, lbias = CrownOracle(g, inject=inject).compute_bounds(
        d["x_L"], d["x_U"], d["C"], constraints=(d["A"], d["b"]))
    assert _rel(lb, d["lb"]).max() < TOL
    assert _rel(lbias, d["lbias"]).max() < TOL
    assert np.abs(lA - d["lA"]).max() <= TOL * max(1.0, np.abs(d["lA"]).max())


@pytest.mark.parametrize("case", cut_cases())
def test_bounds_sound_on_feasible_points(case):
    m, g, d, _ = load_cuts(case)
    A, b = d["A"], d["b"]
    lb, _, lA, lbias = CrownOracle(g).compute_bounds(d["x_L"], d["x_U"], d["C"], constraints=(A, b))
    rng = np.random.default_rng(3)
    B, n = d["x_L"].shape
    for bi in range(B):
        pts = d["x_L"][bi] + (d["x_U"][bi] - d["x_L"][bi]) * rng.random((20000, n))
        feas = (pts @ A[bi].T + b[bi] <= 0).all(1)
        if not feas.any():
            continue
        y = g.forward_numpy(pts[feas]) @ d["C"][bi].T
        assert np.all(lb[bi] <= y.min(0) + 1e-9 * np.maximum(1.0, np.abs(y.min(0))))
