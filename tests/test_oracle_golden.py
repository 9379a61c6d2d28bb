"""The CPU oracle against fixtures recorded from the reference implementation.

The fixtures hold the reference's compute_bounds(method='CROWN') outputs and the
intermediate bounds it kept. With those intermediates injected (tie_tol=0, the
reference's float comparison) the oracle must reproduce lb / lA / lbias; its own
intermediates must match the recorded ones. With its own intermediates it must match the
reference's exact-tie run on every row (tie_tol = EXACT_TIE_TOL) and the plain run on every
row the reference determines to 1e-5 under a one-ulp change of its boxes (lb_ulp_dev), and
stay sound against sampling."""
import numpy as np
import pytest

from golden_cases import cases, load
from oracle.crown import CrownOracle, EXACT_TIE_TOL


def _rel(a, b):
    same_inf = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
    with np.errstate(invalid="ignore"):
        return np.where(same_inf, 0.0, np.abs(a - b) / np.maximum(1.0, np.abs(b)))


@pytest.mark.parametrize("case", cases())
def test_oracle_matches_reference_with_injected_intermediates(case):
    m, g, d, inject = load(case)
    o = CrownOracle(g, tie_tol=0.0, inject=inject)
    lb, _, lA, lbias = o.compute_bounds(d["x_L"], d["x_U"], d["C"])
    assert _rel(lb, d["lb"]).max() < 1e-9
    assert np.abs(lA - d["lA"]).max() <= 1e-9 * max(1.0, np.abs(d["lA"]).max())
    assert _rel(lbias, d["lbias"]).max() < 1e-9


@pytest.mark.parametrize("case", cases())
def test_oracle_exact_ties_match_reference_exact_ties(case):
    m, g, d, inject = load(case)
    lb, _, lA, lbias = CrownOracle(g, tie_tol=EXACT_TIE_TOL).compute_bounds(d["x_L"], d["x_U"], d["C"])
    assert _rel(lb, d["lb_exact"]).max() < 1e-9
    assert _rel(lbias, d["lbias_exact"]).max() < 1e-9
    assert np.abs(lA - d["lA_exact"]).max() <= 1e-9 * max(1.0, np.abs(d["lA_exact"]).max())


@pytest.mark.parametrize("case", cases())
def test_oracle_default_matches_reference_on_determined_rows(case):
    m, g, d, inject = load(case)
    lb, _, lA, lbias = CrownOracle(g).compute_bounds(d["x_L"], d["x_U"], d["C"])
    stable = d["lb_ulp_dev"] <= 1e-5
    assert _rel(lb, d["lb"])[stable].max(initial=0.0) < 1e-9
    assert _rel(lbias, d["lbias"])[stable].max(initial=0.0) < 1e-9


@pytest.mark.parametrize("case", cases())
def test_oracle_intermediates_match_reference(case):
    m, g, d, inject = load(case)
    o = CrownOracle(g, tie_tol=0.0, inject=inject)
    o.compute_bounds(d["x_L"], d["x_U"], d["C"])
    for v, (lo, hi) in inject.items():
        if v in o.computed:
            clo, chi = o.computed[v]
            for a, b in ((clo, lo), (chi, hi)):
                assert np.array_equal(np.isfinite(a), np.isfinite(b))
                assert np.array_equal(a[~np.isfinite(b)], b[~np.isfinite(b)])
                fin = np.isfinite(b)
                scale = max(1.0, float(np.abs(b[fin]).max(initial=0.0)))
                assert np.abs(a[fin] - b[fin]).max(initial=0.0) <= 1e-12 * scale


@pytest.mark.parametrize("case", cases())
def test_oracle_pass_order_matches_reference(case):
    m, g, d, inject = load(case)
    o = CrownOracle(g)
    o.compute_bounds(d["x_L"], d["x_U"], d["C"])
    mine = [g[v].width for kind, v in o.log if kind == "crown"]
    ref = [int(p.split(":")[1]) for p in d["passes"]][:-1]
    assert mine == ref


@pytest.mark.parametrize("case", cases())
def test_oracle_default_is_sound_by_sampling(case):
    m, g, d, inject = load(case)
    o = CrownOracle(g)
    lb, _, lA, lbias = o.compute_bounds(d["x_L"], d["x_U"], d["C"])
    rng = np.random.default_rng(0)
    B, n = d["x_L"].shape
    P = 2000 if n < 1000 else 200
    for b in range(B):
        pts = d["x_L"][b] + (d["x_U"][b] - d["x_L"][b]) * rng.random((P, n))
        with np.errstate(invalid="ignore"):
            y = g.forward_numpy(pts) @ d["C"][b].T
        ok = np.isfinite(y).all(1)             # points in the operators' real domain (log > 0)
        pts, y = pts[ok], y[ok]
        if not len(y):
            continue
        assert np.all(lb[b] <= y.min(0) + 1e-9 * np.maximum(1, np.abs(y.min(0))))
        # the returned plane is a valid lower bound too
        plane = pts @ lA[b].T + lbias[b]
        assert np.all(plane <= y + 1e-9 * np.maximum(1, np.abs(y)))
