"""CROWN under cut rows on the GPU (gear_crown_lower_cuts, CutEngine, BoundedModule with
PerturbationLpNorm(constraints=(A, b))): every concretisation, the intermediate passes' included,
over box ∩ rows, against the reference's own outputs (tests/golden/cuts_*.npz, recorded by
make_cuts_golden.py) and the oracle.

* Exact-arithmetic McCormick ties against the reference's exact-tie run: every row of every
  fixture within 1e-9 relative (lb, lbias; lA scaled by its largest entry).
* The same call against the oracle's CrownOracle.compute_bounds(constraints=...) with exact ties:
  every row within 1e-9, on the fixtures and on seeded quad_exp_n10 batches with rows that cut
  every box and a zero-row call (K = 0).
* Default tie rule: sound on sampled feasible points (lb <= min f over 2 * 10^4 uniform points that
  satisfy the rows), and the drop-in surface returns the engine's bounds bit for bit.
* Branch and bound with cuts at every concretisation closes the same instance as the final-row
  form, to the same incumbent."""
import numpy as np
import pytest
import torch

from golden_cuts import cut_cases, load_cuts
from gear_b200 import graph, problems
from gear_b200.engine import CutEngine
from oracle.crown import EXACT_TIE_TOL, CrownOracle

pytestmark = pytest.mark.gpu
TOL = 1e-9


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    same = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
    with np.errstate(invalid="ignore"):
        return np.where(same, 0.0, np.abs(a - b) / np.maximum(1.0, np.abs(b)))


def _gpu(g, xL, xU, A, b, C=None, tie_rule="exact", threads=128):
    eng = CutEngine(g, spec_rows=None if C is None else C.shape[1], dense_c=C is not None, cta_threads=threads,
                    tie_rule=tie_rule)
    dev = "cuda"
    out = eng.lower(torch.as_tensor(xL, device=dev), torch.as_tensor(xU, device=dev),
                    None if A is None else torch.as_tensor(A, device=dev),
                    None if b is None else torch.as_tensor(b, device=dev),
                    None if C is None else torch.as_tensor(C, device=dev))
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in out], eng


@pytest.mark.parametrize("case", cut_cases())
@pytest.mark.parametrize("threads", [64, 128, 256])
def test_exact_ties_match_reference_every_row(case, threads):
    m, g, d, _ = load_cuts(case)
    (lb, lA, lbias), eng = _gpu(g, d["x_L"], d["x_U"], d["A"], d["b"], threads=threads)
    assert eng.launches > 0
    assert _rel(lb, d["lb_exact"]).max() < TOL
    assert _rel(lbias, d["lbias_exact"]).max() < TOL
    assert np.abs(lA - d["lA_exact"]).max() <= TOL * max(1.0, np.abs(d["lA_exact"]).max())


@pytest.mark.parametrize("case", cut_cases())
def test_matches_oracle_with_cuts(case):
    m, g, d, _ = load_cuts(case)
    (lb, lA, lbias), _ = _gpu(g, d["x_L"], d["x_U"], d["A"], d["b"])
    olb, _, olA, olbias = CrownOracle(g, tie_tol=EXACT_TIE_TOL).compute_bounds(
        d["x_L"], d["x_U"], constraints=(d["A"], d["b"]))
    assert _rel(lb, olb).max() < TOL
    assert _rel(lbias, olbias).max() < TOL
    assert np.abs(lA - olA).max() <= TOL * max(1.0, np.abs(olA).max())


def _cut_rows(lo, hi, K, seed, t_lo=-1.0, t_hi=0.4):
    g = np.random.default_rng(seed)
    B, n = lo.shape
    A = g.standard_normal((B, K, n))
    t = g.uniform(t_lo, t_hi, (B, K))
    x0, eps = (lo + hi) / 2, (hi - lo) / 2
    b = -(A * x0[:, None]).sum(-1) + t * (np.abs(A) * eps[:, None]).sum(-1)
    return A, b


@pytest.mark.parametrize("K", [0, 3, 8])
def test_seeded_batches_match_oracle(K):
    m = problems.make_instance("quad_exp_n10", 2)
    lo, hi = problems.make_boxes("quad_exp_n10", 40, 2)
    g = graph.trace(m, lo[:2])
    xL, xU = lo.numpy(), hi.numpy()
    A, b = _cut_rows(xL, xU, K, 11 + K)
    (lb, lA, lbias), _ = _gpu(g, xL, xU, A, b)
    olb, _, olA, olbias = CrownOracle(g, tie_tol=EXACT_TIE_TOL).compute_bounds(xL, xU, constraints=(A, b))
    assert _rel(lb, olb).max() < TOL
    assert _rel(lbias, olbias).max() < TOL
    assert np.abs(lA - olA).max() <= TOL * max(1.0, np.abs(olA).max())


@pytest.mark.parametrize("case", cut_cases())
def test_default_rule_sound_on_feasible_points(case):
    m, g, d, _ = load_cuts(case)
    A, b = d["A"], d["b"]
    (lb, lA, lbias), _ = _gpu(g, d["x_L"], d["x_U"], A, b, tie_rule="reference")
    rng = np.random.default_rng(5)
    B, n = d["x_L"].shape
    checked = 0
    for bi in range(B):
        pts = d["x_L"][bi] + (d["x_U"][bi] - d["x_L"][bi]) * rng.random((20000, n))
        feas = (pts @ A[bi].T + b[bi] <= 0).all(1)
        if not feas.any():
            continue
        y = g.forward_numpy(pts[feas])
        assert np.all(lb[bi] <= y.min(0) + 1e-9 * np.maximum(1.0, np.abs(y.min(0))))
        checked += 1
    assert checked > 0


def test_bounded_module_with_constraints():
    from gear_b200.bounded import BoundedModule, BoundedTensor, PerturbationLpNorm
    m, g, d, _ = load_cuts(cut_cases()[0])
    n = d["x_L"].shape[1]
    dev = "cuda"
    xL, xU = torch.as_tensor(d["x_L"], device=dev), torch.as_tensor(d["x_U"], device=dev)
    A, b = torch.as_tensor(d["A"], device=dev), torch.as_tensor(d["b"], device=dev)
    bm = BoundedModule(m, torch.zeros(2, n, dtype=torch.float64), device=dev)
    x = BoundedTensor((xL + xU) / 2, PerturbationLpNorm(x_L=xL, x_U=xU, constraints=(A, b)))
    lb, _, Ad = bm.compute_bounds(x=(x,), method="CROWN", bound_upper=False, return_A=True,
                                  needed_A_dict={"/y": {"/x"}})
    (elb, elA, elbias), _ = _gpu(g, d["x_L"], d["x_U"], d["A"], d["b"], tie_rule="reference")
    assert np.array_equal(lb.cpu().numpy(), elb)
    assert np.array_equal(Ad["/y"]["/x"]["lA"].cpu().numpy(), elA)
    assert np.array_equal(Ad["/y"]["/x"]["lbias"].cpu().numpy(), elbias)


def test_bab_with_cuts_everywhere_closes_like_final_row_form():
    from gear_b200.bab import BaB
    m = problems.make_instance("quad_exp_n10", 0)
    lo, hi = problems.root_box("quad_exp_n10")
    g = graph.trace(m, lo.repeat(2, 1))
    m = m.cuda()
    res = {}
    for every in (True, False):
        bab = BaB(g, lo, hi, batch=256, model=m, constrained=True, cuts_everywhere=every, engine_mode="cta")
        bab.run(rel_gap=1e-4, time_limit=60.0)
        res[every] = bab
        assert bab.gap() <= 1e-4
    assert res[True].cut_engine is not None and res[False].cut_engine is None
    a, b_ = res[True].incumbent, res[False].incumbent
    assert abs(a - b_) <= 1e-4 * max(1.0, abs(a), abs(b_))


@pytest.mark.parametrize("case", cut_cases()[:2])
def test_dense_specification_rows_match_oracle(case):
    """A dense specification C (B, S', w) with cut rows: the engine compiled for C (dense_c) against
    the oracle's compute_bounds(C, constraints) with exact ties, every row to 1e-9."""
    m, g, d, _ = load_cuts(case)
    B = d["x_L"].shape[0]
    w = g[g.output].width
    rng = np.random.default_rng(17)
    C = rng.standard_normal((B, 2, w))
    (lb, lA, lbias), _ = _gpu(g, d["x_L"], d["x_U"], d["A"], d["b"], C=C)
    olb, _, olA, olbias = CrownOracle(g, tie_tol=EXACT_TIE_TOL).compute_bounds(
        d["x_L"], d["x_U"], C, constraints=(d["A"], d["b"]))
    assert _rel(lb, olb).max() < TOL
    assert _rel(lbias, olbias).max() < TOL
    assert np.abs(lA - olA).max() <= TOL * max(1.0, np.abs(olA).max())
