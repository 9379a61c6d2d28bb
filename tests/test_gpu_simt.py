"""Box-per-thread CROWN kernel (crown_simt_kernel) against the float64 CPU oracle and against
the box-per-CTA kernel. Tolerance: 1e-9 relative (same rounding model; the two kernels sum in
different orders, so McCormick ties are decided in exact arithmetic, tie_rule "exact", on every
side of these comparisons)."""
import numpy as np
import pytest
import torch

from golden_cases import cases, load
from gear_b200 import BoundedModule, BoundedTensor, PerturbationLpNorm, problems
from gear_b200.engine import CrownEngine
from oracle.crown import CrownOracle, EXACT_TIE_TOL

pytestmark = pytest.mark.gpu
RTOL = 1e-9


def _close(a, b, rtol=RTOL):
    a, b = np.asarray(a), np.asarray(b)
    both_inf = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
    err = np.where(both_inf, 0.0, np.abs(a - b) / np.maximum(1.0, np.abs(b)))
    return float(np.nanmax(err)) if err.size else 0.0


@pytest.mark.parametrize("case", cases())
def test_simt_matches_oracle_on_fixture_boxes(case):
    m, g, d, inject = load(case)
    eng = CrownEngine(g, mode="simt", tie_rule="exact")
    lo = torch.tensor(d["x_L"], device="cuda")
    hi = torch.tensor(d["x_U"], device="cuda")
    lb, lA, lbias = eng.lower(lo, hi)
    torch.cuda.synchronize()
    olb, _, olA, olbias = CrownOracle(g, tie_tol=EXACT_TIE_TOL).compute_bounds(d["x_L"], d["x_U"], d["C"])
    assert _close(lb.cpu().numpy(), olb) < RTOL
    # On a degenerate box a power's relaxation is a secant over the reference's 1e-8 widening:
    # its slope amplifies the last-bit difference of pow (torch on the CPU vs CUDA) by ~1e8, so
    # the planes (lA, lbias) there agree to 1e-6; the bound itself still agrees to RTOL.
    lA_, lbias_ = lA.cpu().numpy(), lbias.cpu().numpy()
    flat = (d["x_U"] - d["x_L"]).min(1) < 1e-6
    tol = np.where(flat & any(nd.kind == "pow" for nd in g.nodes), 1e-6, RTOL)
    for b in range(lA_.shape[0]):
        assert _close(lA_[b], olA[b]) < tol[b]
        assert _close(lbias_[b], olbias[b]) < tol[b]


# batches that are not a multiple of the 64-box tile exercise the tail threads
@pytest.mark.parametrize("workload,batch", [("quad_exp_n10", 300), ("dense_q_n200", 70)])
def test_simt_matches_oracle_random_boxes(workload, batch):
    m = problems.make_instance(workload, 0)
    lo, hi = problems.make_boxes(workload, batch, 0)
    bm = BoundedModule(m, lo[:2], device="cuda", bound_opts={"gear_mode": "simt", "gear_tie_rule": "exact"})
    x = BoundedTensor(lo.cuda(), PerturbationLpNorm(x_L=lo.cuda(), x_U=hi.cuda()))
    S = bm.final_node_width()
    C = torch.eye(S, dtype=torch.float64).expand(batch, S, S)
    lb, _, A = bm.compute_bounds(x=(x,), C=C.cuda(), method="CROWN", bound_upper=False, return_A=True)
    rec = A[bm.output_name[0]][bm.input_name[0]]
    olb, _, olA, olbias = CrownOracle(bm.graph, tie_tol=EXACT_TIE_TOL).compute_bounds(lo.numpy(), hi.numpy(),
                                                                                       C.numpy())
    assert _close(lb.cpu().numpy(), olb) < RTOL
    assert _close(rec["lA"].cpu().numpy(), olA) < RTOL
    assert _close(rec["lbias"].cpu().numpy(), olbias) < RTOL


def test_simt_dense_c_matches_oracle():
    m = problems.make_instance("quad_exp_n10", 1)
    lo, hi = problems.make_boxes("quad_exp_n10", 32, 1)
    g = torch.Generator().manual_seed(3)
    C = torch.randn(32, 2, 3, generator=g, dtype=torch.float64)
    bm = BoundedModule(m, lo[:2], device="cuda", bound_opts={"gear_mode": "simt"})
    x = BoundedTensor(lo.cuda(), PerturbationLpNorm(x_L=lo.cuda(), x_U=hi.cuda()))
    lb, _, A = bm.compute_bounds(x=(x,), C=C.cuda(), method="CROWN", bound_upper=False, return_A=True)
    olb, _, olA, _ = CrownOracle(bm.graph).compute_bounds(lo.numpy(), hi.numpy(), C.numpy())
    assert _close(lb.cpu().numpy(), olb) < RTOL
    assert _close(A["/y"]["/x"]["lA"].cpu().numpy(), olA) < RTOL


@pytest.mark.parametrize("workload,batch", [("quad_exp_n10", 4096), ("dense_q_n200", 1000),
                                            ("dense_a_n2048", 64)])
def test_simt_matches_cta_kernel(workload, batch):
    m = problems.make_instance(workload, 0)
    lo, hi = problems.make_boxes(workload, batch, 0)
    from gear_b200 import graph
    g = graph.trace(m, lo[:2])
    xL, xU = lo.cuda(), hi.cuda()
    a = CrownEngine(g, mode="cta", tie_rule="exact").lower(xL, xU)
    b = CrownEngine(g, mode="simt", tie_rule="exact").lower(xL, xU)
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert _close(y.cpu().numpy(), x.cpu().numpy()) < RTOL
