"""GPU CROWN (libgear_b200.so megakernel) against the float64 CPU oracle. Tolerance: 1e-9
relative (same rounding model). Both sides decide McCormick ties in exact arithmetic
(tie_rule "exact"), so the comparison does not depend on the last bits of the two
implementations' summation orders; the default rule is compared with the reference's own
outputs in test_gpu_reference.py."""
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
@pytest.mark.parametrize("threads", [64, 128, 256])
def test_gpu_matches_oracle_on_fixture_boxes(case, threads):
    """Every box-per-CTA kernel instance (64, 128, 256 threads) against the oracle."""
    m, g, d, inject = load(case)
    eng = CrownEngine(g, mode="cta", cta_threads=threads, tie_rule="exact")
    lo = torch.tensor(d["x_L"], device="cuda")
    hi = torch.tensor(d["x_U"], device="cuda")
    lb, lA, lbias = eng.lower(lo, hi)
    torch.cuda.synchronize()
    o = CrownOracle(g, tie_tol=EXACT_TIE_TOL)
    olb, _, olA, olbias = o.compute_bounds(d["x_L"], d["x_U"], d["C"])
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


@pytest.mark.parametrize("workload,batch", [("quad_exp_n10", 256), ("dense_q_n200", 64)])
def test_gpu_matches_oracle_random_boxes(workload, batch):
    m = problems.make_instance(workload, 0)
    lo, hi = problems.make_boxes(workload, batch, 0)
    bm = BoundedModule(m, lo[:2], device="cuda", bound_opts={"gear_tie_rule": "exact"})
    x = BoundedTensor(lo.cuda(), PerturbationLpNorm(x_L=lo.cuda(), x_U=hi.cuda()))
    S = bm.final_node_width()
    C = torch.eye(S, dtype=torch.float64).expand(batch, S, S)
    lb, _, A = bm.compute_bounds(x=(x,), C=C.cuda(), method="CROWN", bound_upper=False, return_A=True)
    rec = A[bm.output_name[0]][bm.input_name[0]]
    o = CrownOracle(bm.graph, tie_tol=EXACT_TIE_TOL)
    olb, _, olA, olbias = o.compute_bounds(lo.numpy(), hi.numpy(), C.numpy())
    assert _close(lb.cpu().numpy(), olb) < RTOL
    assert _close(rec["lA"].cpu().numpy(), olA) < RTOL
    assert _close(rec["lbias"].cpu().numpy(), olbias) < RTOL


def test_gpu_dense_c_matches_oracle():
    m = problems.make_instance("quad_exp_n10", 1)
    lo, hi = problems.make_boxes("quad_exp_n10", 32, 1)
    g = torch.Generator().manual_seed(3)
    C = torch.randn(32, 2, 3, generator=g, dtype=torch.float64)
    bm = BoundedModule(m, lo[:2], device="cuda")
    x = BoundedTensor(lo.cuda(), PerturbationLpNorm(x_L=lo.cuda(), x_U=hi.cuda()))
    lb, _, A = bm.compute_bounds(x=(x,), C=C.cuda(), method="CROWN", bound_upper=False, return_A=True)
    o = CrownOracle(bm.graph)
    olb, _, olA, _ = o.compute_bounds(lo.numpy(), hi.numpy(), C.numpy())
    assert _close(lb.cpu().numpy(), olb) < RTOL
    assert _close(A["/y"]["/x"]["lA"].cpu().numpy(), olA) < RTOL


@pytest.mark.parametrize("workload,batch", [("quad_exp_n10", 2048), ("dense_q_n200", 300)])
def test_auto_engine_picks_a_variant_and_matches_oracle(workload, batch):
    """mode="auto" times the variants on the first call and every later call uses the pick."""
    from gear_b200 import graph
    m = problems.make_instance(workload, 0)
    lo, hi = problems.make_boxes(workload, batch, 0)
    g = graph.trace(m, lo[:2])
    eng = CrownEngine(g, mode="auto", tie_rule="exact")
    first = eng.lower(lo.cuda(), hi.cuda())
    second = eng.lower(lo.cuda(), hi.cuda())
    torch.cuda.synchronize()
    assert eng.variant(batch) in {"simt", "cta64", "cta128", "cta256"}
    assert len(eng.timings) == 1
    for a, b in zip(first, second):
        assert torch.equal(a, b)           # same variant, same arithmetic: bit-identical
    olb, _, olA, olbias = CrownOracle(g, tie_tol=EXACT_TIE_TOL).compute_bounds(lo.numpy(), hi.numpy())
    assert _close(first[0].cpu().numpy(), olb) < RTOL
    assert _close(first[1].cpu().numpy(), olA) < RTOL


def test_gpu_bounds_of_a_lowered_node_program():
    """A NodeProgram from the reference's gear front end, lowered to the IR, bounds on the GPU
    exactly like the directly traced model."""
    import os
    from gear_b200.lowering import ProgramModule
    data = torch.load(os.path.join(os.path.dirname(__file__), "golden", "programs.pt"), weights_only=False)
    p = data["programs"]["dense_q_n200"]
    m = problems.make_instance("dense_q_n200", 0)
    lo, hi = problems.make_boxes("dense_q_n200", 96, 0)
    prog = ProgramModule(p["nodes_op"], p["nodes_in"], p["nodes_out"])
    opts = {"gear_mode": "cta"}            # one kernel for both: identical arithmetic
    a = BoundedModule(prog, lo[:2], device="cuda", bound_opts=opts)
    b = BoundedModule(m, lo[:2], device="cuda", bound_opts=opts)
    x = BoundedTensor(lo.cuda(), PerturbationLpNorm(x_L=lo.cuda(), x_U=hi.cuda()))
    la, _, Aa = a.compute_bounds(x=(x,), method="CROWN", bound_upper=False, return_A=True)
    lb, _, Ab = b.compute_bounds(x=(x,), method="CROWN", bound_upper=False, return_A=True)
    assert torch.equal(la, lb)
    assert torch.equal(Aa["/y"]["/x"]["lA"], Ab["/y"]["/x"]["lA"])


@pytest.mark.parametrize("key", ["quad_exp_n10_0_eye", "dense_q_n200_0_eye", "quad_exp_n10_1_dense", "pow_ops_0_eye"])
def test_gpu_ibp_pass_matches_reference(key):
    """gear_crown_lower_ibp: lb_ibp equals the reference's IBP pass (fixtures, 1e-13) and lb is
    the larger of it and the CROWN bound."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from test_ibp_pass import model_graph
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "ibp_out.npz"))
    _, g = model_graph(key)
    dense = key.endswith("dense")
    C = torch.tensor(d[key + "_C"], device="cuda")
    eng = CrownEngine(g, spec_rows=C.shape[1], dense_c=dense, mode="cta")
    xL, xU = torch.tensor(d[key + "_xL"], device="cuda"), torch.tensor(d[key + "_xU"], device="cuda")
    lb_ibp = torch.empty(xL.shape[0], C.shape[1], dtype=torch.float64, device="cuda")
    lb, _, _ = eng.lower(xL, xU, C if dense else None, lb_ibp=lb_ibp)
    plain, _, _ = eng.lower(xL, xU, C if dense else None)
    torch.cuda.synchronize()
    ref = d[key + "_lb"]
    got = lb_ibp.cpu().numpy()
    assert np.max(np.abs(got - ref) / np.maximum(1.0, np.abs(ref))) < 1e-13
    assert torch.equal(lb, torch.maximum(plain, lb_ibp))


def test_compute_bounds_host_matches_device_call():
    """The pipelined host-buffer call (chunks not dividing the batch) gives the device call's bits."""
    m = problems.make_instance("dense_q_n200", 0)
    lo, hi = problems.make_boxes("dense_q_n200", 1000, 0)
    bm = BoundedModule(m, lo[:2], device="cuda", bound_opts={"gear_mode": "cta", "gear_cta_threads": 128})
    hL, hU = lo.pin_memory(), hi.pin_memory()
    lb_h = bm.compute_bounds_host(hL, hU, chunk=300)
    lb_h2 = bm.compute_bounds_host(hL.flip(0).contiguous().pin_memory(), hU.flip(0).contiguous().pin_memory(),
                                   chunk=300)            # a second call right behind the first
    x = BoundedTensor(lo.cuda(), PerturbationLpNorm(x_L=lo.cuda(), x_U=hi.cuda()))
    lb_d, _ = bm.compute_bounds(x=(x,), method="CROWN", bound_upper=False)
    torch.cuda.synchronize()
    assert torch.equal(lb_h, lb_d.cpu())
    assert torch.equal(lb_h2, lb_d.cpu().flip(0))


def test_compute_bounds_host_small_batch_and_empty():
    m = problems.make_instance("quad_exp_n10", 0)
    lo, hi = problems.make_boxes("quad_exp_n10", 37, 0)
    bm = BoundedModule(m, lo[:2], device="cuda", bound_opts={"gear_mode": "simt"})
    lb_h = bm.compute_bounds_host(lo.pin_memory(), hi.pin_memory(), chunk=4096)   # one partial chunk
    x = BoundedTensor(lo.cuda(), PerturbationLpNorm(x_L=lo.cuda(), x_U=hi.cuda()))
    lb_d, _ = bm.compute_bounds(x=(x,), method="CROWN", bound_upper=False)
    torch.cuda.synchronize()
    assert torch.equal(lb_h, lb_d.cpu())
    assert bm.compute_bounds_host(lo[:0], hi[:0]).shape == (0, 3)
