"""Edge cases of the device path against the oracle: empty and single-box batches, degenerate
boxes, boxes wide enough to overflow exp (undefined relaxation rows, interval fallback),
infinite input bounds, and empty BaB steps. Tolerance 1e-9 relative; infinities must match."""
import numpy as np
import pytest
import torch

from gear_b200 import graph, problems
from gear_b200.engine import CrownEngine
from oracle.crown import CrownOracle

pytestmark = pytest.mark.gpu
RTOL = 1e-9
VARIANTS = [("cta", 64), ("cta", 128), ("cta", 256), ("simt", 128)]


def _close(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert np.array_equal(np.isinf(a) & (a > 0), np.isinf(b) & (b > 0))
    assert np.array_equal(np.isinf(a) & (a < 0), np.isinf(b) & (b < 0))
    fin = np.isfinite(a) & np.isfinite(b)
    return float(np.max(np.abs(a - b)[fin] / np.maximum(1.0, np.abs(b[fin])))) if fin.any() else 0.0


def _graph():
    m = problems.make_instance("quad_exp_n10", 0)
    return m, graph.trace(m, torch.zeros(2, 10, dtype=torch.float64))


@pytest.mark.parametrize("mode,threads", VARIANTS)
def test_empty_and_single_box(mode, threads):
    m, g = _graph()
    eng = CrownEngine(g, mode=mode, cta_threads=threads)
    e = torch.empty(0, 10, dtype=torch.float64, device="cuda")
    lb, lA, lbias = eng.lower(e, e)
    assert lb.shape == (0, 3) and lA.shape == (0, 3, 10)
    lo, hi = problems.make_boxes("quad_exp_n10", 1, 0)
    lb, lA, lbias = eng.lower(lo.cuda(), hi.cuda())
    olb, _, olA, olbias = CrownOracle(g).compute_bounds(lo.numpy(), hi.numpy())
    assert _close(lb.cpu().numpy(), olb) < RTOL
    assert _close(lA.cpu().numpy(), olA) < RTOL


@pytest.mark.parametrize("mode,threads", VARIANTS)
def test_overflow_and_infinite_boxes(mode, threads):
    """exp(c x) overflows on [-900, 900]; an infinite side makes every relaxation touching it
    undefined. Rows that touch undefined elements fall back to the output interval."""
    m, g = _graph()
    lo, hi = problems.make_boxes("quad_exp_n10", 8, 0)
    lo, hi = lo.clone(), hi.clone()
    lo[0], hi[0] = -900.0, 900.0                 # exp overflow
    hi[1, 3] = float("inf")                      # an unbounded coordinate
    lo[2, 0] = -float("inf")
    lo[3] = hi[3]                                # a point box
    eng = CrownEngine(g, mode=mode, cta_threads=threads)
    lb, lA, lbias = eng.lower(lo.cuda(), hi.cuda())
    olb, _, olA, olbias = CrownOracle(g).compute_bounds(lo.numpy(), hi.numpy())
    assert _close(lb.cpu().numpy(), olb) < RTOL
    # the point box: a power's secant over the 1e-8 widening amplifies pow's last bit (CPU vs
    # CUDA) by ~1e8 in the planes; the bound itself agrees to RTOL
    tol = np.where((hi - lo).amin(1).numpy() < 1e-6, 1e-6, RTOL)
    for b in range(lo.shape[0]):
        assert _close(lA[b].cpu().numpy(), olA[b]) < tol[b]
        assert _close(lbias[b].cpu().numpy(), olbias[b]) < tol[b]


def test_empty_bab_steps():
    from gear_b200 import _lib
    L = _lib.lib()
    st = torch.cuda.current_stream().cuda_stream
    nk = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    ws = torch.empty(int(L.gear_bab_workspace_bytes(0)) + 64, dtype=torch.uint8, device="cuda")
    z = torch.empty(0, dtype=torch.float64, device="cuda")
    keep = torch.empty(0, dtype=torch.uint8, device="cuda")
    kept = torch.empty(0, dtype=torch.int32, device="cuda")
    dmin = torch.full((1,), float("inf"), dtype=torch.float64, device="cuda")
    _lib.check(L.gear_bab_prune(z.data_ptr(), z.data_ptr(), 0, 3, keep.data_ptr(), kept.data_ptr(),
                                nk.data_ptr(), dmin.data_ptr(), ws.data_ptr(), ws.numel(), st), "prune")
    torch.cuda.synchronize()
    assert int(nk.item()) == 0 and float(dmin.item()) == float("inf")
    nk.fill_(7)
    _lib.check(L.gear_bab_compact(keep.data_ptr(), 0, kept.data_ptr(), nk.data_ptr(), ws.data_ptr(),
                                  ws.numel(), st), "compact")
    torch.cuda.synchronize()
    assert int(nk.item()) == 0


def test_static_entry_argument_checks():
    """gear_crown_lower_static checks its arguments like gear_crown_lower: an empty batch with
    null pointers is accepted, an lA output for a program compiled without A is rejected."""
    from gear_b200 import _lib
    from gear_b200.engine import _Dag
    from gear_b200.program import Program
    L = _lib.lib()
    m, g = _graph()
    st = torch.cuda.current_stream().cuda_stream
    with_a = _Dag.from_program(Program(g, mode="cta"))
    for fn in ("gear_crown_lower_static",):
        assert getattr(L, fn)(with_a.handle, None, None, 0, None, None, None, None, st) == 0
    no_a = _Dag.from_program(Program(g, mode="cta", return_a=False))
    lo, hi = problems.make_boxes("quad_exp_n10", 4, 0)
    xL, xU = lo.cuda(), hi.cuda()
    lb = torch.empty(4, 3, dtype=torch.float64, device="cuda")
    lbias = torch.empty_like(lb)
    lA = torch.empty(4, 3, 10, dtype=torch.float64, device="cuda")
    assert L.gear_crown_lower_static(no_a.handle, xL.data_ptr(), xU.data_ptr(), 4, None, lb.data_ptr(),
                                     lA.data_ptr(), lbias.data_ptr(), st) == -1
    ws = torch.empty(int(L.gear_crown_workspace_bytes(no_a.handle, 4)), dtype=torch.uint8, device="cuda")
    assert L.gear_crown_lower(no_a.handle, xL.data_ptr(), xU.data_ptr(), 4, None, lb.data_ptr(), lA.data_ptr(),
                              lbias.data_ptr(), ws.data_ptr(), ws.numel(), st) == -1
    # without lA both entry points run and agree
    assert L.gear_crown_lower_static(no_a.handle, xL.data_ptr(), xU.data_ptr(), 4, None, lb.data_ptr(),
                                     None, lbias.data_ptr(), st) == 0
    lb2 = torch.empty_like(lb)
    assert L.gear_crown_lower(no_a.handle, xL.data_ptr(), xU.data_ptr(), 4, None, lb2.data_ptr(), None,
                              lbias.data_ptr(), ws.data_ptr(), ws.numel(), st) == 0
    torch.cuda.synchronize()
    assert torch.equal(lb, lb2)
