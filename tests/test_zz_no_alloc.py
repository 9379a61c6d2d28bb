"""gear_crown_lower_static: the CROWN entry point that allocates no device memory.

It serves callers that cannot call cudaMalloc -- a solver host that owns a fixed device
memory plan and gives the library no allocator, or a loop that must not take cudaMalloc's
implicit synchronisation -- by using a scratch array built into the library. This test calls
it through the C ABI twice in a row and compares both results with the workspace entry point
gear_crown_lower, to the tolerance the other GPU tests use (1e-9 relative). It lives in a file
of its own that pytest collects last, and passes alone or after the other tests.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
RTOL = 1e-9


@pytest.mark.parametrize("workload,batch", [("quad_exp_n10", 700), ("dense_q_n200", 600)])
def test_static_scratch_entry_matches_workspace_entry(workload, batch):
    from gear_b200 import _lib, graph, problems
    from gear_b200.engine import CrownEngine
    L = _lib.lib()
    m = problems.make_instance(workload, 0)
    lo, hi = problems.make_boxes(workload, batch, 0)
    g = graph.trace(m, lo[:2])
    eng = CrownEngine(g)
    xL, xU = lo.cuda().contiguous(), hi.cuda().contiguous()
    ref_lb, ref_lA, ref_lbias = eng.lower(xL, xU)
    torch.cuda.synchronize()
    assert L.gear_crown_static_scratch_bytes() > 0
    st = torch.cuda.current_stream().cuda_stream
    for _ in range(2):   # two calls in a row share (and reuse) the built-in scratch
        lb = torch.full_like(ref_lb, np.nan)
        lA = torch.full_like(ref_lA, np.nan)
        lbias = torch.full_like(ref_lbias, np.nan)
        status = L.gear_crown_lower_static(eng.handle, xL.data_ptr(), xU.data_ptr(), batch, None, lb.data_ptr(),
                                           lA.data_ptr(), lbias.data_ptr(), st)
        _lib.check(status, "gear_crown_lower_static")
        torch.cuda.synchronize()
        for got, want in ((lb, ref_lb), (lA, ref_lA), (lbias, ref_lbias)):
            g_, w_ = got.cpu().numpy(), want.cpu().numpy()
            assert np.all(np.isfinite(g_) == np.isfinite(w_))
            err = np.abs(g_ - w_) / np.maximum(1.0, np.abs(w_))
            assert float(np.nanmax(np.where(np.isfinite(w_), err, 0.0))) < RTOL


def test_static_scratch_entry_loops_boxes_beyond_its_slots():
    """A batch that needs more CTA scratch slots than the 64 MiB array holds: the entry runs the
    batch on as many CTAs as fit, each taking several boxes in turn. Boxes are independent and
    run the same code, so the results equal the workspace entry point's bit for bit."""
    from gear_b200 import _lib, graph, problems
    from gear_b200.engine import CrownEngine
    L = _lib.lib()
    m = problems.make_instance("dense_a_n2048", 0)
    batch = 600
    lo, hi = problems.make_boxes("dense_a_n2048", batch, 0)
    eng = CrownEngine(graph.trace(m, lo[:2]), mode="cta", cta_threads=256)
    # more slots than the static array holds: the capped path runs
    assert L.gear_crown_workspace_bytes(eng.handle, batch) > L.gear_crown_static_scratch_bytes()
    xL, xU = lo.cuda().contiguous(), hi.cuda().contiguous()
    ref = eng.lower(xL, xU)
    st = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out = [torch.full_like(t, np.nan) for t in ref]
        _lib.check(L.gear_crown_lower_static(eng.handle, xL.data_ptr(), xU.data_ptr(), batch, None,
                                             out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), st),
                   "gear_crown_lower_static")
        torch.cuda.synchronize()
        for got, want in zip(out, ref):
            assert torch.equal(got, want)
