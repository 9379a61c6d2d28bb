"""gear_clip_domains (one warp per box) against the reference's clip_domains fixtures and the
oracle: identical emptiness, other boxes' bounds within 1e-12 of the box width; rows
addressed through a parent index; BaB with clipping and constrained concretisation (the
reference's complete clipping mode) closes the gap soundly."""
import os

import numpy as np
import pytest
import torch

from oracle.clip import clip_domains

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "clip.npz")
CASES = sorted({k.rsplit("_", 1)[0] for k in np.load(GOLD).files})


def gpu_clip(xl, xu, thr, lA, lbias, iters, parent=None):
    from gear_b200 import _lib
    t = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda").contiguous()
    cl, cu, th, A, lb = t(xl), t(xu), t(thr), t(lA), t(lbias)
    B, n = cl.shape
    S = th.shape[1]
    ne = torch.empty(B, dtype=torch.uint8, device="cuda")
    par = None if parent is None else torch.tensor(parent, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().gear_clip_domains(cl.data_ptr(), cu.data_ptr(), th.data_ptr(), A.data_ptr(), lb.data_ptr(),
                                            None if par is None else par.data_ptr(), B, S, n, iters, ne.data_ptr(), st),
               "gear_clip_domains")
    torch.cuda.synchronize()
    return cl.cpu().numpy(), cu.cpu().numpy(), ne.cpu().numpy()


def compare(cl, cu, rl, ru, xl, xu, tol=1e-12):
    emp_r = (rl > ru).any(1)
    assert np.array_equal(emp_r, (cl > cu).any(1))
    ne = ~emp_r
    scale = np.maximum(1.0, np.abs(xu - xl))[ne]
    assert np.max(np.abs(cl - rl)[ne] / scale) <= tol
    assert np.max(np.abs(cu - ru)[ne] / scale) <= tol


@pytest.mark.parametrize("case", CASES)
def test_matches_reference_fixtures(case):
    d = np.load(GOLD)
    it = int(case.split("it")[1])
    args = [d[case + s] for s in ("_xl", "_xu", "_thr", "_lA", "_lbias")]
    cl, cu, ne = gpu_clip(*args, it)
    compare(cl, cu, d[case + "_cl"], d[case + "_cu"], args[0], args[1])
    assert np.array_equal(ne.astype(bool), ~(cl > cu).any(1))


def test_parent_rows():
    d = np.load(GOLD)
    case = "small_it1"
    xl, xu, thr, lA, lb = (d[case + s] for s in ("_xl", "_xu", "_thr", "_lA", "_lbias"))
    parent = np.arange(xl.shape[0])[::-1].copy()
    cl, cu, _ = gpu_clip(xl[parent], xu[parent], thr, lA, lb, 1, parent=parent)
    rl, ru = clip_domains(xl[parent], xu[parent], thr[parent], lA[parent], lb[parent])
    compare(cl, cu, rl, ru, xl[parent], xu[parent])


def test_complete_clipping_bab_closes_gap_soundly():
    from gear_b200 import problems, graph
    from gear_b200.bab import BaB
    m = problems.make_instance("quad_exp_n10", 0)
    lo, hi = problems.root_box("quad_exp_n10")
    g = graph.trace(m, lo.repeat(2, 1))
    plain = BaB(g, lo, hi, batch=2048, model=m.cuda())
    plain.run(rel_gap=1e-4, max_iterations=400, time_limit=120)
    full = BaB(g, lo, hi, batch=2048, model=m.cuda(), constrained=True, clip=True)
    P, Dd, gap = full.run(rel_gap=1e-4, max_iterations=400, time_limit=120)
    print("iterations plain", plain.stats.iterations, "complete clipping", full.stats.iterations,
          "clipped empty", full.stats.clipped_empty)
    assert gap <= 1e-4
    assert full.stats.iterations <= plain.stats.iterations
    x = lo + (hi - lo) * torch.rand(200000, lo.shape[1], dtype=torch.float64)
    y = m(x.cuda()).cpu()
    feas = (y[:, 1:] <= 0).all(1)
    assert Dd <= float(y[feas, 0].min()) + 1e-9
