"""Tensor-core fold (fold_tc.cuh): the int8 digit-sliced tcgen05 GEMMs that give the fold vectors of
dense nodes on the input for a whole batch.

* Enclosure: for every box and output, [c^ - r', c^ + r'] contains [c - r, c + r] with c = W x0 and
  r = |W| eps evaluated in extended precision (numpy longdouble), and t' >= |W| max(|x_L|, |x_U|):
  the error term is a rigorous bound. Tightness: r' - r is below 1e-7 of the row's scale
  sum |W| (|x0| + eps).
* Bounds: CROWN with the tensor-core fold agrees with the CUDA-core fold to 1e-6 relative on every
  row (both with exact-arithmetic McCormick ties), and its bounds are sound by sampling."""
import numpy as np
import pytest
import torch

from gear_b200 import _lib, graph, problems
from gear_b200.engine import CrownEngine

pytestmark = pytest.mark.gpu


def _boxes(workload, batch, seed):
    lo, hi = problems.make_boxes(workload, batch, seed)
    rl, rh = problems.root_box(workload)
    lo, hi = torch.cat([rl, lo]), torch.cat([rh, hi])
    lo[1] = hi[1]                                    # a point box
    return lo, hi


@pytest.mark.parametrize("workload,batch", [("dense_q_n200", 300), ("dense_a_n2048", 66)])
def test_fold_vectors_enclose_the_exact_products(workload, batch):
    m = problems.make_instance(workload, 0)
    lo, hi = _boxes(workload, batch - 2, 3)
    g = graph.trace(m, lo[:2])
    eng = CrownEngine(g, mode="cta", cta_threads=128, fold_tc=True)
    prog = eng.prog
    assert int(prog.header[23]) == 1 and prog.fold_w > 0
    L = _lib.lib()
    B = lo.shape[0]
    xL, xU = lo.cuda().contiguous(), hi.cuda().contiguous()
    ws = torch.empty(int(L.gear_crown_fold_workspace_bytes(eng.handle, B)), dtype=torch.uint8, device="cuda")
    fold = torch.full((B, prog.fold_w), np.nan, dtype=torch.float64, device="cuda")
    flag = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    _lib.check(L.gear_crown_fold_vectors(eng.handle, xL.data_ptr(), xU.data_ptr(), B, fold.data_ptr(),
                                         flag.data_ptr(), ws.data_ptr(), ws.numel(),
                                         torch.cuda.current_stream().cuda_stream), "gear_crown_fold_vectors")
    torch.cuda.synchronize()
    assert int(flag.item()) == 0
    f = fold.cpu().numpy()
    xl, xu = lo.numpy().astype(np.longdouble), hi.numpy().astype(np.longdouble)
    x0 = (lo.numpy() + hi.numpy()) / 2.0                 # the float64 centre and radius the kernels use
    eps = (hi.numpy() - lo.numpy()) / 2.0
    xm = np.maximum(np.abs(lo.numpy()), np.abs(hi.numpy()))
    for v, off in prog.fold_off.items():
        nd = g[v]
        W = nd.attrs["W"] if nd.kind == "linear" else nd.attrs["W"].T      # (out, in)
        w = W.shape[0]
        Wl = W.astype(np.longdouble)
        c = x0.astype(np.longdouble) @ Wl.T
        r = eps.astype(np.longdouble) @ np.abs(Wl).T
        t = xm.astype(np.longdouble) @ np.abs(Wl).T
        scale = (np.abs(x0) + eps).astype(np.longdouble) @ np.abs(Wl).T
        ch, rh_, th = f[:, off:off + w], f[:, off + w:off + 2 * w], f[:, off + 2 * w:off + 3 * w]
        slack = 1e-15 * scale                            # longdouble evaluation of the references
        assert np.all(ch - rh_ <= c - r + slack)
        assert np.all(ch + rh_ >= c + r - slack)
        assert np.all(th >= t - slack)
        assert np.all(rh_ - r <= 1e-7 * scale + 1e-300)


@pytest.mark.parametrize("workload,batch", [("dense_q_n200", 300), ("dense_a_n2048", 96)])
def test_tensor_core_fold_bounds_match_cuda_core_fold(workload, batch):
    m = problems.make_instance(workload, 0)
    lo, hi = _boxes(workload, batch - 2, 4)
    g = graph.trace(m, lo[:2])
    xL, xU = lo.cuda(), hi.cuda()
    a = CrownEngine(g, mode="cta", cta_threads=128, tie_rule="exact", fold_tc=True).lower(xL, xU)
    b = CrownEngine(g, mode="cta", cta_threads=128, tie_rule="exact").lower(xL, xU)
    torch.cuda.synchronize()
    la, lb_ = a[0].cpu().numpy(), b[0].cpu().numpy()
    same_inf = np.isinf(la) & np.isinf(lb_) & (np.sign(la) == np.sign(lb_))
    err = np.where(same_inf, 0.0, np.abs(la - lb_) / np.maximum(1.0, np.abs(lb_)))
    assert float(err.max()) < 1e-6


@pytest.mark.parametrize("workload", ["dense_q_n200", "dense_a_n2048"])
def test_tensor_core_fold_bounds_sound_on_sampled_points(workload):
    m = problems.make_instance(workload, 0).cuda()
    lo, hi = problems.make_boxes(workload, 16, 6)
    g = graph.trace(problems.make_instance(workload, 0), lo[:2])
    xL, xU = lo.cuda(), hi.cuda()
    lb, lA, lbias = CrownEngine(g, mode="cta", cta_threads=256, fold_tc=True).lower(xL, xU)
    gen = torch.Generator(device="cuda").manual_seed(99)
    for b in range(lo.shape[0]):
        u = torch.rand(10_000, lo.shape[1], generator=gen, dtype=torch.float64, device="cuda")
        pts = torch.minimum(torch.maximum(xL[b] + (xU[b] - xL[b]) * u, xL[b]), xU[b])
        with torch.no_grad():
            y = m(pts)
        slack = 1e-9 * torch.clamp(y.abs(), min=1.0)
        assert torch.all(lb[b] <= (y + slack).min(0).values)
        plane = pts @ lA[b].T + lbias[b]
        assert torch.all(plane <= y + slack + 1e-9 * torch.clamp(plane.abs(), min=1.0))


@pytest.mark.parametrize("spec", [None, "two_rows"])
def test_final_pass_product_on_tensor_cores(spec):
    """dense_a_n2048's final pass ends with the product through its 1024 x 2048 node (A_v W): with the
    tensor-core fold that product runs as one tcgen05 GEMM over the batch (split_tc.cuh). Its lA rows
    agree with the float64 CUDA-core product to 1e-9 of the row's scale, lb and lbias to 1e-6
    relative, a box with an infinite coordinate falls back to the same interval bound, and the
    launch sequence is box digits, fold GEMM, CROWN kernel, row digits, product GEMM, tail."""
    wl = "dense_a_n2048"
    m = problems.make_instance(wl, 0)
    lo, hi = _boxes(wl, 62, 8)
    hi[5, 7] = float("inf")                          # an open box
    g = graph.trace(m, lo[:2])
    B = lo.shape[0]
    xL, xU = lo.cuda(), hi.cuda()
    kw = {}
    C = None
    if spec == "two_rows":
        kw = dict(spec_rows=2, dense_c=True)
        C = torch.tensor([[[1.0], [-1.0]]], dtype=torch.float64, device="cuda").expand(B, 2, 1).contiguous()
    tc = CrownEngine(g, mode="cta", cta_threads=256, tie_rule="exact", fold_tc=True, **kw)
    cc = CrownEngine(g, mode="cta", cta_threads=256, tie_rule="exact", **kw)
    assert tc.prog.split_op >= 0 and cc.prog.split_op == -1
    a = tc.lower(xL, xU, C)
    launches = _lib.lib().gear_last_launch_count()
    b = cc.lower(xL, xU, C)
    torch.cuda.synchronize()
    assert launches == 2 + len(tc.prog.fold_off) + 3
    la, lb_ = a[0].cpu().numpy(), b[0].cpu().numpy()
    fin = np.isfinite(lb_)
    assert np.array_equal(fin, np.isfinite(la))
    assert np.all(np.abs(la - lb_)[fin] <= 1e-6 * np.maximum(1.0, np.abs(lb_[fin])))
    assert np.array_equal(la[5], lb_[5])             # the open box: the same interval fallback
    Aa, Ab = a[1].cpu().numpy(), b[1].cpu().numpy()
    scale = np.abs(Ab).max(axis=2, keepdims=True)
    assert np.all(np.abs(Aa - Ab) <= 1e-9 * np.maximum(scale, 1e-300))
    ba, bb = a[2].cpu().numpy(), b[2].cpu().numpy()
    fb = np.isfinite(bb)
    assert np.array_equal(fb, np.isfinite(ba))
    assert np.all(np.abs(ba - bb)[fb] <= 1e-6 * np.maximum(1.0, np.abs(bb[fb])))
