"""Many instances in one launch (gear_crown_lower_multi / MultiEngine): every instance's
results are bit-identical to the same program launched alone, and agree with the oracle
(1e-9 relative; McCormick ties decided in exact arithmetic on both sides, tie_rule "exact"). Also the box-per-CTA program whose pass working set lives in global scratch:
identical to the shared-memory one."""
import numpy as np
import pytest
import torch

from gear_b200 import _lib, graph, problems
from gear_b200.engine import CrownEngine, MultiEngine, _Dag
from gear_b200.program import Program
from oracle.crown import CrownOracle, EXACT_TIE_TOL

pytestmark = pytest.mark.gpu
RTOL = 1e-9
SMALL = [0, 1, 3, 4, 5, 8, 10, 16]          # mixed instances with n <= 30


def _close(a, b):
    a, b = np.asarray(a), np.asarray(b)
    both_inf = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
    err = np.where(both_inf, 0.0, np.abs(a - b) / np.maximum(1.0, np.abs(b)))
    return float(np.nanmax(err)) if err.size else 0.0


def _graph(m, n):
    return graph.trace(m, torch.zeros(2, n, dtype=torch.float64))


def _instances():
    ms = [problems.mixed_instance(k) for k in SMALL]
    qe = problems.make_instance("quad_exp_n10", 0)
    graphs = [_graph(m, m.n) for m in ms] + [_graph(qe, 10)]
    boxes = [problems.mixed_boxes(m, b, k) for m, k, b in zip(ms, SMALL, (37, 0, 64, 1, 200, 65, 128, 3))]
    boxes.append(problems.make_boxes("quad_exp_n10", 300, 0))
    return graphs, boxes


@pytest.mark.parametrize("mode", ["auto", "cta", "simt"])
def test_multi_equals_alone_and_oracle(mode):
    graphs, boxes = _instances()
    me = MultiEngine(graphs, mode=mode, cta_threads=128, tie_rule="exact")
    dev_boxes = [(lo.cuda(), hi.cuda()) for lo, hi in boxes]
    outs = me.lower(dev_boxes)
    torch.cuda.synchronize()
    assert me.launches() == len(me.groups)
    for i, (g, (lo, hi)) in enumerate(zip(graphs, boxes)):
        lb, lA, lbias = outs[i]
        assert lb.shape == (lo.shape[0], me.S[i]) and lA.shape == (lo.shape[0], me.S[i], me.n[i])
        if lo.shape[0] == 0:
            continue
        var = me.variants[i]
        alone = CrownEngine(g, mode=var[0], cta_threads=var[1] if var[0] == "cta" else 128, tie_rule="exact")
        lb1, lA1, lbias1 = alone.lower(dev_boxes[i][0], dev_boxes[i][1])
        torch.cuda.synchronize()
        assert torch.equal(lb, lb1) and torch.equal(lA, lA1) and torch.equal(lbias, lbias1)
        olb, _, olA, olbias = CrownOracle(g, tie_tol=EXACT_TIE_TOL).compute_bounds(lo.numpy(), hi.numpy())
        assert _close(lb.cpu().numpy(), olb) < RTOL
        assert _close(lA.cpu().numpy(), olA) < RTOL


def test_multi_reuses_engine_across_batches():
    graphs, boxes = _instances()
    me = MultiEngine(graphs)
    for scale in (1, 2):
        bx = [(lo.repeat(scale, 1).cuda(), hi.repeat(scale, 1).cuda()) for lo, hi in boxes]
        outs = me.lower(bx)
        for i, (lo, hi) in enumerate(bx):
            if lo.shape[0]:
                alone = CrownEngine(graphs[i], mode=me.variants[i][0], cta_threads=me.variants[i][1] or 128)
                assert torch.equal(outs[i][0], alone.lower(lo, hi)[0])


def test_multi_rejects_mixed_modes():
    graphs, boxes = _instances()
    a = _Dag(graphs[0], None, False, "cta", 128)
    b = _Dag(graphs[1], None, False, "simt", 128)
    lo, hi = boxes[0]
    lo, hi = lo.cuda(), hi.cuda()
    out = torch.empty(lo.shape[0], 4096, dtype=torch.float64, device="cuda")
    args = (_lib.LowerArgs * 2)()
    for k, d in enumerate((a, b)):
        args[k] = _lib.LowerArgs(d.handle.value, lo.data_ptr(), hi.data_ptr(), 1, None, out.data_ptr(),
                                 out.data_ptr(), out.data_ptr())
    assert _lib.lib().gear_crown_multi_workspace_bytes(args, 2) == -1
    assert b"same execution mode" in _lib.lib().gear_last_error()


@pytest.mark.parametrize("k", [4, 5])
def test_global_pass_working_set_matches_shared(k):
    """A working set forced out of shared memory (smem_limit) gives the same bits."""
    m = problems.mixed_instance(k)
    g = _graph(m, m.n)
    lo, hi = problems.mixed_boxes(m, 150, k)
    lo, hi = lo.cuda(), hi.cuda()
    res = []
    for limit in (232448, 1024):
        prog = Program(g, mode="cta", cta_threads=128, smem_limit=limit)
        assert (prog.pass_global > 0) == (limit == 1024)
        me = MultiEngine([g], programs=[prog])
        res.append(me.lower([(lo, hi)])[0])
    torch.cuda.synchronize()
    for a, b in zip(res[0], res[1]):
        assert torch.equal(a, b)


@pytest.mark.parametrize("workload,k", [("quad_exp_n10", None), ("dense_q_n200", None), ("mixed", 4), ("mixed", 8)])
def test_plain_form_matches_fused(workload, k):
    """The plain form (one launch per step / per op) gives the fused kernel's bits."""
    from gear_b200.engine import PlainEngine
    if workload == "mixed":
        m = problems.mixed_instance(k)
        n = m.n
        lo, hi = problems.mixed_boxes(m, 100, k)
    else:
        m = problems.make_instance(workload, 0)
        n = problems.WORKLOADS[workload]["n"]
        lo, hi = problems.make_boxes(workload, 100, 0)
    g = _graph(m, n)
    lo, hi = lo.cuda(), hi.cuda()
    pe = PlainEngine(g)
    a = pe.lower(lo, hi)
    assert pe.launches > 3
    b = CrownEngine(g, mode="cta", cta_threads=128).lower(lo, hi)
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert torch.equal(x, y)


def test_multi_bab_matches_single_runs():
    """MultiBaB: each instance's search equals BaB run alone with the same kernel variant."""
    from gear_b200.bab import BaB, MultiBaB
    from gear_b200.engine import MultiEngine
    ks = [0, 1, 3, 8, 10]
    ms = [problems.mixed_instance(k) for k in ks]
    graphs = [_graph(m, m.n) for m in ms]
    roots = [(torch.full((1, m.n), -2.0, dtype=torch.float64), torch.full((1, m.n), 2.0, dtype=torch.float64))
             for m in ms]
    models = [m.cuda() for m in ms]
    me = MultiEngine(graphs)
    mb = MultiBaB(graphs, roots, models, batch=64, engine=me)
    res = mb.run(rel_gap=1e-4, time_limit=120, max_iterations=12)
    for i, g in enumerate(graphs):
        var = me.variants[i]
        eng = CrownEngine(g, mode=var[0], cta_threads=var[1] or 128)
        bb = BaB(g, roots[i][0], roots[i][1], batch=64, engine=eng, model=models[i])
        for _ in range(res[i]["iterations"]):
            bb.step()
        assert bb.incumbent == res[i]["P"]
        assert bb.stats.bounded == res[i]["bounded"]
        assert bb.dual_bound() == float(torch.minimum(mb.babs[i].queue.min_key_tensor(), mb.babs[i].disc_min))


def test_multi_ibp_pass_and_empty_groups():
    """The IBP pass through the packed launch equals CrownEngine's, and groups whose instances
    all have empty batches launch nothing (their outputs are empty)."""
    graphs, boxes = _instances()
    me = MultiEngine(graphs, mode="auto", cta_threads=128)
    # empty every instance of one group, keep the others
    first_group = next(iter(me.groups.values()))
    bx, ibp = [], []
    for i, (lo, hi) in enumerate(boxes):
        if i in first_group:
            lo, hi = lo[:0], hi[:0]
        bx.append((lo.cuda(), hi.cuda()))
        ibp.append(torch.empty(lo.shape[0], me.S[i], dtype=torch.float64, device="cuda"))
    outs = me.lower(bx, lb_ibp=ibp)
    torch.cuda.synchronize()
    for i, g in enumerate(graphs):
        B = bx[i][0].shape[0]
        assert outs[i][0].shape == (B, me.S[i])
        if B == 0:
            continue
        var = me.variants[i]
        eng = CrownEngine(g, mode=var[0], cta_threads=var[1] or 128)
        ib = torch.empty(B, me.S[i], dtype=torch.float64, device="cuda")
        lb1, _, _ = eng.lower(bx[i][0], bx[i][1], lb_ibp=ib)
        torch.cuda.synchronize()
        assert torch.equal(outs[i][0], lb1) and torch.equal(ibp[i], ib)


def test_plain_form_empty_batch():
    from gear_b200.engine import PlainEngine
    m = problems.make_instance("quad_exp_n10", 0)
    pe = PlainEngine(_graph(m, 10))
    e = torch.empty(0, 10, dtype=torch.float64, device="cuda")
    lb, lA, lbias = pe.lower(e, e)
    assert lb.shape == (0, 3) and lA.shape == (0, 3, 10)
