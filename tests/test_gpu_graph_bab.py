"""The device-resident queue (gear_queue_*) and the graph-captured branch-and-bound iteration
(gear_bab_step, GraphBaB).

* Queue: pops return the open domains in the reference's order (objective key descending, ties by
  insertion id; the batch is the tail), padded with the first popped box, and the counters follow.
* GraphBaB runs the search BaB runs: after the same number of iterations the incumbent, the dual
  bound and the number of domains bounded are identical (same kernels, same queue order), with
  the iterations replayed from a CUDA graph; and it reaches the relative gap."""
import ctypes
import math

import numpy as np
import pytest
import torch

from gear_b200 import _lib, graph, problems
from gear_b200.bab import BaB, GraphBaB
from gear_b200.engine import CrownEngine

pytestmark = pytest.mark.gpu


def test_queue_pop_order_and_counters():
    L = _lib.lib()
    n, S, batch = 3, 2, 4
    root_lo = torch.zeros(n, dtype=torch.float64)
    root_hi = torch.ones(n, dtype=torch.float64)
    h = ctypes.c_void_p()
    _lib.check(L.gear_queue_create(n, S, 64, batch, root_lo.data_ptr(), root_hi.data_ptr(), ctypes.byref(h)),
               "gear_queue_create")
    st = torch.cuda.current_stream().cuda_stream
    try:
        # pop the root, then push 8 domains with tied keys
        lo = torch.empty(batch, n, dtype=torch.float64, device="cuda")
        hi = torch.empty_like(lo)
        _lib.check(L.gear_queue_pop(h, lo.data_ptr(), hi.data_ptr(), st), "pop")
        torch.cuda.synchronize()
        assert torch.equal(lo.cpu(), torch.zeros(batch, n, dtype=torch.float64))     # root, then padding copies
        keys = torch.tensor([3.0, 1.0, 2.0, 1.0, 5.0, 1.0, 2.0, 0.5], dtype=torch.float64)
        m = keys.numel()
        plo = torch.arange(m, dtype=torch.float64).repeat_interleave(n).reshape(m, n).cuda()
        pkey = torch.stack([keys, torch.zeros(m, dtype=torch.float64)], 1).cuda()
        _lib.check(L.gear_queue_push(h, plo.data_ptr(), (plo + 1).data_ptr(), pkey.data_ptr(), m, st), "push")
        open_ = ctypes.c_int64()
        _lib.check(L.gear_queue_size(h, ctypes.byref(open_), st), "size")
        assert open_.value == m
        # expected pop order: stable sort by key descending (ids = push order), batches from the tail
        order = sorted(range(m), key=lambda i: (-float(keys[i]), i))
        popped = []
        for _ in range(2):
            _lib.check(L.gear_queue_pop(h, lo.data_ptr(), hi.data_ptr(), st), "pop")
            torch.cuda.synchronize()
            popped.append(lo[:, 0].cpu().numpy().astype(int).tolist())
        assert popped[0] == order[-batch:]
        assert popped[1] == order[-2 * batch:-batch]
        cnt = torch.zeros(8, dtype=torch.int64, device="cuda")
        dual = torch.zeros(1, dtype=torch.float64, device="cuda")
        _lib.check(L.gear_queue_counters(h, cnt.data_ptr(), dual.data_ptr(), st), "counters")
        torch.cuda.synchronize()
        c = cnt.cpu().tolist()
        assert c[0] == 0 and c[1] == 64 and c[2] == 1 + m and c[6] == 3
        assert float(dual.item()) == math.inf
    finally:
        L.gear_queue_destroy(h)


@pytest.mark.parametrize("inst", [0, 1])
def test_graph_bab_runs_the_search_bab_runs(inst):
    m = problems.make_instance("quad_exp_n10", inst)
    lo, hi = problems.root_box("quad_exp_n10")
    g = graph.trace(m, lo.repeat(2, 1))
    md = m.cuda()
    a = BaB(g, lo, hi, batch=512, model=md, device="cuda", engine_mode="cta")
    Pa, Da, _ = a.run(rel_gap=-1.0, max_iterations=40, time_limit=600)
    b = GraphBaB(g, lo, hi, batch=512, model=md, device="cuda", engine_mode="cta", chunk=8)
    Pb, Db, _ = b.run(rel_gap=-1.0, max_iterations=40, time_limit=600)
    assert b.graph_obj is not None and b.replays >= 3
    assert b.status["iterations"] == a.stats.iterations == 40
    assert b.status["bounded"] == a.stats.bounded
    assert Pa == Pb and Da == Db
    assert b.status["open"] == len(a.queue)


def test_graph_bab_tensor_core_program():
    """A tensor-core program (dense_a_n2048: the fold and the final pass's product on tcgen05) in
    the device-queue step (gear_bab_step) runs the same search as the host-driven loop."""
    m = problems.make_instance("dense_a_n2048", 0)
    lo, hi = problems.root_box("dense_a_n2048")
    g = graph.trace(m, lo.repeat(2, 1))
    md = m.cuda()
    eng = CrownEngine(g, mode="cta", cta_threads=256, fold_tc=True)
    assert eng.prog.split_op >= 0
    a = BaB(g, lo, hi, batch=64, model=md, device="cuda", engine=eng)
    Pa, Da, _ = a.run(rel_gap=-1.0, max_iterations=6, time_limit=600)
    b = GraphBaB(g, lo, hi, batch=64, model=md, device="cuda", engine=eng, chunk=2)
    Pb, Db, _ = b.run(rel_gap=-1.0, max_iterations=6, time_limit=600)
    assert b.status["iterations"] == a.stats.iterations == 6
    assert b.status["bounded"] == a.stats.bounded
    assert Pa == Pb and Da == Db


def test_graph_bab_reaches_the_gap():
    m = problems.make_instance("quad_exp_n10", 2)
    lo, hi = problems.root_box("quad_exp_n10")
    g = graph.trace(m, lo.repeat(2, 1))
    # a small first capacity: the queue grows during the run and the iterations are captured again
    b = GraphBaB(g, lo, hi, batch=2048, model=m.cuda(), device="cuda", capacity=20000)
    P, D, gap = b.run(rel_gap=1e-4, time_limit=120)
    assert gap <= 1e-4 and math.isfinite(P) and D <= P
    assert b.status["overflow"] == 0 and b.regrown > 0


def test_multi_graph_bab_equals_each_instance_alone():
    """Every instance of the graph-captured many-instance run searches as GraphBaB does alone
    (the packed launch is bit-identical to a launch per instance)."""
    from gear_b200.bab import MultiGraphBaB
    from gear_b200.engine import CrownEngine, MultiEngine
    ks = [0, 1, 3, 4, 8]
    insts = [problems.mixed_instance(k) for k in ks]
    graphs = [graph.trace(m, torch.zeros(2, m.n, dtype=torch.float64)) for m in insts]
    roots = [(torch.full((1, m.n), -2.0, dtype=torch.float64), torch.full((1, m.n), 2.0, dtype=torch.float64))
             for m in insts]
    models = [m.cuda() for m in insts]
    me = MultiEngine(graphs, mode="auto", cta_threads=128)
    # small first queues (70 slots for batches of 32): they grow during the run
    mb = MultiGraphBaB(graphs, roots, models, batch=32, engine=me, queue_slots=70)
    res = mb.run(rel_gap=-1.0, time_limit=600, max_rounds=10)
    assert mb.rounds == 10 and mb.prepares >= 1
    assert mb.captures_regrown > 0                        # queues grew (their graphs captured again)
    compared = 0
    for i, g in enumerate(graphs):
        if res[i]["status"] != "running":
            continue                                      # retired early (emptied its queue)
        var = me.variants[i]
        eng = CrownEngine(g, mode=var[0], cta_threads=var[1] or 128)
        b = GraphBaB(g, roots[i][0], roots[i][1], batch=32, model=models[i], engine=eng, chunk=2)
        P, D, _ = b.run(rel_gap=-1.0, max_iterations=10, time_limit=600)
        assert b.status["iterations"] == 10
        assert res[i]["P"] == P and res[i]["D"] == D and res[i]["bounded"] == b.status["bounded"]
        compared += 1
    assert compared >= 3
