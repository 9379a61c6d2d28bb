"""Serving loop (continuous batching): requests submitted while others run are admitted at the
next round, and every request's result -- incumbent, domains bounded, relative gap, rounds --
is the same as its own branch and bound run alone with the same kernel variant. Both forms: the
host-driven rounds (Server) and device queues with per-request CUDA graphs (DeviceServer)."""
import math

import pytest
import torch

from gear_b200 import problems
from gear_b200.bab import BaB
from gear_b200.engine import CrownEngine
from gear_b200.serve import DeviceServer, Server

pytestmark = pytest.mark.gpu


def _req(k, n):
    m = problems.QuadExpN10(n=n, seed=5000 + k)
    return m, torch.full((1, n), -2.0, dtype=torch.float64), torch.full((1, n), 2.0, dtype=torch.float64)


@pytest.mark.parametrize("cls", [Server, DeviceServer])
def test_serve_same_alone_and_in_mix(cls):
    sizes = [(0, 6), (1, 10), (2, 14), (3, 8), (4, 12), (5, 20)]
    # the clock advances one unit per round: a request leaves after at most 25 rounds in the
    # system (closed, emptied or at its budget), so the rounds each took part in differ
    srv = cls(batch=64, rel_gap=1e-4, time_budget=25.0, admission="small_first", incumbent_every=3,
                 round_cap=3)
    reqs = {}
    clock = 0.0
    pending = list(sizes)
    while pending or not srv.idle():
        if pending:                       # two new requests every other round, while others run
            for k, n in pending[:2]:
                m, lo, hi = _req(k, n)
                reqs[k] = srv.submit(k, m, lo, hi, arrival=clock)
            pending = pending[2:]
        srv.step(now=clock)
        clock += 1.0
        assert srv.rounds < 100
    assert srv.max_live >= 3              # requests overlapped on the device
    for k, n in sizes:
        r = srv.done[k]
        assert r.status in ("closed", "emptied", "budget") and r.rounds > 0
        m, lo, hi = _req(k, n)
        mode, threads = r.group[:2]
        g = r.graph
        eng = CrownEngine(g, mode=mode, cta_threads=threads or 128)
        bb = BaB(g, lo, hi, batch=64, engine=eng, model=m.cuda(), incumbent_every=3)
        for _ in range(r.rounds):
            bb.step()
        assert bb.incumbent == r.P
        assert bb.stats.bounded == r.bounded
        g_alone = bb.gap()
        assert (g_alone == r.gap) or (math.isinf(g_alone) and math.isinf(r.gap))


@pytest.mark.parametrize("cls", [Server, DeviceServer])
def test_serve_admission_waits_for_memory(cls):
    """A request that does not fit the HBM budget waits; it is admitted once memory frees up."""
    srv = cls(batch=32, rel_gap=1e-4, time_budget=1e9, hbm_budget=torch.cuda.memory_allocated() + 1)
    m, lo, hi = _req(9, 6)
    r = srv.submit("a", m, lo, hi, arrival=0.0)
    srv.step(now=0.0)
    assert r.status == "waiting" and not srv.live
    srv.hbm_budget = torch.cuda.memory_allocated() + (1 << 30)
    for t in range(200):
        srv.step(now=1.0 + t)
        if srv.idle():
            break
    assert r.status in ("closed", "emptied") and r.admitted == 1.0


def test_serve_compile_pool_same_results():
    """Requests traced and compiled in the spawned pool (compile_workers) give the same results as
    ones compiled in the serving process, once their programs are ready."""
    sizes = [(0, 6), (1, 10), (2, 14), (3, 25)]
    out = {}
    for workers in (0, 2):
        srv = DeviceServer(batch=64, rel_gap=1e-4, time_budget=25.0, incumbent_every=3, round_cap=3,
                           compile_workers=workers)
        try:
            reqs = [srv.submit(k, *_req(k, n), arrival=0.0) for k, n in sizes]
            for r in reqs:
                if r.compiled is not None:
                    r.compiled.result(timeout=600)
            clock = 0.0
            while not srv.idle():
                srv.step(now=clock)
                clock += 1.0
                assert srv.rounds < 100
            out[workers] = {k: (r.P, r.bounded, r.gap, r.rounds, r.group) for k, r in srv.done.items()}
        finally:
            srv.close()
    assert out[0] == out[2]


@pytest.mark.parametrize("cls", [Server, DeviceServer])
def test_serve_preempts_the_widest(cls):
    """With max_live running and preempt on, a narrower arrival replaces the widest live request
    (status "preempted"); without preempt it waits."""
    for preempt in (False, True):
        srv = cls(batch=32, rel_gap=1e-12, time_budget=1e9, max_live=2, preempt=preempt)
        srv.submit("w30", *_req(30, 30), arrival=0.0)
        srv.submit("w20", *_req(20, 20), arrival=0.0)
        srv.step(now=0.0)
        assert set(srv.live) == {"w30", "w20"}
        narrow = srv.submit("n6", *_req(6, 6), arrival=1.0)
        srv.step(now=1.0)
        if preempt:
            assert srv.done["w30"].status == "preempted" and srv.preempted == 1
            assert set(srv.live) == {"w20", "n6"} and narrow.admitted == 1.0
        else:
            assert "w30" in srv.live and narrow.status == "waiting" and srv.preempted == 0
        srv.close()
