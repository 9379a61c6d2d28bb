"""Device BaB kernels (libgear_b200.so) against the BaB oracle, and BaB to gap."""
import math
import os

import numpy as np
import pytest
import torch

from oracle import bab as obab

pytestmark = pytest.mark.gpu
D = np.load(os.path.join(os.path.dirname(__file__), "golden", "bab_steps.npz"))
CASES = sorted({k.split("_")[0] for k in D.files})


def _t(a, dt=torch.float64):
    return torch.tensor(a, dtype=dt, device="cuda").contiguous()


@pytest.mark.parametrize("c", CASES)
def test_device_step_kernels_match_reference_fixture(c):
    from gear_b200 import _lib
    L = _lib.lib()
    g = lambda k: D[f"{c}_{k}"]
    lb, thr, lA, lo, hi = _t(g("lb")), _t(g("thr")), _t(g("lA")), _t(g("lo")), _t(g("hi"))
    B, S, n = lA.shape
    st = torch.cuda.current_stream().cuda_stream
    keep = torch.empty(B, dtype=torch.uint8, device="cuda")
    kept = torch.empty(B, dtype=torch.int32, device="cuda")
    nk = torch.zeros(1, dtype=torch.int32, device="cuda")
    disc = torch.full((1,), math.inf, dtype=torch.float64, device="cuda")
    ws = torch.empty(int(L.gear_bab_workspace_bytes(B)), dtype=torch.uint8, device="cuda")
    _lib.check(L.gear_bab_prune(lb.data_ptr(), thr.data_ptr(), B, S, keep.data_ptr(), kept.data_ptr(),
                                nk.data_ptr(), disc.data_ptr(), ws.data_ptr(), ws.numel(), st), "prune")
    torch.cuda.synchronize()
    assert np.array_equal(keep.cpu().numpy().astype(bool), g("keep"))
    K = int(nk.item())
    assert np.array_equal(kept[:K].cpu().numpy(), np.nonzero(g("keep"))[0])
    _, dmin = obab.prune_mask(g("lb"), g("thr"))
    assert float(disc.item()) == dmin
    lbf = _t(g("lb_f"))
    idx = torch.empty(B, dtype=torch.int32, device="cuda")
    rw = _t(g("root_w"))
    _lib.check(L.gear_bab_branch(lA.data_ptr(), lo.data_ptr(), hi.data_ptr(), lbf.data_ptr(), thr.data_ptr(), B, S,
                                 n, rw.data_ptr(), 1e-3, 1e-3, idx.data_ptr(), ws.data_ptr(), ws.numel(), st), "branch")
    torch.cuda.synchronize()
    assert np.array_equal(idx.cpu().numpy(), g("idx"))
    # split + child keys on the reference's kept list
    kt = _t(g("kept"), torch.int32)
    Kr = kt.numel()
    clo = torch.empty(2 * Kr, n, dtype=torch.float64, device="cuda")
    chi = torch.empty_like(clo)
    ck = torch.empty(2 * Kr, S, dtype=torch.float64, device="cuda")
    lbias = _t(g("lbias"))
    _lib.check(L.gear_bab_split(lo.data_ptr(), hi.data_ptr(), kt.data_ptr(), Kr, n, idx.data_ptr(), lbf.data_ptr(),
                                lA.data_ptr(), lbias.data_ptr(), S, clo.data_ptr(), chi.data_ptr(), ck.data_ptr(), st),
               "split")
    torch.cuda.synchronize()
    assert np.array_equal(clo.cpu().numpy(), g("child_lo")) and np.array_equal(chi.cpu().numpy(), g("child_hi"))
    ref = g("child_key")
    assert np.all(np.abs(ck.cpu().numpy() - ref) <= 1e-14 * np.maximum(1.0, np.abs(ref)))
    # queue order
    key = _t(g("qkey"))
    ids = torch.arange(B, dtype=torch.int64, device="cuda")
    slots = torch.arange(B, dtype=torch.int32, device="cuda")
    n2 = 1 << (B - 1).bit_length()
    order = torch.empty(n2, dtype=torch.int32, device="cuda")
    _lib.check(L.gear_queue_order(key.data_ptr(), ids.data_ptr(), slots.data_ptr(), B, order.data_ptr(), n2, st), "order")
    torch.cuda.synchronize()
    assert np.array_equal(order[:B].cpu().numpy(), g("order"))


def test_bab_closes_gap_and_is_sound():
    from gear_b200 import problems, graph
    from gear_b200.bab import BaB
    m = problems.make_instance("quad_exp_n10", 0)
    lo, hi = problems.root_box("quad_exp_n10")
    g = graph.trace(m, lo.repeat(2, 1))
    bb = BaB(g, lo, hi, batch=2048, model=m.cuda())
    P, Dd, gap = bb.run(rel_gap=1e-4, max_iterations=400, time_limit=120)
    assert gap <= 1e-4, (P, Dd, gap, bb.stats.iterations)
    # the dual bound is below every sampled feasible objective value
    x = lo + (hi - lo) * torch.rand(200000, lo.shape[1], dtype=torch.float64)
    y = m(x.cuda()).cpu()
    feas = (y[:, 1:] <= 0).all(1)
    assert Dd <= float(y[feas, 0].min()) + 1e-9


def test_constrained_concretisation_bab_is_sound_and_not_slower():
    """The complete-clipping mode: children keep their parents' planes as cut rows and the
    objective row is concretised over box and cuts. It closes the gap in at most as many
    iterations as plain BaB, and its dual bound stays below sampled feasible values."""
    from gear_b200 import problems, graph
    from gear_b200.bab import BaB
    m = problems.make_instance("quad_exp_n10", 0)
    lo, hi = problems.root_box("quad_exp_n10")
    g = graph.trace(m, lo.repeat(2, 1))
    plain = BaB(g, lo, hi, batch=2048, model=m.cuda())
    plain.run(rel_gap=1e-4, max_iterations=400, time_limit=120)
    cons = BaB(g, lo, hi, batch=2048, model=m.cuda(), constrained=True)
    P, Dd, gap = cons.run(rel_gap=1e-4, max_iterations=400, time_limit=120)
    assert gap <= 1e-4, (P, Dd, gap, cons.stats.iterations)
    assert cons.stats.iterations <= plain.stats.iterations
    x = lo + (hi - lo) * torch.rand(200000, lo.shape[1], dtype=torch.float64)
    y = m(x.cuda()).cpu()
    feas = (y[:, 1:] <= 0).all(1)
    assert Dd <= float(y[feas, 0].min()) + 1e-9


@pytest.mark.parametrize("N", [3000, 8192, 10000])
def test_queue_order_single_and_multi_launch(N):
    """gear_queue_order: one shared-memory CTA up to 8192 slots, the multi-launch network
    beyond; both give (key desc, insertion id asc), ties included."""
    from gear_b200 import _lib
    g = np.random.default_rng(N)
    key = np.round(g.normal(size=N), 1)                 # many ties
    key[::97] = -np.inf
    ids = g.permutation(N).astype(np.int64)
    slots = g.permutation(N).astype(np.int32)[: N - 5]   # a subset of the slots is active
    n = slots.size
    n2 = 1 << (n - 1).bit_length()
    k_t = torch.tensor(key, device="cuda")
    i_t = torch.tensor(ids, device="cuda")
    s_t = torch.tensor(slots, device="cuda")
    order = torch.empty(n2, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().gear_queue_order(k_t.data_ptr(), i_t.data_ptr(), s_t.data_ptr(), n, order.data_ptr(), n2, st),
               "gear_queue_order")
    torch.cuda.synchronize()
    ref = slots[np.lexsort((ids[slots], -key[slots]))]
    assert np.array_equal(order[:n].cpu().numpy(), ref)


def test_ordered_queue_pops_what_a_full_sort_pops():
    """Pushes merged into the ordered list and pops from its tail give, batch by batch, what a
    full sort of the open domains by (key descending, id ascending) gives; keys with many ties."""
    from gear_b200.bab import DomainQueue
    g = torch.Generator().manual_seed(7)
    n, S = 3, 2
    q = DomainQueue(n, S, 16, "cuda")
    ref = []                                           # (key, id) of the open domains
    next_id = 0
    for rnd in range(12):
        m = int(torch.randint(1, 3000, (1,), generator=g))
        key = torch.randint(-5, 5, (m, S), generator=g).to(torch.float64) / 2
        key[::7, 0] = float("-inf")
        lo = torch.rand(m, n, generator=g, dtype=torch.float64)
        q.push(lo.cuda(), (lo + 1).cuda(), key.cuda(), torch.zeros(m, S, dtype=torch.float64, device="cuda"))
        ref += [(float(key[i, 0]), next_id + i) for i in range(m)]
        next_id += m
        b = int(torch.randint(1, 2500, (1,), generator=g))
        popped = q.pop(b)
        ref.sort(key=lambda t: (-t[0], t[1]))
        want, ref = ref[len(ref) - min(b, len(ref)):], ref[:len(ref) - min(b, len(ref))]
        got = popped[2][:, 0].cpu().tolist()
        assert got == [k for k, _ in want]
        assert len(q) == len(ref)
        assert float(q.min_key_tensor()) == (min(k for k, _ in ref) if ref else float("inf"))
