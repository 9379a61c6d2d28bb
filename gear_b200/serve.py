"""Serving loop: continuous batching of branch-and-bound requests on one GPU.

Requests (NLP instances: a model, its root box) arrive at any time. Each loop iteration admits
waiting requests while the device memory in use plus the request's estimated footprint stays
within the HBM budget, runs one branch-and-bound round over every admitted instance -- one
persistent CROWN launch per kernel group for all their batches (gear_crown_lower_multi), then
prune / branch / split per instance on the device (``bab.bab_round``) -- and retires the
instances that reached the relative gap, emptied their queue or used up their time budget.
Requests that arrive while others are on the GPU join at the next round, so their work overlaps
on the device with the others'. An instance's search does not depend on what else is in the mix
(its batches, bounds and splits are those of its own BaB run; tested).

The reference solves one instance per process (``complete_verifier/input_split/
batch_branch_and_bound.py``); this loop is the batching layer above that search.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass
from typing import Dict, List, Optional

import torch

from . import _lib, graph as _graph
from .bab import BaB, _Shape, bab_round, relative_gaps
from .engine import PACK_SMEM_LIMIT, SIMT_PACK_ITEMS, _Dag, smem_class
from .program import Program, simt_items


@dataclass
class Request:
    key: object
    model: torch.nn.Module
    lo: torch.Tensor
    hi: torch.Tensor
    rhs: Optional[torch.Tensor]
    arrival: float
    graph: object = None
    admitted: Optional[float] = None
    finished: Optional[float] = None
    gap: float = math.inf
    P: float = math.inf
    rounds: int = 0
    bounded: int = 0
    status: str = "waiting"            # waiting, running, closed, emptied, budget
    group: tuple = ()                  # kernel group: (mode, threads, global working set, smem class)


@dataclass
class _Live:
    req: Request
    dag: _Dag
    bab: BaB
    group: tuple
    cost: int
    est_bytes: int


class Server:
    """Continuous batching of branch-and-bound requests on one device.

    batch: domains popped per instance per round; rel_gap: the closing gap; time_budget: seconds
    an instance may spend in the system (from its arrival); hbm_budget: bytes of device memory
    the loop may hold (default 80% of the device's free memory at start). Instances whose
    box-per-thread state is at most simt_items_max doubles run one box per thread, the others
    one box per CTA of cta_threads threads. round_bytes: when given, an instance pops
    round_bytes / (its algorithmic bytes per box) domains per round, clamped to
    [min_batch, batch]: small instances take large batches (fewer rounds to their gap) and
    large ones do not stretch every round. max_live: at most this many instances run at once
    (a round's host work grows with the number of live instances); the others wait. admission:
    "fifo" admits waiting requests in arrival order, "small_first" the narrowest boxes first
    (the quickest to close). incumbent_every: each instance evaluates its model at the popped
    midpoints on every k-th of its rounds only (BaB(incumbent_every=k)). round_cap: a round
    runs at most this many live instances, the narrowest boxes first (then by arrival); the
    others keep their state and wait for a later round (their budget keeps running)."""

    def __init__(self, device="cuda", batch: int = 256, rel_gap: float = 1e-4, time_budget: float = 30.0,
                 hbm_budget: Optional[int] = None, cta_threads: int = 256, simt_items_max: int = SIMT_PACK_ITEMS,
                 ibp_enhancement: bool = True, clock=time.perf_counter, round_bytes: Optional[int] = None,
                 min_batch: int = 16, max_live: Optional[int] = None, admission: str = "fifo",
                 incumbent_every: int = 1, round_cap: Optional[int] = None):
        if not torch.cuda.is_available():
            raise _lib.GearError("gear_b200 needs a CUDA device (no CPU fallback)")
        self.device = torch.device(device)
        self.batch, self.rel_gap, self.time_budget = batch, rel_gap, time_budget
        self.cta_threads, self.simt_items_max = cta_threads, simt_items_max
        self.ibp_enhancement = ibp_enhancement
        self.clock = clock
        self.round_bytes, self.min_batch = round_bytes, min_batch
        self.live_cap = max_live
        if admission not in ("fifo", "small_first"):
            raise ValueError(f"unknown admission order {admission!r}")
        self.admission = admission
        self.incumbent_every = incumbent_every
        self.round_cap = round_cap
        self.t_bound = 0.0                 # host seconds in the CROWN launches / the rest of a round
        self.t_round = 0.0
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = int(0.8 * (free + torch.cuda.memory_allocated(self.device)))
        self.hbm_budget = hbm_budget
        self.waiting: List[Request] = []
        self.live: Dict[object, _Live] = {}
        self.done: Dict[object, Request] = {}
        self.rounds = 0
        self.bounded = 0
        self.max_live = 0
        self._ws: Dict[tuple, torch.Tensor] = {}

    # ------------------------------------------------------------------ requests
    def submit(self, key, model: torch.nn.Module, lo: torch.Tensor, hi: torch.Tensor,
               rhs: Optional[torch.Tensor] = None, arrival: Optional[float] = None):
        """Queue a request: minimise model(x)[0] s.t. model(x)[1:] <= rhs over lo <= x <= hi."""
        lo = lo.reshape(1, -1).to(torch.float64).cpu()
        hi = hi.reshape(1, -1).to(torch.float64).cpu()
        r = Request(key, model, lo, hi, rhs, self.clock() if arrival is None else arrival)
        r.graph = _graph.trace(model.to(torch.float64).cpu(), lo.repeat(2, 1))
        self.waiting.append(r)
        return r

    def _estimate(self, n, S, prog):
        """Device bytes an instance holds: its program, a queue of 8 batches and one round's
        batch buffers (boxes, lb / lbias / lA, IBP rows)."""
        row = 8 * (2 * n + 2 * S + 1)
        per_box = 8 * (2 * n + 3 * S + S * n)
        prog_b = 4 * prog.int_pool.size + 8 * prog.dbl_pool.size + 4 * (prog.node_arr.size + prog.op_arr.size)
        batch = self.batch
        if self.round_bytes:
            batch = int(min(self.batch, max(self.min_batch, self.round_bytes // max(prog.alg_bytes_per_box(), 1))))
        return prog_b + 8 * batch * row + 2 * batch * per_box

    def _admit(self, now):
        still = []
        order = self.waiting
        if self.admission == "small_first":
            order = sorted(self.waiting, key=lambda r: (r.lo.shape[1], r.arrival))
        for r in order:
            if r.arrival <= now and now - r.arrival > self.time_budget:
                r.status, r.finished = "budget", now     # its budget ran out before a slot freed up
                self.done[r.key] = r
                continue
            if r.arrival > now or (self.live_cap is not None and len(self.live) >= self.live_cap):
                still.append(r)
                continue
            g = r.graph
            prog = Program(g, mode="simt")
            group = ("simt", 0, False, 0)
            if simt_items(prog) > self.simt_items_max:
                prog = Program(g, mode="cta", cta_threads=self.cta_threads, smem_limit=PACK_SMEM_LIMIT)
                group = ("cta", self.cta_threads, prog.pass_global > 0, smem_class(prog))
            est = self._estimate(prog.n, prog.S, prog)
            if torch.cuda.memory_allocated(self.device) + est > self.hbm_budget:
                still.append(r)                      # no room yet: admitted when memory frees up
                continue
            dag = _Dag.from_program(prog)
            model = r.model.to(self.device)
            batch = self.batch
            if self.round_bytes:
                batch = int(min(self.batch, max(self.min_batch, self.round_bytes // max(prog.alg_bytes_per_box(), 1))))
            bab = BaB(g, r.lo, r.hi, rhs=r.rhs, device=str(self.device), batch=batch,
                      engine=_Shape(prog.n, prog.S), model=model, ibp_enhancement=self.ibp_enhancement,
                      incumbent_every=self.incumbent_every)
            r.admitted = now
            r.status = "running"
            r.group = group
            self.live[r.key] = _Live(r, dag, bab, group, prog.alg_bytes_per_box(), est)
        self.waiting = sorted(still, key=lambda r: r.arrival)

    # ------------------------------------------------------------------ one round
    def _bound(self, popped, ibp):
        """One gear_crown_lower_multi launch per kernel group over every popped batch."""
        L = _lib.lib()
        dev = self.device
        stream = torch.cuda.current_stream(dev).cuda_stream
        outs, groups = {}, {}
        for k in popped:
            groups.setdefault(self.live[k].group, []).append(k)
        for gkey, keys in groups.items():
            keys.sort(key=lambda k: -self.live[k].cost)      # expensive boxes first
            args = (_lib.LowerArgs * len(keys))()
            for j, k in enumerate(keys):
                lo, hi = popped[k][0], popped[k][1]
                B, n = lo.shape
                bab = self.live[k].bab
                S = bab.S
                # the instance's own buffers, reused every round (consumed within the round)
                lb = bab._buf("lb", B * S, torch.float64).view(B, S)
                lA = bab._buf("lA", B * S * n, torch.float64).view(B, S, n)
                lbias = bab._buf("lbias", B * S, torch.float64).view(B, S)
                outs[k] = (lb, lA, lbias)
                ib = ibp.get(k)
                args[j] = _lib.LowerArgs(self.live[k].dag.handle.value, lo.data_ptr(), hi.data_ptr(), B, None,
                                         lb.data_ptr(), lA.data_ptr(), lbias.data_ptr(),
                                         ib.data_ptr() if ib is not None else None)
            nbytes = int(L.gear_crown_multi_workspace_bytes(args, len(args)))
            if nbytes < 0:
                _lib.check(-1, "gear_crown_multi_workspace_bytes")
            ws = self._ws.get(gkey)
            if ws is None or ws.numel() < nbytes:
                self._ws[gkey] = None
                ws = self._ws[gkey] = torch.empty(max(nbytes, 8), dtype=torch.uint8, device=dev)
            _lib.check(L.gear_crown_lower_multi(args, len(args), ws.data_ptr(), ws.numel(), stream),
                       "gear_crown_lower_multi")
        return outs

    def _timed_bound(self, popped, ibp):
        t0 = time.perf_counter()
        out = self._bound(popped, ibp)
        self.t_bound += time.perf_counter() - t0
        return out

    def step(self, now: Optional[float] = None) -> int:
        """Admit, run one round over the live instances, retire; returns the domains bounded."""
        given = now is not None
        now = now if given else self.clock()
        self._admit(now)
        self.max_live = max(self.max_live, len(self.live))
        if not self.live:
            return 0
        keys = list(self.live)
        if self.round_cap is not None and len(keys) > self.round_cap:
            keys = sorted(keys, key=lambda k: (self.live[k].req.lo.shape[1], self.live[k].req.arrival))
            keys = keys[:self.round_cap]
        babs = {k: self.live[k].bab for k in keys}
        t0 = time.perf_counter()
        B = bab_round(babs, self._timed_bound, self.ibp_enhancement)
        self.t_round += time.perf_counter() - t0
        self.rounds += 1
        self.bounded += B
        gaps = relative_gaps(babs)
        t = now if given else self.clock()
        for k in list(self.live):
            lv = self.live[k]
            r = lv.req
            status = None
            if k in babs:
                r.rounds += 1
                r.gap, r.P, r.bounded = gaps[k], lv.bab.incumbent, lv.bab.stats.bounded
                if gaps[k] <= self.rel_gap:
                    status = "closed"
                elif len(lv.bab.queue) == 0:
                    status = "emptied"
            if status is None and t - r.arrival > self.time_budget:
                status = "budget"
            if status:
                r.status, r.finished = status, t
                self.done[k] = r
                del self.live[k]
        return B

    def idle(self) -> bool:
        return not self.live and not self.waiting
