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
import pickle
import time
from dataclasses import dataclass
from typing import Dict, List, Optional

import torch

from . import _lib, graph as _graph
from .bab import BaB, _Shape, bab_round, relative_gaps
from .engine import PACK_SMEM_LIMIT, SIMT_PACK_ITEMS, _Dag, smem_class
from .program import Program, simt_items


def _compile_program(graph, cta_threads, simt_items_max):
    """A request's program: one box per thread when its per-box state is small, else one box per
    CTA (the choice of Server._admit)."""
    prog = Program(graph, mode="simt")
    if simt_items(prog) > simt_items_max:
        prog = Program(graph, mode="cta", cta_threads=cta_threads, smem_limit=PACK_SMEM_LIMIT)
    return prog


def _compile_request(blob):
    """Pool job: trace a request's model and compile its program (stripped for the trip back).
    Arguments and result travel as plain pickles (tensors by value): torch's process-sharing
    reductions would hold a file descriptor per tensor in the server for as long as it lives."""
    from .program import stripped
    model, lo, cta_threads, simt_items_max = pickle.loads(blob)
    g = _graph.trace(model, lo.repeat(2, 1))
    return pickle.dumps((g, stripped(_compile_program(g, cta_threads, simt_items_max))))


def _warm(_):
    return 0


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
    status: str = "waiting"            # waiting, running, closed, emptied, budget, memory, preempted
    group: tuple = ()                  # kernel group: (mode, threads, global working set, smem class)
    compiled: object = None            # future of (graph, program) from the compile pool, or None
    program: object = None             # the compiled program once known


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
    (a round's host work grows with the number of live instances); the others wait. compile_workers:
    trace and compile arriving requests in a pool of that many processes (spawned) instead of in
    the loop (a program of n = 2000 takes tens of milliseconds to compile). admission:
    "fifo" admits waiting requests in arrival order, "small_first" the narrowest boxes first
    (the quickest to close). incumbent_every: each instance evaluates its model at the popped
    midpoints on every k-th of its rounds only (BaB(incumbent_every=k)). round_cap: a round
    runs at most this many live instances, the narrowest boxes first (then by arrival); the
    others keep their state and wait for a later round (their budget keeps running). preempt: when
    max_live instances run and an arrived request is narrower (fewer inputs) than the widest of
    them, that one leaves with status "preempted" to make room (the narrow requests are the ones
    that can close within their budget; a wide one would otherwise hold its slot until its
    budget runs out while narrow arrivals wait out theirs)."""

    def __init__(self, device="cuda", batch: int = 256, rel_gap: float = 1e-4, time_budget: float = 30.0,
                 hbm_budget: Optional[int] = None, cta_threads: int = 256, simt_items_max: int = SIMT_PACK_ITEMS,
                 ibp_enhancement: bool = True, clock=time.perf_counter, round_bytes: Optional[int] = None,
                 min_batch: int = 16, max_live: Optional[int] = None, admission: str = "fifo",
                 incumbent_every: int = 1, round_cap: Optional[int] = None, compile_workers: int = 0,
                 preempt: bool = False):
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
        self.preempt = preempt
        self.preempted = 0
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
        self.pool = None
        if compile_workers:
            import multiprocessing as mp
            from concurrent.futures import ProcessPoolExecutor
            self.pool = ProcessPoolExecutor(max_workers=compile_workers, mp_context=mp.get_context("spawn"))
            list(self.pool.map(_warm, range(compile_workers)))   # workers import torch before arrivals

    # ------------------------------------------------------------------ requests
    def submit(self, key, model: torch.nn.Module, lo: torch.Tensor, hi: torch.Tensor,
               rhs: Optional[torch.Tensor] = None, arrival: Optional[float] = None):
        """Queue a request: minimise model(x)[0] s.t. model(x)[1:] <= rhs over lo <= x <= hi.
        With compile_workers, the request's trace and program compile run in the pool and it
        becomes admissible when they are done."""
        lo = lo.reshape(1, -1).to(torch.float64).cpu()
        hi = hi.reshape(1, -1).to(torch.float64).cpu()
        r = Request(key, model, lo, hi, rhs, self.clock() if arrival is None else arrival)
        if self.pool is not None:
            r.compiled = self.pool.submit(_compile_request, pickle.dumps(
                (model.to(torch.float64).cpu(), lo, self.cta_threads, self.simt_items_max)))
        else:
            r.graph = _graph.trace(model.to(torch.float64).cpu(), lo.repeat(2, 1))
        self.waiting.append(r)
        return r

    def close(self):
        """Stop the compile pool (if any)."""
        if self.pool is not None:
            self.pool.shutdown(wait=False, cancel_futures=True)
            self.pool = None

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
            if r.arrival > now:
                still.append(r)
                continue
            if self.live_cap is not None and len(self.live) >= self.live_cap:
                widest = max(self.live, key=lambda k: (self.live[k].req.lo.shape[1], self.live[k].req.arrival)) \
                    if self.preempt and self.live else None
                if widest is None or self.live[widest].req.lo.shape[1] <= r.lo.shape[1] or \
                        (r.compiled is not None and not r.compiled.done()):
                    still.append(r)
                    continue
                self._retire(widest, "preempted", now)
                self.preempted += 1
            if r.compiled is not None:
                if not r.compiled.done():
                    still.append(r)                  # its program is still being compiled
                    continue
                r.graph, prog = pickle.loads(r.compiled.result())
                r.compiled = None
                r.program = prog
            elif r.program is not None:
                prog = r.program
            else:
                prog = _compile_program(r.graph, self.cta_threads, self.simt_items_max)
            group = ("simt", 0, False, 0) if prog.mode == "simt" else \
                ("cta", self.cta_threads, prog.pass_global > 0, smem_class(prog))
            est = self._estimate(prog.n, prog.S, prog)
            if torch.cuda.memory_allocated(self.device) + est > self.hbm_budget:
                still.append(r)                      # no room yet: admitted when memory frees up
                continue
            dag = _Dag.from_program(prog)
            batch = self.batch
            if self.round_bytes:
                batch = int(min(self.batch, max(self.min_batch, self.round_bytes // max(prog.alg_bytes_per_box(), 1))))
            r.admitted = now
            r.status = "running"
            r.group = group
            self.live[r.key] = self._make_live(r, prog, dag, group, batch, est)
        self.waiting = sorted(still, key=lambda r: r.arrival)

    def _retire(self, k, status, t):
        """Move a live request to done with this status (and free its device state)."""
        lv = self.live.pop(k)
        lv.req.status, lv.req.finished = status, t
        self.done[k] = lv.req
        release = getattr(lv, "release", None)
        if release is not None:
            release()

    def _make_live(self, r, prog, dag, group, batch, est):
        """The running state of an admitted request (a host-driven BaB over its device queue)."""
        model = r.model.to(self.device)
        bab = BaB(r.graph, r.lo, r.hi, rhs=r.rhs, device=str(self.device), batch=batch,
                  engine=_Shape(prog.n, prog.S), model=model, ibp_enhancement=self.ibp_enhancement,
                  incumbent_every=self.incumbent_every)
        return _Live(r, dag, bab, group, prog.alg_bytes_per_box(), est)

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
                self._retire(k, status, t)
        return B

    def idle(self) -> bool:
        return not self.live and not self.waiting


@dataclass
class _LiveDQ:
    req: Request
    dag: _Dag
    q: object                  # gear_queue handle (ctypes.c_void_p)
    batch: int
    group: tuple
    cost: int
    est_bytes: int
    cap: int
    boxes: tuple               # (lo, hi) (batch, n): the popped batch
    outs: tuple                # (lb, lA, lbias) of the batch
    ibp: Optional[torch.Tensor]
    status: torch.Tensor       # (10,) float64: 8 counters, dual bound, incumbent (written on the device)
    graphs: dict               # "pop", "pop_propose", "step": CUDA graphs of the instance's round
    keep: tuple                # tensors the graphs read or write (kept alive with them)

    def release(self):
        self.graphs = {}
        if self.q is not None and self.q.value:
            _lib.lib().gear_queue_destroy(self.q)
            self.q = None


class DeviceServer(Server):
    """The serving loop with every admitted request's queue on the device and its round captured
    into CUDA graphs once, at admission.

    Each request gets a gear_queue (capacity from queue_bytes) and three graphs: its pop, its pop
    followed by the incumbent proposal (the model at the popped midpoints), and its
    gear_bab_step_bounded followed by a copy of its counters, dual bound and incumbent into a
    status row. A round replays the pop graph of every running request, makes one prepared
    many-instance CROWN launch per kernel group for all their batches (re-planned only when the
    set of running requests changes), replays their step graphs and reads every status row in one
    copy: the host cost of a request per round is two graph launches instead of dozens of launches
    and a synchronisation. Same admission, time budget and retirement rules as Server, and each
    request's search is the one BaB runs for it alone (tested)."""

    def __init__(self, *args, queue_bytes: int = 256 << 20, **kwargs):
        super().__init__(*args, **kwargs)
        self.queue_bytes = queue_bytes
        self._plan_keys = None
        self._plans = []

    def _estimate(self, n, S, prog):
        batch = self.batch
        if self.round_bytes:
            batch = int(min(self.batch, max(self.min_batch, self.round_bytes // max(prog.alg_bytes_per_box(), 1))))
        per_box = 8 * (2 * n + 4 * S + S * n)
        prog_b = 4 * prog.int_pool.size + 8 * prog.dbl_pool.size + 4 * (prog.node_arr.size + prog.op_arr.size)
        return prog_b + self._cap(n, S, batch) * (8 * (2 * n + S + 2) + 12) + 4 * batch * per_box

    def _cap(self, n, S, batch):
        return int(max(4 * batch + 1, min(256 * batch, self.queue_bytes // (8 * (2 * n + S + 2) + 12))))

    def _make_live(self, r, prog, dag, group, batch, est):
        import ctypes
        L = _lib.lib()
        dev = self.device
        n, S = prog.n, prog.S
        cap = self._cap(n, S, batch)
        lo = r.lo.reshape(-1).contiguous()
        hi = r.hi.reshape(-1).contiguous()
        h = ctypes.c_void_p()
        _lib.check(L.gear_queue_create(n, S, cap, batch, lo.data_ptr(), hi.data_ptr(), ctypes.byref(h)),
                   "gear_queue_create")
        plo = torch.empty(batch, n, dtype=torch.float64, device=dev)
        phi = torch.empty_like(plo)
        lb = torch.empty(batch, S, dtype=torch.float64, device=dev)
        lA = torch.empty(batch, S, n, dtype=torch.float64, device=dev)
        lbias = torch.empty_like(lb)
        ibp = torch.empty_like(lb) if self.ibp_enhancement else None
        inc = torch.full((1,), math.inf, dtype=torch.float64, device=dev)
        x_best = ((r.lo + r.hi) / 2).reshape(-1).to(dev)
        rr = r.rhs if r.rhs is not None else torch.zeros(S - 1, dtype=torch.float64)
        rhs = torch.cat([rr.to(torch.float64).reshape(-1).to(dev), torch.zeros(1, dtype=torch.float64, device=dev)])
        counters = torch.zeros(8, dtype=torch.int64, device=dev)
        dual = torch.full((1,), -math.inf, dtype=torch.float64, device=dev)
        status = torch.zeros(10, dtype=torch.float64, device=dev)
        model = r.model.to(dev)

        def pop():
            st = torch.cuda.current_stream(dev).cuda_stream
            _lib.check(L.gear_queue_pop(h, plo.data_ptr(), phi.data_ptr(), st), "gear_queue_pop")

        def propose():
            with torch.no_grad():
                x = (plo + phi) / 2
                y = model(x)
                feas = (y[:, 1:] <= rhs[:S - 1]).all(1) if y.shape[1] > 1 else \
                    torch.ones(y.shape[0], dtype=torch.bool, device=dev)
                obj = torch.where(feas, y[:, 0], torch.full_like(y[:, 0], math.inf))
                best = obj.min(0)
                val = best.values.reshape(1)
                pt = x.index_select(0, best.indices.reshape(1)).reshape(-1)
                x_best.copy_(torch.where(val < inc, pt, x_best))
                inc.copy_(torch.minimum(inc, val))

        def step():
            st = torch.cuda.current_stream(dev).cuda_stream
            _lib.check(L.gear_bab_step_bounded(h, plo.data_ptr(), phi.data_ptr(), lb.data_ptr(), lA.data_ptr(),
                                               lbias.data_ptr(), inc.data_ptr(), rhs.data_ptr(), 1e-3, 1e-3, st),
                       "gear_bab_step_bounded")
            _lib.check(L.gear_queue_counters(h, counters.data_ptr(), dual.data_ptr(), st), "gear_queue_counters")
            status.copy_(torch.cat([counters.to(torch.float64), dual, inc]))

        graphs = {}
        for name, fns in (("pop", (pop,)), ("pop_propose", (pop, propose)), ("step", (step,))):
            gr = torch.cuda.CUDAGraph()
            with torch.cuda.graph(gr):
                for f in fns:
                    f()
            graphs[name] = gr
        keep = (plo, phi, lb, lA, lbias, ibp, inc, x_best, rhs, counters, dual, model, lo, hi)
        return _LiveDQ(r, dag, h, batch, group, prog.alg_bytes_per_box(), est, cap, (plo, phi), (lb, lA, lbias), ibp,
                       status, graphs, keep)

    def _prepare(self, keys):
        """One prepared many-instance launch per kernel group for these requests' batches."""
        L = _lib.lib()
        for h, _ in self._plans:
            L.gear_crown_multi_plan_destroy(h)
        self._plans = []
        groups = {}
        for k in keys:
            groups.setdefault(self.live[k].group, []).append(k)
        import ctypes
        for gkey, ks in groups.items():
            ks.sort(key=lambda k: -self.live[k].cost)        # expensive boxes first
            args = (_lib.LowerArgs * len(ks))()
            for j, k in enumerate(ks):
                lv = self.live[k]
                (plo, phi), (lb, lA, lbias) = lv.boxes, lv.outs
                args[j] = _lib.LowerArgs(lv.dag.handle.value, plo.data_ptr(), phi.data_ptr(), lv.batch, None,
                                         lb.data_ptr(), lA.data_ptr(), lbias.data_ptr(),
                                         lv.ibp.data_ptr() if lv.ibp is not None else None)
            nbytes = int(L.gear_crown_multi_workspace_bytes(args, len(args)))
            if nbytes < 0:
                _lib.check(-1, "gear_crown_multi_workspace_bytes")
            ws = torch.empty(max(nbytes, 8), dtype=torch.uint8, device=self.device)
            h = ctypes.c_void_p()
            _lib.check(L.gear_crown_multi_prepare(args, len(args), ws.data_ptr(), ws.numel(), ctypes.byref(h)),
                       "gear_crown_multi_prepare")
            self._plans.append((h, ws))
        self._plan_keys = tuple(keys)

    def step(self, now: Optional[float] = None) -> int:
        """Admit, run one round over the running requests, retire; returns the domains bounded."""
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
        t0 = time.perf_counter()
        if self._plan_keys != tuple(keys):
            self._prepare(keys)
        every = max(1, int(self.incumbent_every))
        for k in keys:
            lv = self.live[k]
            lv.graphs["pop_propose" if lv.req.rounds % every == 0 else "pop"].replay()
        t1 = time.perf_counter()
        L = _lib.lib()
        st = torch.cuda.current_stream(self.device).cuda_stream
        for h, _ in self._plans:
            _lib.check(L.gear_crown_multi_launch(h, st), "gear_crown_multi_launch")
        self.t_bound += time.perf_counter() - t1
        for k in keys:
            self.live[k].graphs["step"].replay()
        rows = torch.stack([self.live[k].status for k in keys]).cpu().tolist()
        self.t_round += time.perf_counter() - t0
        self.rounds += 1
        t = now if given else self.clock()
        bounded = 0
        for k, row in zip(keys, rows):
            lv = self.live[k]
            r = lv.req
            r.rounds += 1
            prev = r.bounded
            r.bounded = int(row[3])
            bounded += r.bounded - prev
            r.P = row[9]
            r.gap = BaB._gap(row[9], row[8])
        self.bounded += bounded
        for k in list(self.live):
            lv = self.live[k]
            r = lv.req
            status = None
            if k in keys:
                row = rows[keys.index(k)]
                if r.gap <= self.rel_gap:
                    status = "closed"
                elif int(row[0]) == 0:
                    status = "emptied"
                elif int(row[0]) + lv.batch > lv.cap or int(row[7]):
                    status = "memory"
            if status is None and t - r.arrival > self.time_budget:
                status = "budget"
            if status:
                self._retire(k, status, t)
        if self._plan_keys is not None and any(k not in self.live for k in self._plan_keys):
            self._plan_keys = None          # re-plan next round (its instances' buffers may be freed)
            for h, _ in self._plans:
                L.gear_crown_multi_plan_destroy(h)
            self._plans = []
        return bounded
