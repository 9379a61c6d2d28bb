"""Input-space branch and bound on the GPU: select / bound / prune / branch / split.

One iteration mirrors the reference's reordered loop (``complete_verifier/input_split/
batch_branch_and_bound.py:275-652`` with ``reorder_bab``) restricted to the hot path:

  select   the domains with the smallest objective key (queue sorted by the objective
           row's lower bound, descending, ties by insertion id; the batch is the tail)
           -- ``branching_domains.py:831-962, 1171``
  bound    CROWN ``compute_bounds`` over the batch (the GPU megakernel)
           -- ``bounding.py:124``
  prune    ``get_remaining_index`` in solving mode -- ``branching_domains.py:412-558``
  branch   SB score with sb_sum, top-1, width guard -- ``branching_heuristics.py:25-202``
  split    midpoint bisection, children [upper halves; lower halves] -- ``split.py:26-122``
  keys     children keyed by max(parent lb, parent plane minimum over the child box)
           -- ``batch_branch_and_bound.py:189-225``

Every step is a kernel of libgear_b200.so on device-resident data; the host only reads the
number of surviving domains once per iteration. The global dual bound D is the minimum
objective key over the open domains, capped by the smallest threshold of the domains
discarded by the objective row (``batch_branch_and_bound.py:628-636``).
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field
from typing import List, Optional

import torch

from . import _lib
from .engine import CrownEngine
from .graph import Graph


def _p(t):
    return None if t is None else t.data_ptr()


@dataclass
class BaBStats:
    iterations: int = 0
    bounded: int = 0
    pruned: int = 0
    clipped_empty: int = 0
    history: List[dict] = field(default_factory=list)


class DomainQueue:
    """Device-resident pool of open subdomains (structure of arrays over slots).

    The active slot list is kept in the reference's pop order, (objective key descending,
    insertion id ascending): keys do not change while a domain is queued, so a push sorts only
    the new domains and merges them in (gear_queue_merge), and a pop takes the list's tail, the
    same batch a full sort of the open domains gives."""

    def __init__(self, n: int, S: int, capacity: int, device, cuts: bool = False):
        """cuts: also keep per domain the cut rows A (S, n), b (S) inherited from its parent."""
        self.n, self.S, self.device = n, S, device
        self.cuts = cuts
        self.cap = 0
        self.lo = self.hi = self.key = self.thr = self.ids = self.cutA = self.cutb = None
        self.free: List[torch.Tensor] = []
        self.active = torch.empty(0, dtype=torch.int32, device=device)
        self.next_id = 0
        self._pop_bufs = {}
        self._grow(max(capacity, 1))

    def _fields(self):
        f = [("lo", self.n), ("hi", self.n), ("key", self.S), ("thr", self.S)]
        if self.cuts:
            f += [("cutA", self.S * self.n), ("cutb", self.S)]
        return f

    def _grow(self, cap):
        dev = self.device
        new = dict(lo=torch.empty(cap, self.n, dtype=torch.float64, device=dev),
                   hi=torch.empty(cap, self.n, dtype=torch.float64, device=dev),
                   key=torch.full((cap, self.S), math.inf, dtype=torch.float64, device=dev),
                   thr=torch.empty(cap, self.S, dtype=torch.float64, device=dev),
                   ids=torch.zeros(cap, dtype=torch.int64, device=dev),
                   key0=torch.full((cap,), math.inf, dtype=torch.float64, device=dev))
        if self.cuts:
            new["cutA"] = torch.empty(cap, self.S * self.n, dtype=torch.float64, device=dev)
            new["cutb"] = torch.empty(cap, self.S, dtype=torch.float64, device=dev)
        if self.cap:
            for k in new:
                new[k][:self.cap] = getattr(self, k)
        for k, v in new.items():
            setattr(self, k, v)
        self.free_slots = torch.cat([getattr(self, "free_slots", torch.empty(0, dtype=torch.int32, device=dev)),
                                     torch.arange(self.cap, cap, dtype=torch.int32, device=dev)])
        self.cap = cap

    def __len__(self):
        return int(self.active.numel())

    def push(self, lo, hi, key, thr, cutA=None, cutb=None):
        m = lo.shape[0]
        if m == 0:
            return
        if self.free_slots.numel() < m:
            self._grow(max(2 * self.cap, self.cap + m))
        slots = self.free_slots[-m:]
        self.free_slots = self.free_slots[:-m]
        L = _lib.lib()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        vals = {"lo": lo, "hi": hi, "key": key, "thr": thr, "cutA": cutA, "cutb": cutb}
        for name, w in self._fields():
            src = vals[name].reshape(m, w).contiguous()
            _lib.check(L.gear_scatter_rows(_p(src), _p(slots), m, w, _p(getattr(self, name)), stream),
                       "gear_scatter_rows")
        sl = slots.long()
        self.ids[sl] = torch.arange(self.next_id, self.next_id + m, device=self.device)
        self.key0[sl] = key.reshape(m, self.S)[:, 0]
        self.next_id += m
        # the new domains in pop order, merged into the ordered active list
        n2 = 1 << max(0, (m - 1).bit_length())
        order = torch.empty(max(n2, 1), dtype=torch.int32, device=self.device)
        _lib.check(L.gear_queue_order(_p(self.key0), _p(self.ids), _p(slots), m, _p(order), order.numel(), stream),
                   "gear_queue_order")
        na = int(self.active.numel())
        merged = torch.empty(na + m, dtype=torch.int32, device=self.device)
        _lib.check(L.gear_queue_merge(_p(self.key0), _p(self.ids), _p(self.active) if na else None, na, _p(order), m,
                                      _p(merged), stream), "gear_queue_merge")
        self.active = merged

    def pop(self, batch: int):
        """The last `batch` domains in (objective key desc, id asc) order: the tail of the ordered
        active list. The returned rows live in buffers the next pop reuses."""
        N = len(self)
        b = min(batch, N)
        L = _lib.lib()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        slots = self.active[N - b:]
        self.active = self.active[:N - b]
        out = []
        for name, w in self._fields():
            # popped rows live until the end of the iteration that pops them: reused buffers
            buf = self._pop_bufs.get(name)
            if buf is None or buf.numel() < b * w:
                buf = self._pop_bufs[name] = torch.empty(max(b * w, 1), dtype=torch.float64, device=self.device)
            dst = buf[:b * w].view(b, w)
            _lib.check(L.gear_gather_rows(_p(getattr(self, name)), _p(slots), b, w, _p(dst), stream),
                       "gear_gather_rows")
            out.append(dst)
        self.free_slots = torch.cat([self.free_slots, slots])
        return out

    def min_key(self) -> float:
        return float(self.min_key_tensor())

    def min_key_tensor(self) -> torch.Tensor:
        """The smallest objective key of the open domains as a (1,) device tensor (no host
        read): the key of the ordered list's last slot."""
        if len(self) == 0:
            return torch.full((1,), math.inf, dtype=torch.float64, device=self.device)
        return self.key0[self.active[-1:].long()]


class BaB:
    """Branch and bound to a relative gap on one NLP instance (x in [lo, hi]).

    The model maps x (B, n) to y (B, 1 + m): row 0 the objective, rows 1..m constraints
    g_k(x) <= rhs_k (rhs given already relaxed by the instance's feasibility tolerance)."""

    def __init__(self, graph: Graph, lo: torch.Tensor, hi: torch.Tensor, rhs: Optional[torch.Tensor] = None,
                 device="cuda", batch: int = 4096, sb_coeff_thresh: float = 1e-3, engine: Optional[CrownEngine] = None,
                 engine_mode: str = "auto", cta_threads: int = 128,
                 sb_min_width_ratio: float = 1e-3, model: Optional[torch.nn.Module] = None,
                 constrained: bool = False, max_constraint_rows: int = 16, clip: bool = False,
                 clip_iterations: int = 1, ibp_enhancement: bool = True, incumbent_every: int = 1,
                 cuts_everywhere: bool = True):
        """constrained: the reference's complete clipping mode's constrained concretisation
        (batch_branch_and_bound.py:422-428): every child keeps its parent's planes
        lA_j x + lbias_j <= thr_j as cut rows, and the objective row of its CROWN bound is
        concretised over the box intersected with them (concretize_func.py:415-850, at most
        max_constraint_rows rows per box, the f3 setting's concretize_max_constraint_rows);
        a box that the cuts exclude is pruned. cuts_everywhere (the reference's behaviour): the
        cut rows enter every concretisation of the CROWN call, the intermediate passes'
        included (PerturbationLpNorm(constraints=...), gear_crown_lower_cuts, the plain form's
        launch sequence); False: the fused kernel bounds the box and only the objective row is
        concretised again over box ∩ rows (looser, one fused launch).
        clip: domain clipping of the children with their parent's planes (clip.py:237-470,
        clip_iterations rounds); children that become empty are dropped.
        ibp_enhancement: every bound is the larger of CROWN's and the plain IBP bound of the
        output (get_lower_bound_with_ibp_enhancement, bounding.py:789-948, on by default in the
        reference).
        incumbent_every: evaluate the model at the popped boxes' midpoints (the primal points of
        the incumbent) on every k-th iteration only; 1 = every iteration."""
        self.device = torch.device(device)
        self.graph = graph
        # an engine can be shared between runs on the same graph (its kernel choice is kept)
        self.engine = engine if engine is not None else CrownEngine(graph, mode=engine_mode, cta_threads=cta_threads)
        if self.engine.mode == "auto":
            # pick the kernel once, at the full batch, on sub-boxes of the root box
            gen = torch.Generator(device="cpu").manual_seed(0)
            r0, r1 = lo.reshape(1, -1).cpu(), hi.reshape(1, -1).cpu()
            c = r0 + (r1 - r0) * torch.rand(batch, r0.shape[1], generator=gen, dtype=torch.float64)
            w = (r1 - r0) * torch.rand(batch, r0.shape[1], generator=gen, dtype=torch.float64) * 0.25
            sl, su = torch.maximum(r0, c - w), torch.minimum(r1, c + w)
            self.engine.freeze(sl.to(self.device), su.to(self.device))
        self.n = self.engine.n
        self.S = self.engine.S
        self.batch = batch
        self.coeff_thresh = sb_coeff_thresh
        self.min_width_ratio = sb_min_width_ratio
        self.model = model
        lo = lo.reshape(1, -1).to(self.device, torch.float64)
        hi = hi.reshape(1, -1).to(self.device, torch.float64)
        self.root_width = (hi - lo).reshape(-1).contiguous()
        self.rhs = (torch.zeros(self.S - 1, dtype=torch.float64) if rhs is None else rhs.to(torch.float64)).to(self.device)
        self.incumbent = math.inf
        self.x_best = None
        self.incumbent_every = max(1, int(incumbent_every))
        self._bufs = {}
        # the incumbent on the device: thresholds read it there, so proposing a better one needs
        # no host read; the host copy (self.incumbent) is refreshed with the survivor count
        self._inc_dev = torch.full((1,), math.inf, dtype=torch.float64, device=self.device)
        self._x_best_dev = None
        self.ibp_enhancement = ibp_enhancement
        self.clip = clip
        self.clip_iterations = clip_iterations
        self.constrained = constrained
        self.max_constraint_rows = max_constraint_rows
        self.cut_engine = None
        if constrained and cuts_everywhere:
            from .engine import CutEngine
            self.cut_engine = CutEngine(graph, cta_threads=cta_threads,
                                        tie_rule=getattr(self.engine, "tie_rule", "reference"),
                                        max_rows=max_constraint_rows)
        self.queue = DomainQueue(self.n, self.S, 4 * batch, self.device, cuts=constrained)
        key = torch.full((1, self.S), -math.inf, dtype=torch.float64, device=self.device)
        cutA = torch.zeros(1, self.S * self.n, dtype=torch.float64, device=self.device) if constrained else None
        cutb = torch.full((1, self.S), -1.0, dtype=torch.float64, device=self.device) if constrained else None
        self.queue.push(lo, hi, key, self._thresholds(1), cutA, cutb)
        self.disc_min = torch.full((1,), math.inf, dtype=torch.float64, device=self.device)
        self.stats = BaBStats()
        self._ws = torch.empty(1, dtype=torch.uint8, device=self.device)

    def _thresholds(self, m):
        t = torch.empty(m, self.S, dtype=torch.float64, device=self.device)
        t[:, 0] = self.incumbent
        t[:, 1:] = self.rhs
        return t

    def _ws_bytes(self, nbytes):
        if self._ws.numel() < nbytes:
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        return self._ws

    def _buf(self, name, n, dtype):
        """A flat scratch tensor of at least n elements kept across iterations (every use ends
        within the iteration that takes it; the stream orders the next one after it)."""
        t = self._bufs.get(name)
        if t is None or t.numel() < n or t.dtype != dtype:
            t = self._bufs[name] = torch.empty(max(n, 1), dtype=dtype, device=self.device)
        return t[:n]

    def incumbent_candidate(self, x: torch.Tensor):
        """Best feasible objective among the primal points x (model in float64), on the device:
        (value (1,) tensor, +inf if none, and its point), without a host read. With
        incumbent_every = k only every k-th iteration evaluates (None otherwise)."""
        if self.model is None or x.numel() == 0 or self.stats.iterations % self.incumbent_every:
            return None
        with torch.no_grad():
            y = self.model(x.to(self.device, torch.float64))
        feas = (y[:, 1:] <= self.rhs).all(1) if y.shape[1] > 1 else torch.ones(y.shape[0], dtype=torch.bool,
                                                                                device=self.device)
        obj = torch.where(feas, y[:, 0], torch.full_like(y[:, 0], math.inf))
        best = obj.min(0)
        # index_select keeps the index on the device (x[tensor] would read it on the host)
        return best.values.reshape(1), x.index_select(0, best.indices.reshape(1)).reshape(-1)

    def propose_incumbent(self, x: torch.Tensor):
        """Fold the best feasible point among x into the device-side incumbent (no host read)."""
        c = self.incumbent_candidate(x)
        if c is None:
            return
        val, pt = c
        pt = pt.reshape(-1)
        if self._x_best_dev is None:
            self._x_best_dev = pt.clone()
        else:
            self._x_best_dev = torch.where(val < self._inc_dev, pt, self._x_best_dev)
        self._inc_dev = torch.minimum(self._inc_dev, val)

    def sync_incumbent(self, value: float):
        """Host copy of the device incumbent (value read from it by the caller)."""
        if value < self.incumbent:
            self.incumbent = value
            self.x_best = self._x_best_dev.clone()

    def update_incumbent(self, x: torch.Tensor):
        """Primal points: evaluate the model (float64) and keep the best feasible objective."""
        self.propose_incumbent(x)
        self.sync_incumbent(float(self._inc_dev))

    def dual_bound(self) -> float:
        """min(open objective keys, smallest discarded threshold): one host read."""
        return float(torch.minimum(self.queue.min_key_tensor(), self.disc_min))

    @staticmethod
    def _gap(P, D):
        if not math.isfinite(P):
            return math.inf
        if not math.isfinite(D):
            return 0.0 if D > 0 else math.inf
        return (P - D) / max(1.0, abs(P), abs(D))

    def gap(self) -> float:
        return self._gap(self.incumbent, self.dual_bound())

    def select(self):
        """Pop the next batch (thresholds at the current incumbent): [lo, hi, key, thr, (cuts)]."""
        popped = self.queue.pop(self.batch)
        popped[3][:, 0] = self._inc_dev
        return popped

    def prune_branch(self, popped, lb, lA, lbias):
        """Prune against the thresholds and pick split variables on the device (no host read):
        the state finish() needs, with the survivor count in state["nk"]."""
        lo, hi, key, thr = popped[:4]
        thr[:, 0] = self._inc_dev                         # after this iteration's proposals
        if self.constrained:
            self._constrained_objective(lo, hi, lb, lA, lbias, popped[4], popped[5])
        B = lo.shape[0]
        L = _lib.lib()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        keep = self._buf("keep", B, torch.uint8)
        kept = self._buf("kept", B, torch.int32)
        nk = self._buf("nk", 1, torch.int32)              # written by the prune (0 first)
        ws = self._ws_bytes(int(L.gear_bab_workspace_bytes(B)))
        _lib.check(L.gear_bab_prune(_p(lb), _p(thr), B, self.S, _p(keep), _p(kept), _p(nk), _p(self.disc_min),
                                    _p(ws), ws.numel(), stream), "gear_bab_prune")
        split_idx = self._buf("split", B, torch.int32)
        _lib.check(L.gear_bab_branch(_p(lA), _p(lo), _p(hi), _p(lb), _p(thr), B, self.S, self.n,
                                     _p(self.root_width), self.coeff_thresh, self.min_width_ratio, _p(split_idx),
                                     _p(ws), ws.numel(), stream), "gear_bab_branch")
        return {"popped": popped, "lb": lb, "lA": lA, "lbias": lbias, "kept": kept, "nk": nk,
                "split_idx": split_idx, "B": B}

    def finish(self, st, K: int):
        """Split the K survivors (K = st["nk"], read by the caller) and push the children."""
        lo, hi, key, thr = st["popped"][:4]
        lb, lA, lbias, kept, split_idx, B = st["lb"], st["lA"], st["lbias"], st["kept"], st["split_idx"], st["B"]
        q = self.queue
        L = _lib.lib()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        self.stats.iterations += 1
        self.stats.bounded += B
        self.stats.pruned += B - K
        if K > 0:
            clo = self._buf("clo", 2 * K * self.n, torch.float64).view(2 * K, self.n)
            chi = self._buf("chi", 2 * K * self.n, torch.float64).view(2 * K, self.n)
            ckey = self._buf("ckey", 2 * K * self.S, torch.float64).view(2 * K, self.S)
            parents = torch.cat([kept[:K], kept[:K]])
            if not self.clip:
                _lib.check(L.gear_bab_split(_p(lo), _p(hi), _p(kept), K, self.n, _p(split_idx), _p(lb), _p(lA),
                                            _p(lbias), self.S, _p(clo), _p(chi), _p(ckey), stream), "gear_bab_split")
            else:
                # split, clip the children with their parent's planes, then key the clipped boxes
                # (the reordered loop: split -> clip -> child key, batch_branch_and_bound.py:505-535)
                _lib.check(L.gear_bab_split(_p(lo), _p(hi), _p(kept), K, self.n, _p(split_idx), None, None, None,
                                            self.S, _p(clo), _p(chi), None, stream), "gear_bab_split")
                nonempty = torch.empty(2 * K, dtype=torch.uint8, device=self.device)
                _lib.check(L.gear_clip_domains(_p(clo), _p(chi), _p(thr), _p(lA), _p(lbias), _p(parents), 2 * K,
                                               self.S, self.n, self.clip_iterations, _p(nonempty), stream),
                           "gear_clip_domains")
                _lib.check(L.gear_bab_child_keys(_p(lb), _p(lA), _p(lbias), _p(clo), _p(chi), _p(kept), K, self.S,
                                                 self.n, _p(ckey), stream), "gear_bab_child_keys")
            cuts = self._cuts(lA, lbias, thr, kept[:K].long()) if self.constrained else (None, None)
            cthr = torch.cat([thr[kept[:K].long()]] * 2)
            fields = [clo, chi, ckey, cthr, *cuts]
            if self.clip:
                # children the clipping emptied are done: drop them before they enter the queue
                live = torch.empty(2 * K, dtype=torch.int32, device=self.device)
                nl = torch.zeros(1, dtype=torch.int32, device=self.device)
                ws2 = self._ws_bytes(int(L.gear_bab_workspace_bytes(2 * K)))
                _lib.check(L.gear_bab_compact(_p(nonempty), 2 * K, _p(live), _p(nl), _p(ws2), ws2.numel(), stream),
                           "gear_bab_compact")
                m = int(nl.item())
                self.stats.clipped_empty += 2 * K - m
                out = []
                for f in fields:
                    if f is None:
                        out.append(None)
                        continue
                    g = torch.empty(m, f.shape[1], dtype=torch.float64, device=self.device)
                    if m:
                        _lib.check(L.gear_gather_rows(_p(f.contiguous()), _p(live), m, f.shape[1], _p(g), stream),
                                   "gear_gather_rows")
                    out.append(g)
                fields = out
            q.push(*fields)

    def step(self):
        """One iteration; returns the number of domains bounded."""
        if len(self.queue) == 0:
            return 0
        popped = self.select()
        lo, hi = popped[0], popped[1]
        B = lo.shape[0]
        self.propose_incumbent((lo + hi) / 2)
        lb_ibp = torch.empty(B, self.S, dtype=torch.float64, device=self.device) if self.ibp_enhancement else None
        if self.cut_engine is not None:
            lb, lA, lbias = self.cut_engine.lower(lo, hi, popped[4].reshape(B, self.S, self.n), popped[5],
                                                  lb_ibp=lb_ibp)
        else:
            lb, lA, lbias = self.engine.lower(lo, hi, lb_ibp=lb_ibp)
        st = self.prune_branch(popped, lb, lA, lbias)
        K, inc = torch.cat([st["nk"].to(torch.float64), self._inc_dev]).tolist()   # the iteration's host read
        self.sync_incumbent(inc)
        self.finish(st, int(K))
        return B

    def _cuts(self, lA, lbias, thr, parents):
        """Cut rows of the children (both halves of every kept parent) in standard form
        A x + b <= 0 from the parents' planes lA_j x + lbias_j <= thr_j
        (construct_cut_constraints, input_split/utils.py:113-129); a row with an infinite
        threshold (the objective before any incumbent) is the inert row 0 x - 1 <= 0."""
        A = lA[parents].reshape(parents.numel(), self.S, self.n)
        t = thr[parents]
        b = lbias[parents] - t
        inactive = torch.isposinf(t)
        A = A.masked_fill(inactive.unsqueeze(-1), 0.0)
        b = b.masked_fill(inactive, -1.0)
        A = A.reshape(parents.numel(), -1)
        return torch.cat([A, A]), torch.cat([b, b])

    def _constrained_objective(self, lo, hi, lb, lA, lbias, cutA, cutb):
        """Raise the objective row's bound to lbias_0 + min of lA_0 x over the box intersected
        with the inherited cut rows; +inf (pruned) when the rows exclude the box."""
        from .concretize import constraints_solving
        B = lo.shape[0]
        obj = lA[:, :1, :]
        val, infeasible = constraints_solving(lo, hi, obj, (cutA.reshape(B, self.S, self.n), cutb),
                                              sign=-1.0, max_rows=self.max_constraint_rows,
                                              return_infeasible=True)
        new = val[:, 0, 0] + lbias[:, 0]
        # the addition is rounded: widen it down by u |result| (fp_enclosure.add_bound)
        new = torch.where(torch.isfinite(new), new - torch.abs(new) * (17 * 4 * 2.220446049250313e-16), new)
        new = torch.where(torch.isnan(new), lb[:, 0], new)
        lb[:, 0] = torch.maximum(lb[:, 0], new)
        lb[:, 0] = torch.where(infeasible, torch.full_like(new, math.inf), lb[:, 0])

    def run(self, rel_gap: float = 1e-4, max_iterations: int = 10000, time_limit: float = 60.0):
        t0 = time.perf_counter()
        while len(self.queue) and self.stats.iterations < max_iterations:
            self.step()
            D = self.dual_bound()
            g = self._gap(self.incumbent, D)
            self.stats.history.append(dict(it=self.stats.iterations, P=self.incumbent, D=D, gap=g,
                                           open=len(self.queue)))
            if g <= rel_gap or time.perf_counter() - t0 > time_limit:
                break
        return self.incumbent, self.dual_bound(), self.gap()


def bab_round(babs, bound, ibp_enhancement=True):
    """One branch-and-bound iteration over several instances: select on each, their incumbent
    candidates folded in on the device, one bound(popped, lb_ibp) call for all batches (it returns
    {key: (lb, lA, lbias)}), prune and branch on each, all survivor counts and incumbents in one
    host read, then split and push on each. babs: {key: BaB}. Returns the domains bounded."""
    popped = {k: b.select() for k, b in babs.items() if len(b.queue)}
    if not popped:
        return 0
    for k, p in popped.items():
        babs[k].propose_incumbent((p[0] + p[1]) / 2)                   # on the device
    ibp = {k: babs[k]._buf("lb_ibp", p[0].shape[0] * babs[k].S, torch.float64).view(p[0].shape[0], babs[k].S)
           for k, p in popped.items()} if ibp_enhancement else {}
    outs = bound(popped, ibp)
    sts = {k: babs[k].prune_branch(popped[k], *outs[k]) for k in popped}
    vals = torch.cat([t for k in sts for t in (sts[k]["nk"].to(torch.float64), babs[k]._inc_dev)]).tolist()
    for j, k in enumerate(sts):                                            # one host read above
        babs[k].sync_incumbent(vals[2 * j + 1])
        babs[k].finish(sts[k], int(vals[2 * j]))
    return sum(p[0].shape[0] for p in popped.values())


def relative_gaps(babs):
    """{key: relative gap} of several BaB instances in one host read."""
    keys = list(babs)
    if not keys:
        return {}
    D = torch.cat([torch.minimum(babs[k].queue.min_key_tensor(), babs[k].disc_min) for k in keys]).tolist()
    out = {}
    for k, d in zip(keys, D):
        P = babs[k].incumbent
        if not math.isfinite(P):
            out[k] = math.inf
        elif not math.isfinite(d):
            out[k] = 0.0 if d > 0 else math.inf
        else:
            out[k] = (P - d) / max(1.0, abs(P), abs(d))
    return out


class _Shape:
    """Stands in for a CrownEngine where only the widths are needed (the bounds come from a
    shared MultiEngine)."""
    mode = "fixed"

    def __init__(self, n, S):
        self.n, self.S = n, S


class MultiBaB:
    """Branch and bound on many instances at once (the uneven batch).

    Every iteration pops a batch from each open instance's queue, bounds all of them in one
    persistent CROWN launch per kernel variant (MultiEngine), then prunes, branches and splits
    each instance with the device kernels of BaB. Host reads are batched over the instances:
    one for all incumbent candidates, one for all survivor counts, one for all dual bounds per
    iteration. Each instance's search is the one BaB runs for it alone (same batch order, same
    bounds: the packed launch is bit-identical to a launch per instance)."""

    def __init__(self, graphs, roots, models=None, rhs=None, batch: int = 256, programs=None, engine=None,
                 device="cuda", ibp_enhancement: bool = True, sb_coeff_thresh: float = 1e-3,
                 sb_min_width_ratio: float = 1e-3):
        from .engine import MultiEngine
        self.device = torch.device(device)
        self.engine = engine if engine is not None else MultiEngine(graphs, programs=programs)
        self.ibp_enhancement = ibp_enhancement
        N = len(graphs)
        models = models if models is not None else [None] * N
        rhs = rhs if rhs is not None else [None] * N
        self.babs = [BaB(graphs[i], roots[i][0], roots[i][1], rhs=rhs[i], device=device, batch=batch,
                         engine=_Shape(self.engine.n[i], self.engine.S[i]), model=models[i],
                         ibp_enhancement=ibp_enhancement, sb_coeff_thresh=sb_coeff_thresh,
                         sb_min_width_ratio=sb_min_width_ratio) for i in range(N)]
        self.iterations = 0
        self.bounded = 0

    def step(self, active):
        """One iteration over the instances in `active`; returns the number of domains bounded."""
        dev = self.device

        def bound(popped, ibp):
            boxes, ibps = [], []
            for i, b in enumerate(self.babs):
                if i in popped:
                    boxes.append((popped[i][0], popped[i][1]))
                    ibps.append(ibp.get(i))
                else:
                    e = torch.empty(0, b.n, dtype=torch.float64, device=dev)
                    boxes.append((e, e))
                    ibps.append(None)
            outs = self.engine.lower(boxes, lb_ibp=ibps)
            return {i: outs[i] for i in popped}
        B = bab_round({i: self.babs[i] for i in active}, bound, self.ibp_enhancement)
        self.iterations += 1
        self.bounded += B
        return B

    def gaps(self, idx):
        """Relative gaps of the instances in idx (one host read)."""
        g = relative_gaps({i: self.babs[i] for i in idx})
        return [g[i] for i in idx]

    def run(self, rel_gap: float = 1e-4, time_limit: float = 60.0, max_iterations: int = 10000):
        """Iterate until every instance reaches the gap (or empties its queue), or a limit.
        Returns per instance: incumbent, dual bound, gap, wall time to the gap (None if not
        reached), iterations it took part in."""
        N = len(self.babs)
        t0 = time.perf_counter()
        active = list(range(N))
        reached = [None] * N
        rounds = [0] * N
        last = [math.inf] * N
        while active and self.iterations < max_iterations and time.perf_counter() - t0 < time_limit:
            self.step(active)
            for i in active:
                rounds[i] += 1
            gaps = self.gaps(active)
            now = time.perf_counter() - t0
            nxt = []
            for i, g in zip(active, gaps):
                last[i] = g
                if g <= rel_gap or len(self.babs[i].queue) == 0:
                    reached[i] = now if g <= rel_gap else None
                else:
                    nxt.append(i)
            active = nxt
        return [{"P": b.incumbent, "gap": last[i], "time_to_gap": reached[i], "iterations": rounds[i],
                 "bounded": b.stats.bounded} for i, b in enumerate(self.babs)]


class GraphBaB:
    """Branch and bound to a relative gap on one instance with its queue on the device.

    The open domains live in a gear_queue (slot arrays, the ordered active list, free list and
    counters in device memory); an iteration is gear_queue_pop, the incumbent proposal from the
    popped boxes' midpoints (the model in float64, on the device), and gear_bab_step (CROWN, prune,
    SB branch, split, child keys, sort and merge of the children). Every size is read on the
    device, so `chunk` iterations are captured once into a CUDA graph and replayed; the host reads
    the counters, the dual bound and the incumbent once per replay to test the gap. The search is
    the one BaB runs: same queue order, same kernels."""

    N_COUNTERS = 8
    (C_ACTIVE, C_FREE, C_NEXT_ID, C_BOUNDED, C_POPPED, C_KEPT_TOTAL, C_ITER, C_OVERFLOW) = range(8)

    def __init__(self, graph: Graph, lo: torch.Tensor, hi: torch.Tensor, rhs: Optional[torch.Tensor] = None,
                 device="cuda", batch: int = 2048, model: Optional[torch.nn.Module] = None,
                 capacity: Optional[int] = None, sb_coeff_thresh: float = 1e-3, sb_min_width_ratio: float = 1e-3,
                 ibp_enhancement: bool = True, chunk: int = 8, use_graph: bool = True,
                 engine: Optional[CrownEngine] = None, engine_mode: str = "auto", cta_threads: int = 128):
        """capacity: the queue's first capacity in slots (default 64 x batch); each iteration grows
        the open list by at most `batch`, a replay of `chunk` iterations starts only with that much
        room, and the queue doubles (gear_queue_reserve) when it has less."""
        self.device = torch.device(device)
        self.graph = graph
        self.batch = int(batch)
        self.chunk = max(1, int(chunk))
        self.use_graph = use_graph
        self.model = model
        self.coeff_thresh = sb_coeff_thresh
        self.min_width_ratio = sb_min_width_ratio
        self.ibp_enhancement = ibp_enhancement
        self.engine = engine if engine is not None else CrownEngine(graph, mode=engine_mode, cta_threads=cta_threads)
        if self.engine.mode == "auto":
            gen = torch.Generator(device="cpu").manual_seed(0)
            r0, r1 = lo.reshape(1, -1).cpu().double(), hi.reshape(1, -1).cpu().double()
            c = r0 + (r1 - r0) * torch.rand(batch, r0.shape[1], generator=gen, dtype=torch.float64)
            w = (r1 - r0) * torch.rand(batch, r0.shape[1], generator=gen, dtype=torch.float64) * 0.25
            self.engine.freeze(torch.maximum(r0, c - w).to(self.device), torch.minimum(r1, c + w).to(self.device))
        self.n, self.S = self.engine.n, self.engine.S
        dev = self.device
        root_lo = lo.reshape(-1).to(torch.float64).cpu().contiguous()
        root_hi = hi.reshape(-1).to(torch.float64).cpu().contiguous()
        self.capacity = int(capacity or 64 * self.batch)
        L = _lib.lib()
        h = ctypes.c_void_p()
        _lib.check(L.gear_queue_create(self.n, self.S, self.capacity, self.batch, root_lo.data_ptr(),
                                       root_hi.data_ptr(), ctypes.byref(h)), "gear_queue_create")
        self.q = h
        self.plo = torch.empty(self.batch, self.n, dtype=torch.float64, device=dev)
        self.phi = torch.empty_like(self.plo)
        self.inc = torch.full((1,), math.inf, dtype=torch.float64, device=dev)
        self.x_best = ((root_lo + root_hi) / 2).to(dev)
        rhs = torch.zeros(self.S - 1, dtype=torch.float64) if rhs is None else rhs.to(torch.float64).reshape(-1)
        self.rhs = torch.cat([rhs.to(dev), torch.zeros(1, dtype=torch.float64, device=dev)])   # never empty
        self.ws = torch.empty(int(L.gear_bab_step_workspace_bytes(self.engine.handle, self.batch)), dtype=torch.uint8,
                              device=dev)
        self.counters = torch.zeros(self.N_COUNTERS, dtype=torch.int64, device=dev)
        self.dual = torch.full((1,), -math.inf, dtype=torch.float64, device=dev)
        _lib.check(L.gear_queue_counters(self.q, self.counters.data_ptr(), self.dual.data_ptr(),
                                         torch.cuda.current_stream(dev).cuda_stream), "gear_queue_counters")
        self.graph_obj = None
        self.incumbent = math.inf
        self.replays = 0
        self.regrown = 0
        self.status = {}

    def __del__(self):
        q = getattr(self, "q", None)
        if q is not None and q.value:
            try:
                self.graph_obj = None
                _lib.lib().gear_queue_destroy(q)
            except Exception:
                pass
            self.q = None

    def _propose(self):
        """Best feasible model value among the popped boxes' midpoints into the device incumbent."""
        if self.model is None:
            return
        with torch.no_grad():
            x = (self.plo + self.phi) / 2
            y = self.model(x)
            if y.shape[1] > 1:
                feas = (y[:, 1:] <= self.rhs[:self.S - 1]).all(1)
            else:
                feas = torch.ones(y.shape[0], dtype=torch.bool, device=self.device)
            obj = torch.where(feas, y[:, 0], torch.full_like(y[:, 0], math.inf))
            best = obj.min(0)
            val = best.values.reshape(1)
            pt = x.index_select(0, best.indices.reshape(1)).reshape(-1)
            self.x_best.copy_(torch.where(val < self.inc, pt, self.x_best))
            self.inc.copy_(torch.minimum(self.inc, val))

    def _iteration(self):
        L = _lib.lib()
        st = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(L.gear_queue_pop(self.q, self.plo.data_ptr(), self.phi.data_ptr(), st), "gear_queue_pop")
        self._propose()
        _lib.check(L.gear_bab_step(self.q, self.engine.handle, self.plo.data_ptr(), self.phi.data_ptr(),
                                   self.inc.data_ptr(), self.rhs.data_ptr(), self.coeff_thresh, self.min_width_ratio,
                                   1 if self.ibp_enhancement else 0, self.ws.data_ptr(), self.ws.numel(), st),
                   "gear_bab_step")

    def _chunk(self):
        for _ in range(self.chunk):
            self._iteration()
        L = _lib.lib()
        _lib.check(L.gear_queue_counters(self.q, self.counters.data_ptr(), self.dual.data_ptr(),
                                         torch.cuda.current_stream(self.device).cuda_stream), "gear_queue_counters")

    def _read(self):
        vals = torch.cat([self.counters.to(torch.float64), self.dual, self.inc]).tolist()
        c = [int(v) for v in vals[:self.N_COUNTERS]]
        self.status = dict(open=c[self.C_ACTIVE], bounded=c[self.C_BOUNDED], iterations=c[self.C_ITER],
                           kept=c[self.C_KEPT_TOTAL], overflow=c[self.C_OVERFLOW], dual=vals[-2], incumbent=vals[-1])
        self.incumbent = vals[-1]
        return self.status

    def run(self, rel_gap: float = 1e-4, time_limit: float = 60.0, max_iterations: int = 100000):
        """Iterate until the relative gap, an empty queue or a limit; returns (P, D, gap)."""
        t0 = time.perf_counter()
        st = self._read()
        while True:
            if st["open"] == 0 or st["iterations"] >= max_iterations or time.perf_counter() - t0 > time_limit:
                break
            if st["open"] + self.chunk * self.batch > self.capacity:
                # grow the queue (its device pointers change: capture the iterations again)
                L = _lib.lib()
                new = max(2 * self.capacity, st["open"] + 2 * self.chunk * self.batch)
                _lib.check(L.gear_queue_reserve(self.q, new, torch.cuda.current_stream(self.device).cuda_stream),
                           "gear_queue_reserve")
                self.capacity = int(L.gear_queue_capacity(self.q))
                self.graph_obj = None
                self.regrown += 1
            if self.use_graph:
                if self.graph_obj is None:
                    self._chunk()                       # eager first chunk: loads, workspaces, warm caches
                    torch.cuda.synchronize(self.device)
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g):
                        self._chunk()
                    self.graph_obj = g
                    st = self._read()                   # the captured chunk did not run yet
                    gap = self._gap(st["incumbent"], st["dual"])
                    if gap <= rel_gap:
                        break
                    continue
                self.graph_obj.replay()
            else:
                self._chunk()
            self.replays += 1
            st = self._read()
            if st["overflow"]:
                raise RuntimeError("gear_queue overflow: children were not pushed")
            if self._gap(st["incumbent"], st["dual"]) <= rel_gap:
                break
        return st["incumbent"], st["dual"], self._gap(st["incumbent"], st["dual"])

    @staticmethod
    def _gap(P, D):
        return BaB._gap(P, D)


class MultiGraphBaB:
    """Branch and bound on many instances at once (the uneven batch), every instance's queue on
    the device (gear_queue) and its round captured once into CUDA graphs: one for its pop and
    incumbent proposal (its model at the popped boxes' midpoints), one for its
    gear_bab_step_bounded and a copy of its counters, dual bound and incumbent into a status row.
    A round replays every running instance's first graph, makes one prepared many-instance CROWN
    launch per kernel group for all the batches (MultiEngine.prepare / launch_prepared, re-planned
    only when the running set changes), replays the second graphs and reads all status rows in one
    copy. An instance retires when it reaches the gap or empties its queue; a queue about to fill
    grows (gear_queue_reserve, up to max_queue_bytes) and that instance's graphs are captured
    again. Each instance's search is the one GraphBaB runs for it alone (same kernels, same order;
    tested)."""

    def __init__(self, graphs, roots, models=None, rhs=None, batch: int = 256, engine=None, programs=None,
                 device="cuda", ibp_enhancement: bool = True, sb_coeff_thresh: float = 1e-3,
                 sb_min_width_ratio: float = 1e-3, queue_slots: Optional[int] = None,
                 max_queue_bytes: int = 1 << 30):
        """roots: [(lo (1, n_i), hi (1, n_i))]; queue_slots: the first capacity of every queue
        (default 16 x batch); a queue doubles when fewer than 2 x batch slots stay free, while its
        memory stays within max_queue_bytes."""
        from .engine import MultiEngine
        self.device = dev = torch.device(device)
        self.engine = engine if engine is not None else MultiEngine(graphs, programs=programs)
        N = len(graphs)
        self.N, self.batch = N, int(batch)
        self.coeff_thresh, self.min_width_ratio = sb_coeff_thresh, sb_min_width_ratio
        self.models = list(models) if models is not None else [None] * N
        self.n, self.S = list(self.engine.n), list(self.engine.S)
        self.max_queue_bytes = max_queue_bytes
        L = _lib.lib()
        st = torch.cuda.current_stream(dev).cuda_stream
        self.status = torch.zeros(N, GraphBaB.N_COUNTERS + 2, dtype=torch.float64, device=dev)
        self.inc, self.counters, self.dual = [], [], []
        self.boxes, self.x_best, self.rhs, self.queues = [], [], [], []
        first = int(queue_slots or 16 * self.batch)
        for i in range(N):
            n, S = self.n[i], self.S[i]
            lo = roots[i][0].reshape(-1).to(torch.float64).cpu().contiguous()
            hi = roots[i][1].reshape(-1).to(torch.float64).cpu().contiguous()
            h = ctypes.c_void_p()
            _lib.check(L.gear_queue_create(n, S, max(first, 2 * self.batch + 1), self.batch, lo.data_ptr(),
                                           hi.data_ptr(), ctypes.byref(h)), "gear_queue_create")
            self.queues.append(h)
            self.boxes.append((torch.empty(self.batch, n, dtype=torch.float64, device=dev),
                               torch.empty(self.batch, n, dtype=torch.float64, device=dev)))
            self.x_best.append(((lo + hi) / 2).to(dev))
            r = rhs[i] if rhs is not None and rhs[i] is not None else torch.zeros(S - 1, dtype=torch.float64)
            self.rhs.append(torch.cat([r.to(torch.float64).reshape(-1).to(dev),
                                       torch.zeros(1, dtype=torch.float64, device=dev)]))
            self.inc.append(torch.full((1,), math.inf, dtype=torch.float64, device=dev))
            self.counters.append(torch.zeros(GraphBaB.N_COUNTERS, dtype=torch.int64, device=dev))
            self.dual.append(torch.full((1,), -math.inf, dtype=torch.float64, device=dev))
            _lib.check(L.gear_queue_counters(h, self.counters[i].data_ptr(), self.dual[i].data_ptr(), st),
                       "gear_queue_counters")
        self.outs = self.engine.outputs([self.batch] * N, dev)
        self.ibp = ([torch.empty(self.batch, self.S[i], dtype=torch.float64, device=dev) for i in range(N)]
                    if ibp_enhancement else None)
        self.graphs = [None] * N
        for i in range(N):
            self._capture(i)
        self._planned = None
        self.rounds = self.captures_regrown = self.prepares = 0

    def __del__(self):
        try:
            self.graphs = []
            self.engine.release_prepared()
            L = _lib.lib()
            for h in getattr(self, "queues", []):
                if h is not None and h.value:
                    L.gear_queue_destroy(h)
            self.queues = []
        except Exception:
            pass

    def _pre(self, i):
        L = _lib.lib()
        dev = self.device
        plo, phi = self.boxes[i]
        _lib.check(L.gear_queue_pop(self.queues[i], plo.data_ptr(), phi.data_ptr(),
                                    torch.cuda.current_stream(dev).cuda_stream), "gear_queue_pop")
        m = self.models[i]
        if m is None:
            return
        S = self.S[i]
        with torch.no_grad():
            x = (plo + phi) / 2
            y = m(x)
            feas = (y[:, 1:] <= self.rhs[i][:S - 1]).all(1) if y.shape[1] > 1 else \
                torch.ones(y.shape[0], dtype=torch.bool, device=dev)
            obj = torch.where(feas, y[:, 0], torch.full_like(y[:, 0], math.inf))
            best = obj.min(0)
            val = best.values.reshape(1)
            pt = x.index_select(0, best.indices.reshape(1)).reshape(-1)
            inc = self.inc[i]
            self.x_best[i].copy_(torch.where(val < inc, pt, self.x_best[i]))
            inc.copy_(torch.minimum(inc, val))

    def _post(self, i):
        L = _lib.lib()
        st = torch.cuda.current_stream(self.device).cuda_stream
        plo, phi = self.boxes[i]
        lb, lA, lbias = self.outs[i]
        _lib.check(L.gear_bab_step_bounded(self.queues[i], plo.data_ptr(), phi.data_ptr(), lb.data_ptr(), lA.data_ptr(),
                                           lbias.data_ptr(), self.inc[i].data_ptr(), self.rhs[i].data_ptr(),
                                           self.coeff_thresh, self.min_width_ratio, st), "gear_bab_step_bounded")
        _lib.check(L.gear_queue_counters(self.queues[i], self.counters[i].data_ptr(), self.dual[i].data_ptr(), st),
                   "gear_queue_counters")
        self.status[i].copy_(torch.cat([self.counters[i].to(torch.float64), self.dual[i], self.inc[i]]))

    def _capture(self, i):
        self.graphs[i] = None
        gs = {}
        for name, fn in (("pre", self._pre), ("post", self._post)):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                fn(i)
            gs[name] = g
        self.graphs[i] = gs

    def _prepare(self, run):
        e = torch.empty(0, dtype=torch.float64, device=self.device)
        rs = set(run)
        boxes = [self.boxes[i] if i in rs else (e.view(0, self.n[i]), e.view(0, self.n[i])) for i in range(self.N)]
        ibp = [self.ibp[i] if i in rs else None for i in range(self.N)] if self.ibp is not None else None
        self.engine.prepare(boxes, self.outs, ibp)
        self._planned = tuple(run)
        self.prepares += 1

    def run(self, rel_gap: float = 1e-4, time_limit: float = 60.0, max_rounds: int = 100000):
        """Until every instance reaches the gap or empties its queue, or a limit. Returns per
        instance: incumbent, dual bound, gap, wall time to the gap (None if not reached), status,
        domains bounded (counted up to its retirement), rounds."""
        t0 = time.perf_counter()
        N = self.N
        res = [dict(P=math.inf, D=-math.inf, gap=math.inf, time_to_gap=None, status="running", bounded=0, rounds=0)
               for _ in range(N)]
        running = list(range(N))
        L = _lib.lib()
        C = GraphBaB
        while running and self.rounds < max_rounds and time.perf_counter() - t0 < time_limit:
            if self._planned != tuple(running):
                self._prepare(running)
            for i in running:
                self.graphs[i]["pre"].replay()
            self.engine.launch_prepared()
            for i in running:
                self.graphs[i]["post"].replay()
            idx = torch.tensor(running, dtype=torch.int64, device=self.device)
            rows = self.status.index_select(0, idx).cpu().tolist()
            self.rounds += 1
            now = time.perf_counter() - t0
            nxt = []
            for i, row in zip(running, rows):
                D, P = row[C.N_COUNTERS], row[C.N_COUNTERS + 1]
                g = BaB._gap(P, D)
                r = res[i]
                r.update(P=P, D=D, gap=g, bounded=int(row[C.C_BOUNDED]), rounds=r["rounds"] + 1)
                open_ = int(row[C.C_ACTIVE])
                if g <= rel_gap:
                    r.update(time_to_gap=now, status="closed")
                    continue
                if open_ == 0:
                    r.update(status="emptied")
                    continue
                cap = int(L.gear_queue_capacity(self.queues[i]))
                if open_ + 2 * self.batch > cap or int(row[C.C_OVERFLOW]):
                    slot = 8 * (2 * self.n[i] + self.S[i] + 2) + 12
                    new = min(2 * cap, self.max_queue_bytes // slot)
                    if int(row[C.C_OVERFLOW]) or new < open_ + 2 * self.batch:
                        r.update(status="capacity")
                        continue
                    _lib.check(L.gear_queue_reserve(self.queues[i], new,
                                                    torch.cuda.current_stream(self.device).cuda_stream),
                               "gear_queue_reserve")
                    self._capture(i)
                    self.captures_regrown += 1
                nxt.append(i)
            running = nxt
        return res
