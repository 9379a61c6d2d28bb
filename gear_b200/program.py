"""Host compiler: a traced ``Graph`` -> a flat device program for the CROWN megakernel.

Two things are decided here, once per graph, on the host:

1. **The schedule** -- which nodes get intermediate bounds, by IBP or by a CROWN pass, in
   which order, and which transient IBP recomputations ``compare_with_IBP`` needs. It is a
   symbolic replay of the reference's recursion (``auto_LiRPA/bound_general.py:1032-1222``
   ``check_prior_bounds`` / ``compute_intermediate_bounds``, ``interval_bound.py:310-406``),
   which depends only on the graph, never on box values.

2. **Static A sparsity per pass** -- the backward BFS (``backward_bound.py:880-1206``) is
   replayed symbolically and, for every node a pass visits, the set of (spec row, column)
   entries of its A matrix that can be nonzero is computed. Rows of an identity
   specification stay one-hot through elementwise chains, slices and gathers, so the
   intermediate passes (C = I over the node width) cost O(width) instead of
   O(width^2). Zero entries contribute exactly zero in the reference's dense arithmetic,
   so skipping them changes no bound. Each pass op becomes a list of pull "moves"
   (target entry <- source entries) that the kernel executes per box.

   One further exact rewrite: when the only contribution to the input node in a
   non-final pass comes from a Linear/MatMul on the input and every row reaches it with at
   most one nonzero, the input's A row is ``a * W[c, :]`` and its box concretisation
   ``a W[c] x0 -/+ |a| |W[c]| eps`` is read from per-box vectors ``W x0`` and ``|W| eps``
   (``fold``) instead of materialising ``w_out x n`` coefficients.

The output is a handful of int32 / float64 arrays (layout constants below mirror
``csrc/gear_program.h``).
"""
from __future__ import annotations

import os
from collections import deque
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import tables
from .graph import Graph, MAP_KINDS

# ---- node kinds (csrc/gear_program.h: enum NodeKind)
NK = {"input": 0, "linear": 1, "matmul": 2, "mul": 3, "mulc": 4, "add": 5, "sub": 6, "addc": 7,
      "subc": 8, "rsubc": 9, "neg": 10, "sqr": 11, "exp": 12, "log": 13, "sin": 14, "cos": 15,
      "pow": 16, "reducesum": 17, "map": 18, "concat": 19}
NODE_REC = 17
# node record fields (N_WT_OFF: the weights transposed, (in, out), for the forward products)
N_KIND, N_W, N_NIN, N_IN0, N_IN1, N_CUR, N_PLANE, N_CVEC, N_MAP0, N_MAP1, N_W_OFF, N_B_OFF, \
    N_WIN, N_INS, N_FOLD, N_INEXACT, N_WT_OFF = range(17)

# ---- steps
MODES = {"cta": 0, "simt": 1}          # ExecMode in gear_program.h
ST = {"ibp": 0, "mag": 1, "relax": 2, "pass": 3, "compare": 4, "fold": 5, "final": 6, "ibpout": 7}
STEP_REC = 4

PASS_REC = 24
(P_T, P_S, P_SIDES, P_INIT, P_OP0, P_NOP, P_TBUF, P_XNNZ, P_XBUF, P_XRP, P_XCOLS, P_NFOLD,
 P_SMEM, P_TRP, P_TCOLS, P_FINAL, P_NVISIT, P_MAXROW, P_ONEHOT, P_XMAXROW, P_XDENSE, P_TMAXROW, P_R22, P_R23) = range(24)

OP_REC = 32
(O_KIND, O_V, O_SLOT, O_FIRST, O_VBUF, O_VNNZ, O_VRP, O_VCOLS, O_U, O_UBUF, O_UNNZ, O_URP,
 O_UCOLS, O_UMERGE, O_NTGT, O_TGT, O_SPTR, O_SRC, O_DENSE, O_FOLD, O_WOUT, O_VMAXROW, O_UMAXROW, O_VROWS,
 O_TPTR, O_UK, O_TMAXROW, O_SHORT, O_NSHORT, O_LONG, O_NLONG, O_SINGLE) = range(32)
ROW_THREAD_MAX = 16  # rows with at most this much work run on one thread, longer rows on a warp
# bits of the op record's O_SINGLE field (OpFlag in gear_program.h)
OF_SINGLE, OF_SRC_ID, OF_TGT_ID, OF_TPTR_ID, OF_VRP_ID, OF_SPLIT, OF_FUSED, OF_FUSED_T = 1, 2, 4, 8, 16, 32, 64, 128
ROOT_IN_LA = -2     # buffer marker: the input's A of a final pass accumulates in the lA output

PLANES_PER_ELEM = {"mul": 6, "sqr": 4, "exp": 4, "log": 4, "sin": 4, "cos": 4, "pow": 4}

# McCormick tie rules (header field H_TIES): "reference" is the reference's float comparison of
# the two candidate planes' box minima (bivariate.py:250); "exact" counts a relative difference
# below 1e-12 as a tie and picks plane 1 (deterministic across summation orders)
TIE_RULES = {"reference": 0, "exact": 1}


class ProgramError(ValueError):
    pass


@dataclass
class PassInfo:
    t: int
    S: int
    sides: int
    final: bool
    init: int                 # 0 identity, 1 dense C
    order: List[int] = field(default_factory=list)       # BFS visit order (excl. root)
    # node -> (row ids, columns) of the A entries, ordered by row then column (unique)
    patterns: Dict[int, Tuple[np.ndarray, np.ndarray]] = field(default_factory=dict)


class Pools:
    def __init__(self):
        self.ints: List[np.ndarray] = []
        self.n_int = 0
        self.dbl: List[np.ndarray] = []
        self.n_dbl = 0

    def add_int(self, a) -> int:
        a = np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1))
        off = self.n_int
        self.ints.append(a)
        self.n_int += a.size
        return off

    def add_dbl(self, a) -> int:
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
        # 32-byte alignment of every vector (coalesced row reads of W)
        pad = (-self.n_dbl) % 4
        if pad:
            self.dbl.append(np.zeros(pad))
            self.n_dbl += pad
        off = self.n_dbl
        self.dbl.append(a)
        self.n_dbl += a.size
        return off

    def int_array(self):
        return np.concatenate(self.ints) if self.ints else np.zeros(0, np.int32)

    def dbl_array(self):
        return np.concatenate(self.dbl) if self.dbl else np.zeros(0, np.float64)


class Program:
    """Compiled device program for one graph and one final specification shape."""

    def __init__(self, graph: Graph, spec_rows: Optional[int] = None, dense_c: bool = False,
                 return_a: bool = True, smem_limit: int = 232448, mode: str = "cta",
                 cta_threads: int = 128, tie_rule: str = "reference", fold_tc: bool = False,
                 cuts: bool = False):
        """mode: "cta" runs one box per CTA with the pass working set in shared memory, and the
        final pass accumulates the input's A directly in the lA output; "simt" runs one box per
        thread with every per-box array box-interleaved in global scratch, and writes lA from the
        pass buffers at the end. smem_limit: bytes of shared memory one CTA may use (the sm_100
        opt-in maximum); a box-per-CTA pass working set beyond it lives in global scratch.
        tie_rule: how the coefficient-aware McCormick pick decides between two candidate planes
        whose box minima are equal in exact arithmetic (x entirely negative and y entirely
        positive, or the reverse): "reference" compares the two rounded minima as the reference
        does (bivariate.py:250; the outcome then follows the last bits of the intermediate
        bounds), "exact" picks plane 1, the exact-arithmetic outcome.
        fold_tc: compute the fold vectors of the dense nodes on the input (W x0, |W| eps) for the
        whole batch on the tensor cores before the CROWN kernel (int8 digit slicing with a rigorous
        error term; box-per-CTA programs with such nodes only, otherwise ignored).
        cuts: compile for concretisation over the box intersected with cut rows
        (gear_crown_lower_cuts): no pass folds its input rows into per-box vectors (the
        constrained sweep needs every input A row), and with smem_limit=0 the program runs in
        the plain form's launch sequence."""
        if tie_rule not in TIE_RULES:
            raise ProgramError(f"unknown tie rule {tie_rule!r}")
        self.tie_rule = tie_rule
        self.cuts = bool(cuts)
        self.fold_tc = bool(fold_tc) and mode == "cta" and not self.cuts
        self.split_op = -1          # node whose final-pass product runs on the tensor cores (_mark_split)
        if mode not in MODES:
            raise ProgramError(f"unknown execution mode {mode!r}")
        if cta_threads not in (64, 128, 256):
            raise ProgramError("threads per CTA must be 64, 128 or 256")
        self.cta_threads = int(cta_threads)
        self.mode = mode
        self.x_in_la = mode == "cta"
        self.g = graph
        self.n = graph[0].width
        t = graph.output
        self.t = t
        self.S = graph[t].width if spec_rows is None else int(spec_rows)
        self.dense_c = bool(dense_c)
        self.return_a = return_a
        self.smem_limit = smem_limit
        self.pools = Pools()
        self.steps: List[Tuple[int, int, int, int]] = []
        self.passes: List[PassInfo] = []
        self.pass_recs: List[np.ndarray] = []
        self.op_recs: List[np.ndarray] = []
        self.log: List[tuple] = []
        self._layout_nodes()
        self._schedule()
        self._emit_nodes()
        self._finish()

    # ================================================================= node layout
    def _layout_nodes(self):
        g = self.g
        self.cur_off = {}
        off = 0
        for nd in g.nodes:
            self.cur_off[nd.id] = off
            off += nd.width
        self.arena_w = off            # doubles per box per (lo | hi | mag) arena
        self.plane_off = {}
        off = 0
        for nd in g.nodes:
            if nd.kind in PLANES_PER_ELEM:
                self.plane_off[nd.id] = off
                off += nd.width * PLANES_PER_ELEM[nd.kind]
        self.plane_w = off
        # linear/matmul directly on the input: per-box fold vectors W x0, |W| eps, |W| max|x|
        self.fold_off = {}
        off = 0
        for nd in g.nodes:
            if nd.kind in ("linear", "matmul") and nd.inputs[0] == 0:
                self.fold_off[nd.id] = off
                off += 3 * nd.width
        self.fold_w = off
        self.maxw = max(nd.width for nd in g.nodes)

    # ================================================================= schedule
    def _ancestors(self, t):
        seen, stack = set(), [t]
        while stack:
            v = stack.pop()
            if v in seen:
                continue
            seen.add(v)
            stack += self.g[v].inputs
        return seen

    def _schedule(self):
        g = self.g
        self.anc = self._ancestors(self.t)
        self.stored = {0}
        self.prior_checked = set()
        # fold vectors first (they only depend on the input box)
        for v in sorted(self.fold_off):
            self.steps.append((ST["fold"], v, 0, 0))
        # plain IBP of every node: magnitudes of nodes without stored bounds
        self.steps.append((ST["mag"], 0, 0, 0))
        for nd in g.nodes[1:]:
            self.steps.append((ST["ibp"], nd.id, 1, 0))      # b = 1: also write the magnitude
        # the specification rows over the plain IBP interval of the output (the IBP bound of the
        # bounding glue's IBP pass; written only when the caller asks for it)
        self.steps.append((ST["ibpout"], self.t, 0, 0))
        self.relaxed = set()
        self._check_prior(self.t, final=True)
        # interval of the final node for the undefined-row fallback
        self._transient_ibp(self.t, set())
        self.steps.append((ST["ibp"], self.t, 0, 0))
        self._ensure_relax_for_pass(self.t)
        pid = self._add_pass(self.t, self.S, sides=1, final=True, init=1 if self.dense_c else 0)
        self.steps.append((ST["final"], pid, 0, 0))
        self.log.append(("final", self.t))

    def _check_prior(self, v, final=False):
        g = self.g
        n = g[v]
        if v in self.prior_checked or v not in self.anc or n.kind == "input":
            return
        if final and n.kind == "concat" and not self.dense_c:
            # identity C: every concatenated input is used (bound_general.py:1036-1052)
            for p in n.inputs:
                self._check_prior(p)
        else:
            for p in n.inputs:
                self._check_prior(p)
        for i, p in enumerate(n.inputs):
            if i in n.requires_input_bounds or g[p].has_constraint:
                self._compute_intermediate(p)
        self.prior_checked.add(v)

    def _store_ibp(self, v):
        g = self.g
        for p in g[v].inputs:
            if p not in self.stored:
                self._store_ibp(p)
        self.steps.append((ST["ibp"], v, 1, 0))
        self.stored.add(v)
        self.log.append(("ibp", v))

    def _transient_ibp(self, v, done):
        """IBP of v's non-stored ancestors from stored bounds (not stored)."""
        g = self.g
        for p in g[v].inputs:
            if p not in self.stored and p not in done:
                self._transient_ibp(p, done)
                self.steps.append((ST["ibp"], p, 0, 0))
                done.add(p)

    def _compute_intermediate(self, v):
        g = self.g
        if v in self.stored:
            return
        n = g[v]
        if n.kind == "reshape" and n.inputs[0] in self.stored:
            self.steps.append((ST["ibp"], v, 1, 0))
            self.stored.add(v)
            self.log.append(("ibp", v))
            return
        chain, cur, ok = [], v, True
        while cur not in self.stored:
            if not g[cur].ibp_intermediate:
                ok = False
                break
            chain.append(cur)
            cur = g[cur].inputs[0]
        if ok:
            for c in reversed(chain):
                self._store_ibp(c)
            return
        if n.kind == "linear" and n.inputs[0] == 0:
            self._store_ibp(v)
            return
        self._ensure_relax_for_pass(v)
        pid = self._add_pass(v, n.width, sides=2, final=False, init=0)
        self.steps.append((ST["pass"], pid, 0, 0))
        self._transient_ibp(v, set())
        self.steps.append((ST["compare"], v, pid, 1))      # c = 1: also write the magnitude
        self.stored.add(v)
        self.log.append(("crown", v))

    def _ensure_relax_for_pass(self, t):
        """Relaxation planes of every relaxing node the pass visits (their inputs are stored)."""
        for v in sorted(self._ancestors(t)):
            nd = self.g[v]
            if nd.kind in PLANES_PER_ELEM and v not in self.relaxed:
                for p in nd.inputs:
                    if p not in self.stored:
                        raise ProgramError(f"relaxation of node {v} before its input {p} has bounds")
                self.steps.append((ST["relax"], v, 0, 0))
                self.relaxed.add(v)

    # ================================================================= passes
    def _bfs(self, t):
        g = self.g
        deg, added, q = {}, {t}, deque([t])
        while q:
            l = q.popleft()
            for p in g[l].inputs:
                deg[p] = deg.get(p, 0) + 1
                if p not in added:
                    q.append(p)
                    added.add(p)
        order, queue = [], deque([t])
        while queue:
            l = queue.popleft()
            if l == 0:
                continue
            for p in g[l].inputs:
                deg[p] -= 1
                if deg[p] == 0:
                    queue.append(p)
            order.append(l)
        return order

    @staticmethod
    def _pairs(rows, cols, W):
        """The (row, column) pairs ordered by row then column, duplicates removed (columns < W)."""
        key = np.unique(rows * W + cols)
        return key // W, key % W

    def _contrib(self, n, slot, pat):
        """Entries of input `slot` reached from the entries (rows, cols) of node n."""
        g = self.g
        k, a = n.kind, n.attrs
        p = n.inputs[slot]
        w_in = g[p].width
        rows, cols = pat
        W = w_in + 1
        if k in ("linear", "matmul"):
            r = np.unique(rows)
            return np.repeat(r, w_in), np.tile(np.arange(w_in, dtype=np.int64), len(r))
        if k in ("neg", "sqr", "exp", "log", "sin", "cos", "pow"):
            return rows, cols
        if k in ("mulc", "addc", "subc", "rsubc"):
            m = a["map0"]
        elif k in ("mul", "add", "sub"):
            m = a["map0"] if slot == 0 else a["map1"]
        elif k in MAP_KINDS:
            m = a["map"]
        elif k == "reducesum":
            # every input element i with rmap[i] = o, for each entry (row, o)
            rmap = np.asarray(a["rmap"], np.int64)
            order = np.argsort(rmap, kind="stable")
            first = np.searchsorted(rmap[order], cols, side="left")
            cnt = np.searchsorted(rmap[order], cols, side="right") - first
            base = np.repeat(first - np.concatenate([[0], np.cumsum(cnt)[:-1]]), cnt)
            ii = order[base + np.arange(int(cnt.sum()), dtype=np.int64)]
            return self._pairs(np.repeat(rows, cnt), ii, W)
        elif k == "concat":
            off = sum(g[q].width for q in n.inputs[:slot])
            e = np.asarray(a["cmap"], np.int64)[cols] - off
            keep = (e >= 0) & (e < w_in)
            return self._pairs(rows[keep], e[keep], W)
        else:
            raise ProgramError(k)
        return self._pairs(rows, np.asarray(m, np.int64)[cols], W)

    def _add_pass(self, t, S, sides, final, init):
        g = self.g
        order = self._bfs(t)
        pi = PassInfo(t=t, S=S, sides=sides, final=final, init=init, order=order)
        wt = g[t].width
        if init == 0:
            if S != wt:
                raise ProgramError("an identity specification needs one row per output element")
            ar = np.arange(S, dtype=np.int64)
            pi.patterns[t] = (ar, ar.copy())
        else:
            pi.patterns[t] = (np.repeat(np.arange(S, dtype=np.int64), wt), np.tile(np.arange(wt, dtype=np.int64), S))
        # symbolic propagation
        for v in order:
            n = g[v]
            pv = pi.patterns.get(v)
            if pv is None:
                continue
            for slot, p in enumerate(n.inputs):
                c = self._contrib(n, slot, pv)
                if p not in pi.patterns:
                    pi.patterns[p] = c
                else:
                    q = pi.patterns[p]
                    pi.patterns[p] = self._pairs(np.concatenate([q[0], c[0]]), np.concatenate([q[1], c[1]]),
                                                 g[p].width + 1)
        self.passes.append(pi)
        return len(self.passes) - 1

    # ================================================================= emission
    def _emit_nodes(self):
        g = self.g
        P = self.pools
        recs = np.full((len(g), NODE_REC), -1, dtype=np.int32)
        for nd in g.nodes:
            r = recs[nd.id]
            k = nd.kind if nd.kind not in MAP_KINDS else "map"
            r[N_KIND] = NK[k]
            r[N_W] = nd.width
            r[N_NIN] = len(nd.inputs)
            r[N_IN0] = nd.inputs[0] if nd.inputs else -1
            r[N_IN1] = nd.inputs[1] if len(nd.inputs) > 1 else -1
            r[N_CUR] = self.cur_off[nd.id]
            r[N_PLANE] = self.plane_off.get(nd.id, -1)
            r[N_FOLD] = self.fold_off.get(nd.id, -1)
            a = nd.attrs
            if k in ("mulc", "addc", "subc", "rsubc"):
                r[N_CVEC] = P.add_dbl(a["c"])
                r[N_MAP0] = P.add_int(a["map0"])
                if k == "mulc":
                    c = a["c"]
                    exact = (c == 0) | (np.abs(np.frexp(c)[0]) == 0.5)
                    r[N_INEXACT] = P.add_int((~exact).astype(np.int32))
            elif k in ("mul", "add", "sub"):
                r[N_MAP0] = P.add_int(a["map0"])
                r[N_MAP1] = P.add_int(a["map1"])
            elif k == "map":
                r[N_MAP0] = P.add_int(a["map"])
            elif k == "reducesum":
                r[N_MAP0] = P.add_int(a["rmap"])
                r[N_WIN] = g[nd.inputs[0]].width
                # inverse map for the interval sums: ptr (w_out + 1) then input ids
                order = np.argsort(a["rmap"], kind="stable")
                cnt = np.bincount(a["rmap"], minlength=nd.width)
                ptr = np.concatenate([[0], np.cumsum(cnt)])
                r[N_MAP1] = P.add_int(np.concatenate([ptr, order]))
            elif k == "concat":
                r[N_MAP0] = P.add_int(a["cmap"])
                r[N_INS] = P.add_int(nd.inputs)
                r[N_WIN] = sum(g[q].width for q in nd.inputs)
            elif k == "pow":
                # {exponent, class (0 odd, 1 even integer, 2 non-integer), table length}; an odd
                # exponent's tangent tables (d_lower then d_upper) at N_MAP0, a float64-pool offset
                pexp = float(a["exponent"])
                if not (pexp > 0) or not np.isfinite(pexp):
                    raise ProgramError(f"pow with exponent {pexp} is not supported")
                if pexp == int(pexp):
                    cls = 0 if int(pexp) % 2 == 1 else 1
                else:
                    cls = 2
                tlen = 0
                if cls == 0:
                    d_lo, d_up = tables.pow_tables_cached(int(pexp))
                    tlen = d_lo.size
                    r[N_MAP0] = P.add_dbl(np.concatenate([d_lo, d_up]))
                r[N_CVEC] = P.add_dbl(np.array([pexp, float(cls), float(tlen)]))
            elif k in ("linear", "matmul"):
                W = a["W"] if k == "linear" else a["W"].T      # (out, in)
                r[N_W_OFF] = P.add_dbl(np.ascontiguousarray(W))
                r[N_WT_OFF] = P.add_dbl(np.ascontiguousarray(W.T))
                r[N_WIN] = W.shape[1]
                if k == "linear" and a.get("b") is not None:
                    r[N_B_OFF] = P.add_dbl(a["b"])
        self.node_recs = recs
        # sin/cos tables
        tb = tables.build_cached()
        self.sin_off = P.add_dbl(np.concatenate([tb[k] for k in tables.SIN_TABLE_ORDER]))
        self.sin_lens = [len(tb[k]) for k in tables.SIN_TABLE_ORDER]

    def _finish(self):
        # the pass working set doubles as the staging area of the box (centre, radius, magnitude)
        # for the fold products, which run before any pass
        self.max_smem = 3 * self.n + 32 if self.fold_off else 0
        # algorithmic work per box of the executed schedule: A entries read and written by the
        # backward passes (both sides), concretisation reads, and GEMM-shaped flops at dense
        # nodes (2 per multiply-add of A W, plus the fold products W x0, |W| eps, |W| |x|)
        self.work = {"a_read": 0, "a_written": 0, "gemm_flops": 0, "node_visits": 0, "passes": len(self.passes)}
        for v in self.fold_off:
            self.work["gemm_flops"] += 3 * 2 * self.g[v].width * self.n
        self.max_S = 1
        for pid, pi in enumerate(self.passes):
            self._emit_pass(pid, pi)
        self.node_arr = self.node_recs.reshape(-1)
        self.step_arr = np.array(self.steps, dtype=np.int32).reshape(-1)
        self.pass_arr = np.stack(self.pass_recs).reshape(-1) if self.pass_recs else np.zeros(0, np.int32)
        self.op_arr = np.stack(self.op_recs).reshape(-1) if self.op_recs else np.zeros(0, np.int32)
        self.int_pool = self.pools.int_array()
        self.dbl_pool = self.pools.dbl_array()
        max_ops = max((int(r[P_NOP]) for r in self.pass_recs), default=0)
        # box-per-thread kernel: per-box scratch items (pass buffers and row arrays in global memory)
        self.simt_buf = max((int(r[P_SIDES]) * int(r[P_SMEM]) for r in self.pass_recs), default=1)
        self.simt_rows = max((int(r[P_SIDES]) * 3 * int(r[P_S]) for r in self.pass_recs), default=1)
        # shared memory: pass working set + staged node table + staged op records (in doubles)
        stage = (len(self.g) * NODE_REC + max_ops * OP_REC + 1) // 2 + 2
        self.smem_total = self.max_smem + stage
        # a box-per-CTA working set beyond the opt-in shared memory of one CTA goes to the end of
        # the CTA's scratch slot (global memory, L1/L2-cached); shared memory keeps the tables
        self.pass_global = 0
        if self.mode == "cta" and self.smem_total > self.smem_limit // 8:
            self.pass_global = self.max_smem
            self.smem_total = stage
        self.header = np.array([len(self.g), len(self.steps), len(self.passes), len(self.op_recs),
                                self.n, self.S, self.t, self.arena_w, self.plane_w, self.fold_w,
                                self.smem_total, self.max_S, self.sin_off, self.maxw,
                                1 if self.return_a else 0, max_ops, self.simt_buf, self.simt_rows,
                                1 if self.x_in_la else 0, MODES[self.mode], self.cta_threads, self.pass_global,
                                TIE_RULES[self.tie_rule],
                                1 if (self.fold_tc and self.fold_w > 0 and self.pass_global == 0) else 0],
                               dtype=np.int32)

    def _emit_pass(self, pid, pi: PassInfo):
        g = self.g
        P = self.pools
        S = pi.S
        pats = pi.patterns
        # entry tables per node
        rowptr, cols, nnz, lookup = {}, {}, {}, {}
        for v, (pr, pc) in pats.items():
            rp = np.concatenate([[0], np.cumsum(np.bincount(pr, minlength=S))]).astype(np.int64)
            rowptr[v], cols[v], nnz[v] = rp, pc.astype(np.int64), int(rp[-1])
        # fold decision: root contributions only from linear/matmul-on-input ops with
        # at most one entry per row, in a non-final pass
        contributors = [v for v in pi.order if 0 in g[v].inputs and v in pats]
        fold = (not pi.final and not self.cuts and len(contributors) == 1 and
                all(g[v].kind in ("linear", "matmul") and v in self.fold_off and
                    np.diff(rowptr[v]).max(initial=0) <= 1 for v in contributors))
        # liveness-based buffer allocation (doubles per side)
        first_use = {pi.t: -1}
        last_use = {}
        for i, v in enumerate(pi.order):
            last_use[v] = i
            for p in g[v].inputs:
                if p not in first_use:
                    first_use[p] = i
        xdense = pi.final and self.return_a and self.x_in_la and not fold and 0 in pats
        if not fold:
            last_use[0] = len(pi.order)
        free, bufoff, top = [], {}, 0

        def alloc(v):
            nonlocal top
            size = max(nnz.get(v, 0), 1)
            size = (size + 3) // 4 * 4
            for k, (o, s_) in enumerate(free):
                if s_ >= size:
                    free.pop(k)
                    if s_ > size:
                        free.append((o + size, s_ - size))
                    return o
            o = top
            top += size
            return o

        def release(v):
            free.append((bufoff[v], (max(nnz.get(v, 0), 1) + 3) // 4 * 4))

        bufoff[pi.t] = alloc(pi.t)
        op_begin = len(self.op_recs)
        pat_off = {}

        def pattern(v_):
            if v_ not in pat_off:
                pat_off[v_] = (P.add_int(rowptr[v_]), P.add_int(cols[v_]))
            return pat_off[v_]
        kcount = {}
        for v in pi.order:
            if v in pats:
                for p in g[v].inputs:
                    kcount[p] = kcount.get(p, 0) + 1
        merged_before = {pi.t}
        for i, v in enumerate(pi.order):
            n = g[v]
            if v not in pats:
                continue
            for slot, p in enumerate(n.inputs):
                if p == 0 and fold:
                    continue
                if p == 0 and xdense:
                    bufoff[0] = ROOT_IN_LA
                    continue
                if p not in bufoff and p in pats:
                    bufoff[p] = alloc(p)
            k = n.kind
            for slot, p in enumerate(n.inputs):
                r = np.full(OP_REC, -1, dtype=np.int32)
                r[O_SINGLE] = 0                      # index-shape flags, set for pull-move ops below
                kk = k if k not in MAP_KINDS else "map"
                r[O_KIND] = NK[kk]
                r[O_V] = v
                r[O_SLOT] = slot
                r[O_FIRST] = 1 if slot == 0 else 0
                r[O_VBUF] = bufoff[v]
                r[O_VNNZ] = nnz[v]
                r[O_VRP], r[O_VCOLS] = pattern(v)
                r[O_U] = p
                r[O_WOUT] = n.width
                r[O_DENSE] = 1 if k in ("linear", "matmul") else 0
                r[O_FOLD] = 1 if (p == 0 and fold) else 0
                r[O_VMAXROW] = int(np.diff(rowptr[v]).max(initial=0))
                r[O_VROWS] = int((np.diff(rowptr[v]) > 0).sum())
                sd = pi.sides
                self.work["a_read"] += sd * nnz[v]
                if r[O_DENSE] == 1 and r[O_FOLD] == 0:
                    vlen = np.diff(rowptr[v])
                    self.work["gemm_flops"] += sd * 2 * int(vlen.sum()) * g[p].width
                    self.work["a_written"] += sd * int(np.diff(rowptr[p])[vlen > 0].sum())
                if r[O_FOLD] == 1:
                    r[O_UBUF] = -1
                    r[O_UNNZ] = 0
                    r[O_UMERGE] = 0
                    rows = np.nonzero(np.diff(rowptr[v]) > 0)[0]
                    r[O_SHORT] = P.add_int(rows)
                    r[O_NSHORT] = len(rows)
                    r[O_LONG] = P.add_int(np.zeros(0, np.int64))
                    r[O_NLONG] = 0
                    self.op_recs.append(r)
                    continue
                r[O_UBUF] = bufoff[p]
                r[O_UNNZ] = nnz[p]
                r[O_URP], r[O_UCOLS] = pattern(p)
                r[O_UMERGE] = 1 if p in merged_before else 0
                merged_before.add(p)
                r[O_UK] = kcount.get(p, 1)
                r[O_VMAXROW] = int(np.diff(rowptr[v]).max(initial=0))
                r[O_UMAXROW] = int(np.diff(rowptr[p]).max(initial=0))
                r[O_VROWS] = int((np.diff(rowptr[v]) > 0).sum())
                if r[O_DENSE] == 0:
                    tgt, sptr, src = self._moves(n, slot, rowptr, cols, v, p)
                    rows_of = np.repeat(np.arange(S), np.diff(rowptr[p]))
                    trow = rows_of[tgt] if len(tgt) else np.zeros(0, np.int64)
                    tptr = np.searchsorted(trow, np.arange(S + 1), side="left")
                    r[O_TPTR] = P.add_int(tptr)
                    r[O_TMAXROW] = int(np.diff(tptr).max(initial=0))
                    if p == 0 and xdense:
                        # entry (s, c) of the input's A lives at lA[s * n + c]
                        tgt = trow * self.n + cols[0][tgt]
                    r[O_NTGT] = len(tgt)
                    self.work["a_written"] += pi.sides * len(tgt)
                    r[O_TGT] = P.add_int(tgt)
                    r[O_SPTR] = P.add_int(sptr)
                    r[O_SRC] = P.add_int(src)
                    # index-shape flags (OpFlag in gear_program.h): every target pulls exactly one
                    # source; sources, targets, target row pointers or v's row pointers that are the
                    # identity, so the kernel computes the index instead of loading it
                    flags = 0
                    if len(src) == len(tgt):
                        flags |= OF_SINGLE
                    if len(src) and np.array_equal(src, np.arange(len(src))):
                        flags |= OF_SRC_ID
                    if np.array_equal(tgt, np.arange(len(tgt))):
                        flags |= OF_TGT_ID
                    if np.array_equal(tptr, np.arange(S + 1)):
                        flags |= OF_TPTR_ID
                    if np.array_equal(rowptr[v], np.arange(S + 1)):
                        flags |= OF_VRP_ID
                    r[O_SINGLE] = flags
                else:
                    r[O_NTGT] = 0
                # rows this op works on, split by length: short rows one thread, long rows one warp
                vlen = np.diff(rowptr[v])
                ulen = np.diff(rowptr[p]) if r[O_UMERGE] == 0 else np.zeros(S, np.int64)
                if p == 0 and xdense and r[O_UMERGE] == 0:
                    ulen = np.full(S, self.n, np.int64)
                tlen = np.diff(tptr) if r[O_DENSE] == 0 else np.zeros(S, np.int64)
                work = np.maximum(np.maximum(vlen, ulen), tlen)
                rows = np.nonzero(work > 0)[0]
                short = rows[work[rows] <= ROW_THREAD_MAX]
                long_ = rows[work[rows] > ROW_THREAD_MAX]
                r[O_SHORT] = P.add_int(short)
                r[O_NSHORT] = len(short)
                r[O_LONG] = P.add_int(long_)
                r[O_NLONG] = len(long_)
                # entry-wise op: entry e of v's row s moves to entry e of u's row s (one source per
                # target, identity sources and targets, the moves of row s are v's entries of row
                # s, and a fresh u row has exactly those entries): the kernel then takes each
                # entry's bias terms and its move in one sweep, without clearing u's row first
                # OF_FUSED_T: the same sweep with each entry's target read from the op's target list
                # (u's row holds more entries: it is cleared first when the op opens it)
                f = int(r[O_SINGLE])
                if (r[O_DENSE] == 0 and len(long_) == 0 and not (p == 0 and xdense) and
                        (f & (OF_SINGLE | OF_SRC_ID)) == (OF_SINGLE | OF_SRC_ID) and np.array_equal(tptr, rowptr[v])):
                    if (f & OF_TGT_ID) and (r[O_UMERGE] == 1 or np.array_equal(rowptr[p], rowptr[v])):
                        r[O_SINGLE] = f | OF_FUSED
                    else:
                        r[O_SINGLE] = f | OF_FUSED_T
                self.op_recs.append(r)
            if last_use.get(v, -2) == i and v != 0 and bufoff.get(v, 0) >= 0:
                release(v)
        if self.fold_tc and pi.final and xdense and pi.sides == 1:
            self._mark_split(op_begin)
        smem = top
        x_nnz = 0 if fold else nnz.get(0, 0)
        rec = np.full(PASS_REC, -1, dtype=np.int32)
        rec[P_T] = pi.t
        rec[P_S] = S
        rec[P_SIDES] = pi.sides
        rec[P_INIT] = pi.init
        rec[P_OP0] = op_begin
        rec[P_NOP] = len(self.op_recs) - op_begin
        rec[P_TBUF] = bufoff[pi.t]
        rec[P_XNNZ] = x_nnz
        rec[P_XBUF] = bufoff.get(0, -1) if not fold else -1
        if not fold and 0 in pats:
            rec[P_XRP], rec[P_XCOLS] = pattern(0)
        rec[P_NFOLD] = 1 if fold else 0
        rec[P_SMEM] = smem
        rec[P_TRP], rec[P_TCOLS] = pattern(pi.t)
        rec[P_FINAL] = 1 if pi.final else 0
        rec[P_NVISIT] = len([v for v in pi.order if v in pats])
        rec[P_MAXROW] = int(max(np.diff(rowptr[v]).max(initial=0) for v in pats if not (v == 0 and fold)))
        rec[P_ONEHOT] = 1 if rec[P_MAXROW] <= 1 else 0
        rec[P_XMAXROW] = int(np.diff(rowptr[0]).max(initial=0)) if (0 in pats and not fold) else 0
        rec[P_XDENSE] = 1 if xdense else 0
        rec[P_TMAXROW] = int(np.diff(rowptr[pi.t]).max(initial=0))
        self.work["a_written"] += pi.sides * nnz[pi.t]
        self.work["a_read"] += pi.sides * x_nnz
        self.work["node_visits"] += int(rec[P_NVISIT])
        self.pass_recs.append(rec)
        # kernel shared memory: per side the row arrays (S each: VAL, ERR, and ROOT in the final
        # pass) + the entry buffers, then the reduction slots
        nrows = 3 if pi.final else 2
        self.max_smem = max(self.max_smem, pi.sides * (nrows * S + smem) + 32)
        self.max_S = max(self.max_S, S)
        pi.bufoff = bufoff
        pi.fold = fold
        pi.nnz = nnz

    # smallest dense node (outputs) whose final-pass product goes to the tensor cores
    SPLIT_MIN_WIDTH = 128

    def _mark_split(self, op_begin):
        """Flag (OF_SPLIT) the final pass's product through a dense node on the input for the
        tensor cores: the pass's last op, the only one into the input, a Linear/MatMul step of
        at least SPLIT_MIN_WIDTH outputs whose transposed weights the program holds. The kernel
        then hands that product (A_v W over the whole batch) to a tcgen05 GEMM and the
        concretisation to a kernel after it (gear_capi.cu)."""
        ops = self.op_recs[op_begin:]
        into_x = [r for r in ops if r[O_U] == 0]
        if len(into_x) != 1 or ops[-1] is not into_x[0]:
            return
        r = into_x[0]
        v = int(r[O_V])
        nd = self.g[v]
        if (r[O_DENSE] != 1 or r[O_FOLD] != 0 or r[O_UMERGE] != 0 or r[O_UK] > 1 or
                nd.kind not in ("linear", "matmul") or v not in self.fold_off or nd.width < self.SPLIT_MIN_WIDTH):
            return
        r[O_SINGLE] = int(r[O_SINGLE]) | OF_SPLIT
        self.split_op = v

    def _moves(self, n, slot, rowptr, cols, v, p):
        """Pull lists: for each target entry of input p, the source entries of v.

        Rows are handled all at once: an entry (row s, column c) has the sort key s (W + 1) + c,
        which orders entries by row, then column (columns ascend within a row)."""
        g = self.g
        k, a = n.kind, n.attrs
        rp_v, cols_v = np.asarray(rowptr[v], np.int64), np.asarray(cols[v], np.int64)
        rp_u, cols_u = np.asarray(rowptr[p], np.int64), np.asarray(cols[p], np.int64)
        S = len(rp_v) - 1
        w_in = g[p].width
        row_v = np.repeat(np.arange(S, dtype=np.int64), np.diff(rp_v))
        row_u = np.repeat(np.arange(S, dtype=np.int64), np.diff(rp_u))
        if k == "reducesum":
            W = g[v].width + 1
            key_v = row_v * W + cols_v
            key_u = row_u * W + np.asarray(a["rmap"], np.int64)[cols_u]
            pos = np.searchsorted(key_v, key_u)
            hit = pos < len(key_v)
            hit[hit] = key_v[pos[hit]] == key_u[hit]
            tgt = np.nonzero(hit)[0].astype(np.int64)
            src = pos[hit].astype(np.int64)
            sptr = np.arange(len(tgt) + 1, dtype=np.int64)
            return tgt, sptr, src
        if k in ("neg", "sqr", "exp", "log", "sin", "cos", "pow"):
            m = None
        elif k in ("mulc", "addc", "subc", "rsubc"):
            m = a["map0"]
        elif k in ("mul", "add", "sub"):
            m = a["map0"] if slot == 0 else a["map1"]
        elif k in MAP_KINDS:
            m = a["map"]
        elif k == "concat":
            off = sum(g[q].width for q in n.inputs[:slot])
            m = a["cmap"] - off
        else:
            raise ProgramError(k)
        tc = cols_v if m is None else np.asarray(m, np.int64)[cols_v]
        keep = (tc >= 0) & (tc < w_in) if k == "concat" else np.ones(len(tc), bool)
        W = w_in + 1
        key_u = row_u * W + cols_u
        srcs = np.nonzero(keep)[0].astype(np.int64)
        tj = np.searchsorted(key_u, row_v[keep] * W + tc[keep]).astype(np.int64)
        order = np.argsort(tj, kind="stable")
        tj, srcs = tj[order], srcs[order]
        tgt, start, counts = np.unique(tj, return_index=True, return_counts=True)
        sptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        return tgt.astype(np.int64), sptr, srcs

    # ================================================================= info
    def alg_bytes_per_box(self) -> int:
        """Algorithmic bytes per bounded box, float64 throughout: 8 (A read + A written) of the
        executed schedule + the box in (16 n) + lb, lbias out (16 S) + lA out (8 S n)."""
        w = self.work
        return 8 * (w["a_read"] + w["a_written"]) + 16 * self.n + 16 * self.S + 8 * self.S * self.n

    def describe(self) -> str:
        lines = [f"nodes={len(self.g)} steps={len(self.steps)} passes={len(self.passes)} ops={len(self.op_recs)} "
                 f"arena={self.arena_w} planes={self.plane_w} fold={self.fold_w} smem_doubles={self.max_smem}"]
        for pid, pi in enumerate(self.passes):
            r = self.pass_recs[pid]
            lines.append(f"  pass {pid}: t={pi.t}({self.g[pi.t].kind}) S={pi.S} sides={pi.sides} final={pi.final} "
                         f"fold={pi.fold} visits={r[P_NVISIT]} smem={r[P_SMEM]} x_nnz={r[P_XNNZ]} maxrow={r[P_MAXROW]}")
        return "\n".join(lines)


# ===================================================================== compile pools
_KEEP = ("S", "n", "t", "mode", "cta_threads", "tie_rule", "cuts", "fold_tc", "split_op", "x_in_la", "return_a", "dense_c", "arena_w", "plane_w", "fold_w", "maxw",
         "max_S", "max_smem", "smem_total", "pass_global", "simt_buf", "simt_rows", "sin_off", "work", "header",
         "node_arr", "step_arr", "pass_arr", "op_arr", "int_pool", "dbl_pool")


def stripped(prog: Program) -> Program:
    """A copy of prog with only what the device upload and the work counters need (no graph,
    no pass patterns): small to send between processes."""
    out = Program.__new__(Program)
    for k in _KEEP:
        if hasattr(prog, k):
            setattr(out, k, getattr(prog, k))
    return out


def simt_items(prog: Program) -> int:
    """Doubles of box-per-thread scratch one box needs."""
    return 3 * prog.arena_w + prog.plane_w + prog.fold_w + 4 * prog.maxw + prog.simt_buf + prog.simt_rows


def _compile_job(job):
    graph, kw, simt_items_max = job
    if simt_items_max is not None:
        # "auto": one box per thread when the per-box state is small, else one box per CTA
        prog = Program(graph, mode="simt", tie_rule=kw.get("tie_rule", "reference"))
        if simt_items(prog) <= simt_items_max:
            return stripped(prog)
    return stripped(Program(graph, **kw))


def compile_many(graphs, kw=None, simt_items_max=None, workers=None):
    """Programs for many graphs, compiled in a process pool ("spawn" start method, so it is
    safe after CUDA is initialised). kw: Program keyword arguments; simt_items_max: when
    given, a graph whose box-per-thread program needs at most this many doubles per box gets
    that program, the others Program(graph, **kw). Returns stripped programs in order."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    kw = dict(kw or {})
    jobs = [(g, kw, simt_items_max) for g in graphs]
    workers = workers or min(len(jobs), os.cpu_count() or 1)
    if workers <= 1 or len(jobs) <= 1:
        return [_compile_job(j) for j in jobs]
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_compile_job, jobs, chunksize=max(1, len(jobs) // (4 * workers))))
