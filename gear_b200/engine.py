"""Device engine: a compiled program on the GPU and the launch of the CROWN megakernel."""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _lib
from .graph import Graph
from .program import Program


# kernel variants an "auto" engine chooses from: (execution mode, threads per CTA)
VARIANTS = (("simt", 128), ("cta", 64), ("cta", 128), ("cta", 256))
# the box-per-thread kernel keeps every per-box array in global memory: beyond this many
# doubles per box it streams too much to compete, and "auto" does not try it
SIMT_MAX_ITEMS = 65536
# many-instance launches: an instance whose box-per-thread state is at most this many doubles
# joins the box-per-thread group, and a box-per-CTA program whose pass working set exceeds
# PACK_SMEM_LIMIT bytes keeps it in global memory (more CTAs per SM); measured fastest on the
# mixed family over thresholds 2048-65536 and limits 16 KB-227 KB
SIMT_PACK_ITEMS = 8192
PACK_SMEM_LIMIT = 48 << 10
# a many-instance launch gives every CTA the largest shared-memory size of its programs, so
# box-per-CTA programs launch in size classes (upper bounds in bytes; 6 / 3 / 2 / 1 CTAs of
# that size fit an SM's 228 KB)
SMEM_CLASSES = (32 << 10, 72 << 10, 108 << 10, 232448)


def smem_class(prog) -> int:
    """Size class of a box-per-CTA program's dynamic shared memory (0 for other programs)."""
    if prog.mode != "cta":
        return 0
    b = 8 * int(prog.smem_total)
    return next((i for i, c in enumerate(SMEM_CLASSES) if b <= c), len(SMEM_CLASSES))


class _Dag:
    """One compiled program uploaded to the device (a gear_dag handle)."""

    def __init__(self, graph, spec_rows, dense_c, mode, cta_threads, tie_rule="reference", fold_tc=False):
        self._upload(Program(graph, spec_rows=spec_rows, dense_c=dense_c, mode=mode, cta_threads=cta_threads,
                             tie_rule=tie_rule, fold_tc=fold_tc))

    def _upload(self, prog):
        self.prog = p = prog
        mode, cta_threads = prog.mode, prog.cta_threads
        L = _lib.lib()
        h = ctypes.c_void_p()
        arrs = [np.ascontiguousarray(a, dtype=np.int32) for a in
                (p.header, p.node_arr, p.step_arr, p.pass_arr, p.op_arr, p.int_pool)]
        dbl = np.ascontiguousarray(p.dbl_pool, dtype=np.float64)
        st = L.gear_dag_create(_lib.ptr_i32(arrs[0]), arrs[0].size, _lib.ptr_i32(arrs[1]), arrs[1].size,
                               _lib.ptr_i32(arrs[2]), arrs[2].size, _lib.ptr_i32(arrs[3]), arrs[3].size,
                               _lib.ptr_i32(arrs[4]), arrs[4].size, _lib.ptr_i32(arrs[5]), arrs[5].size,
                               _lib.ptr_dbl(dbl), dbl.size, ctypes.byref(h))
        _lib.check(st, "gear_dag_create")
        self.handle = h
        self.name = f"{mode}{cta_threads}" if mode == "cta" else mode

    @classmethod
    def from_program(cls, prog):
        """Upload an already compiled Program."""
        self = cls.__new__(cls)
        self._upload(prog)
        return self

    def simt_items(self):
        p = self.prog
        return 3 * p.arena_w + p.plane_w + p.fold_w + 4 * p.maxw + p.simt_buf + p.simt_rows

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().gear_dag_destroy(h)
            except Exception:
                pass
            self.handle = None


class CrownEngine:
    """One graph and one specification kind (identity or dense C) on the current device.

    mode "cta" runs one box per CTA (cta_threads threads), "simt" one box per thread; both
    give the same bounds. mode "auto" times the kernel variants on the first call for each
    batch size class (powers of two) on the caller's own boxes and keeps the fastest.
    tie_rule: the McCormick tie rule of the compiled programs (``Program``); fold_tc: the fold
    products of dense nodes on the input on the tensor cores (box-per-CTA variants)."""

    def __init__(self, graph: Graph, spec_rows: Optional[int] = None, dense_c: bool = False, mode: str = "auto",
                 cta_threads: int = 128, tie_rule: str = "reference", fold_tc: bool = False):
        if not torch.cuda.is_available():
            raise _lib.GearError("gear_b200 needs a CUDA device (no CPU fallback)")
        if mode not in ("auto", "cta", "simt"):
            raise ValueError(f"unknown mode {mode!r}")
        self.graph = graph
        self.mode = mode
        self.dense_c = dense_c
        self._args = (graph, spec_rows, dense_c)
        self.tie_rule = tie_rule
        self.fold_tc = fold_tc
        self._dags = {}
        first = ("cta", cta_threads) if mode == "auto" else (mode, cta_threads)
        d = self._dag(*first)
        self.prog = d.prog
        self.handle = d.handle
        self.n = d.prog.n
        self.S = d.prog.S
        self._choice = {}          # batch size class -> variant
        self.timings = {}          # batch size class -> {variant name: ms}
        self._ws = None

    def _dag(self, mode, threads):
        key = (mode, threads if mode == "cta" else 0)
        if key not in self._dags:
            self._dags[key] = _Dag(*self._args, mode, threads, self.tie_rule, self.fold_tc)
        return self._dags[key]

    def _candidates(self):
        items = self._dags[next(iter(self._dags))].simt_items()
        return [(m, t) for m, t in VARIANTS if not (m == "simt" and items > SIMT_MAX_ITEMS)]

    def variant(self, batch: int) -> str:
        """Name of the kernel variant used for this batch size ("simt", "cta64", ...)."""
        v = self._choice.get(self._bucket(batch))
        if self.mode == "fixed":
            return self._fixed.name
        if self.mode != "auto":
            return self._dags[next(iter(self._dags))].name
        return None if v is None else self._dag(*v).name

    def kernel_name(self, batch: int) -> Optional[str]:
        """The CROWN kernel instance this batch size launches (crown_megakernel<threads, global
        working set, tensor-core fold> or crown_simt_kernel)."""
        v = self.variant(batch)
        if v is None:
            return None
        if v == "simt":
            return "crown_simt_kernel"
        if self.mode == "fixed":
            prog = self._fixed.prog
        elif self.mode == "auto":
            prog = self._dag(*self._choice[self._bucket(batch)]).prog
        else:
            prog = self._dags[next(iter(self._dags))].prog
        gws = int(prog.pass_global > 0)
        fx = int(int(prog.header[23]) != 0)
        return f"crown_megakernel<{v[3:]}, {gws}, {fx}>"

    def freeze(self, x_L: torch.Tensor, x_U: torch.Tensor, C: Optional[torch.Tensor] = None):
        """Time the variants once on these boxes and use the fastest for every later batch size
        (a caller whose batches vary, like a branch-and-bound loop, pays the timing once)."""
        if self.mode != "auto":
            return self.variant(x_L.shape[0])
        self.lower(x_L, x_U, C)
        choice = self._choice[self._bucket(x_L.shape[0])]
        self._fixed = self._dag(*choice)
        self.handle, self.prog = self._fixed.handle, self._fixed.prog
        self.mode = "fixed"
        return self._fixed.name

    @staticmethod
    def _bucket(batch):
        return max(int(batch) - 1, 0).bit_length()

    def workspace(self, batch: int, device) -> torch.Tensor:
        """Scratch for the current variant (self.handle) at this batch size."""
        return self._workspace_bytes(int(_lib.lib().gear_crown_workspace_bytes(self.handle, batch)), device)

    def lower(self, x_L: torch.Tensor, x_U: torch.Tensor, C: Optional[torch.Tensor] = None,
              return_A: bool = True, out=None, lb_ibp: Optional[torch.Tensor] = None):
        """lb (B, S), lA (B, S, n) or None, lbias (B, S) -- all float64 on x_L's device.

        lb_ibp (B, S): when given, it receives the rows' bounds over the output's plain IBP
        interval and lb is the larger of that and CROWN's (the bounding glue's IBP pass)."""
        B = x_L.shape[0]
        dev = x_L.device
        if dev.type != "cuda":
            raise _lib.GearError("inputs must be CUDA tensors")
        w = -1 if B else self.n                     # an empty batch has no width to infer
        x_L = x_L.reshape(B, w).to(torch.float64).contiguous()
        x_U = x_U.reshape(B, w).to(torch.float64).contiguous()
        if x_L.shape[1] != self.n:
            raise ValueError(f"input width {x_L.shape[1]} != {self.n}")
        if self.dense_c:
            if C is None:
                raise ValueError("this engine expects a dense C")
            C = C.to(torch.float64).contiguous()
        if out is None:
            lb = torch.empty(B, self.S, dtype=torch.float64, device=dev)
            lA = torch.empty(B, self.S, self.n, dtype=torch.float64, device=dev)
            lbias = torch.empty(B, self.S, dtype=torch.float64, device=dev)
        else:
            lb, lA, lbias = out
        if B == 0:
            return lb, (lA if return_A else None), lbias
        if self.mode == "auto":
            dag = self._select(x_L, x_U, C, lb, lA, lbias)
        elif self.mode == "fixed":
            dag = self._fixed
        else:
            dag = self._dags[next(iter(self._dags))]
        self._launch(dag, x_L, x_U, C, lb, lA, lbias, lb_ibp)
        return lb, (lA if return_A else None), lbias

    def _launch(self, dag, x_L, x_U, C, lb, lA, lbias, lb_ibp=None):
        B = x_L.shape[0]
        L = _lib.lib()
        nbytes = int(L.gear_crown_workspace_bytes(dag.handle, B))
        ws = self._workspace_bytes(nbytes, x_L.device)
        stream = torch.cuda.current_stream(x_L.device).cuda_stream
        cptr = C.data_ptr() if self.dense_c else None
        if lb_ibp is None:
            st = L.gear_crown_lower(dag.handle, x_L.data_ptr(), x_U.data_ptr(), B, cptr, lb.data_ptr(), lA.data_ptr(),
                                    lbias.data_ptr(), ws.data_ptr(), ws.numel(), stream)
        else:
            st = L.gear_crown_lower_ibp(dag.handle, x_L.data_ptr(), x_U.data_ptr(), B, cptr, lb.data_ptr(),
                                        lA.data_ptr(), lbias.data_ptr(), lb_ibp.data_ptr(), ws.data_ptr(), ws.numel(),
                                        stream)
        _lib.check(st, "gear_crown_lower")

    def _select(self, x_L, x_U, C, lb, lA, lbias):
        """The variant for this batch size class; timed on these boxes the first time."""
        B = x_L.shape[0]
        key = self._bucket(B)
        if key not in self._choice:
            times = {}
            for cand in self._candidates():
                dag = self._dag(*cand)
                # warm-up at the full batch (module load, this variant's workspace, caches), then
                # the faster of two timed launches: one cold launch has misjudged a variant by 50%
                self._launch(dag, x_L, x_U, C, lb, lA, lbias)
                best = None
                for _ in range(2):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    self._launch(dag, x_L, x_U, C, lb, lA, lbias)
                    e1.record()
                    torch.cuda.synchronize()
                    t = e0.elapsed_time(e1)
                    best = t if best is None else min(best, t)
                times[cand] = best
            best = min(times, key=times.get)
            self._choice[key] = best
            self.timings[key] = {self._dag(*c).name: t for c, t in times.items()}
        dag = self._dag(*self._choice[key])
        self.handle = dag.handle
        self.prog = dag.prog
        return dag

    def _workspace_bytes(self, nbytes, device):
        if self._ws is None or self._ws.numel() < nbytes or self._ws.device != device:
            self._ws = None
            self._ws = torch.empty(max(nbytes, 8), dtype=torch.uint8, device=device)
        return self._ws


class MultiEngine:
    """Many instances (graphs of different widths and depths) in one kernel launch per kernel
    variant.

    ``lower(boxes)`` takes ``[(x_L_i, x_U_i), ...]`` (CUDA float64, x_L_i of shape (B_i, n_i); B_i
    may be 0) and returns ``[(lb_i, lA_i, lbias_i), ...]``; instance i's results are the ones
    ``CrownEngine`` gives for it alone (the same kernel code runs every box). Instances are
    grouped by kernel variant and each group is one persistent launch: with mode "auto" an
    instance whose per-box state fits ``simt_items_max`` doubles runs one box per thread, the
    others one box per CTA of ``cta_threads`` threads; "cta" / "simt" put every instance in
    that mode. Within a group, instances are handed to the launch in decreasing per-box work,
    so the device's work counter deals the expensive boxes first. With ``concurrent`` the
    groups' launches run on side streams at the same time, joined back into the caller's
    stream before lower() returns; off by default: two persistent launches that each size
    their grid for the whole GPU compete for it (measured 11% slower on the mixed family)."""

    def __init__(self, graphs, mode: str = "auto", cta_threads: int = 256, simt_items_max: int = SIMT_PACK_ITEMS,
                 programs=None, concurrent: bool = False, tie_rule: str = "reference"):
        if not torch.cuda.is_available():
            raise _lib.GearError("gear_b200 needs a CUDA device (no CPU fallback)")
        if mode not in ("auto", "cta", "simt"):
            raise ValueError(f"unknown mode {mode!r}")
        self.graphs = list(graphs)
        self.mode = mode
        # programs: optional precompiled Program per instance in its variant (a compile pool)
        self.dags = []
        self.variants = []
        for i, g in enumerate(self.graphs):
            if programs is not None:
                prog = programs[i]
                var = (prog.mode, prog.cta_threads if prog.mode == "cta" else 0)
            else:
                var = ("simt", 0) if mode == "simt" else ("cta", cta_threads)
                if mode == "auto":
                    probe = Program(g, mode="simt", tie_rule=tie_rule)
                    items = 3 * probe.arena_w + probe.plane_w + probe.fold_w + 4 * probe.maxw + probe.simt_buf + \
                        probe.simt_rows
                    var = ("simt", 0) if items <= simt_items_max else ("cta", cta_threads)
                    prog = probe if var[0] == "simt" else None
                else:
                    prog = None
                if prog is None:
                    prog = Program(g, mode=var[0], cta_threads=var[1] if var[0] == "cta" else 128,
                                   smem_limit=PACK_SMEM_LIMIT, tie_rule=tie_rule)
            self.dags.append(_Dag.from_program(prog))
            # a launch also needs one pass working-set placement (shared or global memory); the
            # fourth field is the shared-memory size class
            self.variants.append((var[0], var[1], bool(getattr(prog, "pass_global", 0)), smem_class(prog)))
        self.n = [d.prog.n for d in self.dags]
        self.S = [d.prog.S for d in self.dags]
        cost = [d.prog.alg_bytes_per_box() for d in self.dags]
        self.groups = {}
        for i in sorted(range(len(self.dags)), key=lambda i: (-cost[i], i)):
            self.groups.setdefault(self.variants[i], []).append(i)
        self._ws = {}
        self.group_events = None
        self.concurrent = concurrent
        self._streams = {}

    @staticmethod
    def _name(key):
        m, t, gws, sc = key
        return (f"cta{t}" + ("-global" if gws else f"-smem{sc}")) if m == "cta" else "simt"

    def group_names(self):
        return {self._name(k): len(ix) for k, ix in self.groups.items()}

    def outputs(self, batches, device):
        """Result tensors for these batch sizes: views into three flat buffers."""
        tot_lb = sum(b * s for b, s in zip(batches, self.S))
        tot_la = sum(b * s * n for b, s, n in zip(batches, self.S, self.n))
        lb = torch.empty(max(tot_lb, 1), dtype=torch.float64, device=device)
        lbias = torch.empty(max(tot_lb, 1), dtype=torch.float64, device=device)
        lA = torch.empty(max(tot_la, 1), dtype=torch.float64, device=device)
        outs, o1, o2 = [], 0, 0
        for b, s, n in zip(batches, self.S, self.n):
            outs.append((lb[o1:o1 + b * s].view(b, s), lA[o2:o2 + b * s * n].view(b, s, n),
                         lbias[o1:o1 + b * s].view(b, s)))
            o1 += b * s
            o2 += b * s * n
        return outs

    def _args(self, idx, boxes, outs, lb_ibp=None):
        args = (_lib.LowerArgs * len(idx))()
        for k, i in enumerate(idx):
            x_L, x_U = boxes[i]
            lb, lA, lbias = outs[i]
            B = x_L.shape[0]
            ibp = lb_ibp[i] if lb_ibp is not None else None
            args[k] = _lib.LowerArgs(self.dags[i].handle.value, x_L.data_ptr() if B else None,
                                     x_U.data_ptr() if B else None, B, None, lb.data_ptr() if B else None,
                                     lA.data_ptr() if B else None, lbias.data_ptr() if B else None,
                                     ibp.data_ptr() if (B and ibp is not None) else None)
        return args

    def _launch(self, key, args, device):
        L = _lib.lib()
        nbytes = int(L.gear_crown_multi_workspace_bytes(args, len(args)))
        if nbytes < 0:
            _lib.check(-1, "gear_crown_multi_workspace_bytes")
        ws = self._ws.get(key)
        if ws is None or ws.numel() < nbytes or ws.device != device:
            self._ws[key] = None
            ws = self._ws[key] = torch.empty(max(nbytes, 8), dtype=torch.uint8, device=device)
        stream = torch.cuda.current_stream(device).cuda_stream
        _lib.check(L.gear_crown_lower_multi(args, len(args), ws.data_ptr(), ws.numel(), stream),
                   "gear_crown_lower_multi")

    def lower(self, boxes, out=None, lb_ibp=None):
        """lb_ibp: optional list of (B_i, S_i) tensors (or None entries) receiving the rows' plain
        IBP bounds; lb is then max(CROWN, IBP), as CrownEngine.lower(lb_ibp=...)."""
        if len(boxes) != len(self.graphs):
            raise ValueError(f"{len(boxes)} box sets for {len(self.graphs)} instances")
        dev = None
        norm = []
        for i, (x_L, x_U) in enumerate(boxes):
            if x_L.device.type != "cuda":
                raise _lib.GearError("inputs must be CUDA tensors")
            dev = x_L.device
            B = x_L.shape[0]
            x_L = x_L.reshape(B, self.n[i]).to(torch.float64).contiguous()
            x_U = x_U.reshape(B, self.n[i]).to(torch.float64).contiguous()
            norm.append((x_L, x_U))
        if dev is None:
            return []
        outs = out if out is not None else self.outputs([x.shape[0] for x, _ in norm], dev)
        cur = torch.cuda.current_stream(dev)
        side = self.concurrent and len(self.groups) > 1
        if side:
            # the groups' launches run side by side (one stream each), joined back into the
            # caller's stream: the tail of one group's launch overlaps the others
            ready = torch.cuda.Event()
            ready.record(cur)
        for key, idx in self.groups.items():
            st = cur
            if side:
                st = self._streams.get(key)
                if st is None or st.device != dev:
                    st = self._streams[key] = torch.cuda.Stream(dev)
                st.wait_event(ready)
            with torch.cuda.stream(st):
                if self.group_events is not None:
                    e = self.group_events.setdefault(key, (torch.cuda.Event(enable_timing=True),
                                                           torch.cuda.Event(enable_timing=True)))
                    e[0].record(st)
                self._launch(key, self._args(idx, norm, outs, lb_ibp), dev)
                if self.group_events is not None:
                    e[1].record(st)
            if side:
                done = torch.cuda.Event()
                done.record(st)
                cur.wait_event(done)
        return outs

    def prepare(self, boxes, out, lb_ibp=None):
        """Plan every group's launch for these box buffers and outputs once (instance tables
        uploaded into per-group workspaces); launch_prepared() then runs the call with fixed
        arguments, capturable in a CUDA graph. The buffers must stay allocated and in place;
        a box set of 0 rows leaves its instance out."""
        self.release_prepared()
        L = _lib.lib()
        plans = []
        for key, idx in self.groups.items():
            args = self._args(idx, boxes, out, lb_ibp)
            nbytes = int(L.gear_crown_multi_workspace_bytes(args, len(args)))
            if nbytes < 0:
                _lib.check(-1, "gear_crown_multi_workspace_bytes")
            if nbytes == 0:
                continue
            dev = next(b[0].device for b in boxes)
            ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
            h = ctypes.c_void_p()
            _lib.check(L.gear_crown_multi_prepare(args, len(args), ws.data_ptr(), ws.numel(), ctypes.byref(h)),
                       "gear_crown_multi_prepare")
            plans.append((h, ws, args))
        self._plans = plans

    def launch_prepared(self):
        """The prepared call (prepare()): one launch per kernel group on the current stream."""
        L = _lib.lib()
        for h, ws, _ in self._plans:
            _lib.check(L.gear_crown_multi_launch(h, torch.cuda.current_stream(ws.device).cuda_stream),
                       "gear_crown_multi_launch")

    def release_prepared(self):
        L = _lib.lib()
        for h, _, _ in getattr(self, "_plans", []):
            L.gear_crown_multi_plan_destroy(h)
        self._plans = []

    def __del__(self):
        try:
            self.release_prepared()
        except Exception:
            pass

    def group_ms(self):
        """Device time of each group's launch in the last lower() (after record_groups())."""
        torch.cuda.synchronize()
        return {self._name(k): e[0].elapsed_time(e[1]) for k, e in (self.group_events or {}).items()}

    def record_groups(self, on: bool = True):
        self.group_events = {} if on else None

    def launches(self):
        """Kernel launches per lower() call (one per variant group)."""
        return len(self.groups)


class PlainEngine:
    """The plain GPU form of one instance: the same bounds as CrownEngine(mode="cta"), computed
    unfused (gear_crown_lower_plain): one kernel launch per schedule step, and per CROWN pass one
    launch per op plus one for its initial A and one for its concretisation, with every box's
    state in global memory between launches. The baseline the fused launch is measured against."""

    def __init__(self, graph: Graph, cta_threads: int = 128, tie_rule: str = "reference"):
        if not torch.cuda.is_available():
            raise _lib.GearError("gear_b200 needs a CUDA device (no CPU fallback)")
        self.dag = _Dag.from_program(Program(graph, mode="cta", cta_threads=cta_threads, smem_limit=0,
                                             tie_rule=tie_rule))
        self.prog = self.dag.prog
        self.n, self.S = self.prog.n, self.prog.S
        self._ws = None
        self.launches = 0

    def lower(self, x_L: torch.Tensor, x_U: torch.Tensor, out=None, lb_ibp: Optional[torch.Tensor] = None):
        """lb, lA, lbias as CrownEngine.lower; lb_ibp (B, S) as there (the bounding glue's IBP pass)."""
        B = x_L.shape[0]
        dev = x_L.device
        if dev.type != "cuda":
            raise _lib.GearError("inputs must be CUDA tensors")
        x_L = x_L.reshape(B, self.n).to(torch.float64).contiguous()
        x_U = x_U.reshape(B, self.n).to(torch.float64).contiguous()
        if out is None:
            out = (torch.empty(B, self.S, dtype=torch.float64, device=dev),
                   torch.empty(B, self.S, self.n, dtype=torch.float64, device=dev),
                   torch.empty(B, self.S, dtype=torch.float64, device=dev))
        if B == 0:
            return out
        lb, lA, lbias = out
        L = _lib.lib()
        nbytes = int(L.gear_crown_plain_workspace_bytes(self.dag.handle, B))
        if self._ws is None or self._ws.numel() < nbytes or self._ws.device != dev:
            self._ws = None
            self._ws = torch.empty(max(nbytes, 8), dtype=torch.uint8, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        if lb_ibp is None:
            _lib.check(L.gear_crown_lower_plain(self.dag.handle, x_L.data_ptr(), x_U.data_ptr(), B, None,
                                                lb.data_ptr(), lA.data_ptr(), lbias.data_ptr(), self._ws.data_ptr(),
                                                self._ws.numel(), stream), "gear_crown_lower_plain")
        else:
            _lib.check(L.gear_crown_lower_plain_ibp(self.dag.handle, x_L.data_ptr(), x_U.data_ptr(), B, None,
                                                    lb.data_ptr(), lA.data_ptr(), lbias.data_ptr(), lb_ibp.data_ptr(),
                                                    self._ws.data_ptr(), self._ws.numel(), stream),
                       "gear_crown_lower_plain_ibp")
        self.launches = int(L.gear_last_launch_count())
        return out


class CutEngine:
    """CROWN bounds with every concretisation over the box intersected with cut rows
    (gear_crown_lower_cuts; the reference's compute_bounds with PerturbationLpNorm(x_L, x_U,
    constraints=(A, b)), auto_LiRPA/bound_general.py:1275): each intermediate pass and the final
    pass bound their rows by the constrained dual sweep (concretize_func.py:431-850). Runs the
    plain form's launch sequence on a program compiled for cut rows (no folded passes, pass
    working set in global memory), plus a dense-row launch and a sweep per pass."""

    def __init__(self, graph: Graph, spec_rows: Optional[int] = None, dense_c: bool = False, cta_threads: int = 128,
                 tie_rule: str = "reference", max_rows: int = 0):
        if not torch.cuda.is_available():
            raise _lib.GearError("gear_b200 needs a CUDA device (no CPU fallback)")
        self.dag = _Dag.from_program(Program(graph, spec_rows=spec_rows, dense_c=dense_c, mode="cta",
                                             cta_threads=cta_threads, smem_limit=0, tie_rule=tie_rule, cuts=True))
        self.prog = self.dag.prog
        self.n, self.S = self.prog.n, self.prog.S
        self.max_rows = int(max_rows)
        self._ws = None
        self.launches = 0

    def lower(self, x_L: torch.Tensor, x_U: torch.Tensor, cut_A: Optional[torch.Tensor], cut_b: Optional[torch.Tensor],
              C: Optional[torch.Tensor] = None, out=None, lb_ibp: Optional[torch.Tensor] = None,
              max_rows: Optional[int] = None):
        """lb (B, S), lA (B, S, n), lbias (B, S) under the rows cut_A (B, K, n) x + cut_b (B, K) <= 0
        (K may be 0 or cut_A None: the box bound with the sweep's rounding)."""
        B = x_L.shape[0]
        dev = x_L.device
        if dev.type != "cuda":
            raise _lib.GearError("inputs must be CUDA tensors")
        x_L = x_L.reshape(B, self.n).to(torch.float64).contiguous()
        x_U = x_U.reshape(B, self.n).to(torch.float64).contiguous()
        if cut_A is None:
            K = 0
            cA = cb = None
        else:
            cA = cut_A.reshape(B, -1, self.n).to(dev, torch.float64).contiguous()
            K = int(cA.shape[1])
            cb = cut_b.reshape(B, K).to(dev, torch.float64).contiguous()
        if C is not None:
            C = C.to(dev, torch.float64).contiguous()
        if out is None:
            out = (torch.empty(B, self.S, dtype=torch.float64, device=dev),
                   torch.empty(B, self.S, self.n, dtype=torch.float64, device=dev),
                   torch.empty(B, self.S, dtype=torch.float64, device=dev))
        if B == 0:
            return out
        lb, lA, lbias = out
        L = _lib.lib()
        nbytes = int(L.gear_crown_cuts_workspace_bytes(self.dag.handle, B, K))
        if nbytes < 0:
            raise _lib.GearError("gear_crown_cuts_workspace_bytes: program not compiled for cut rows")
        if self._ws is None or self._ws.numel() < nbytes or self._ws.device != dev:
            self._ws = None
            self._ws = torch.empty(max(nbytes, 8), dtype=torch.uint8, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        mr = self.max_rows if max_rows is None else int(max_rows)
        _lib.check(L.gear_crown_lower_cuts(self.dag.handle, x_L.data_ptr(), x_U.data_ptr(), B,
                                           C.data_ptr() if C is not None else None,
                                           cA.data_ptr() if K else None, cb.data_ptr() if K else None, K, mr,
                                           lb.data_ptr(), lA.data_ptr(), lbias.data_ptr(),
                                           lb_ibp.data_ptr() if lb_ibp is not None else None,
                                           self._ws.data_ptr(), self._ws.numel(), stream), "gear_crown_lower_cuts")
        self.launches = int(L.gear_last_launch_count())
        return out


class PlainMultiEngine:
    """The plain GPU form of many instances (the denominator of the uneven batch): each instance
    bounded alone by its own PlainEngine, one instance after another, one kernel launch per
    schedule step and per op. Same lower(boxes, out, lb_ibp) interface as MultiEngine.
    programs: optional precompiled plain programs (Program(graph, mode="cta", smem_limit=0))."""

    def __init__(self, graphs, programs=None, cta_threads: int = 128):
        if not torch.cuda.is_available():
            raise _lib.GearError("gear_b200 needs a CUDA device (no CPU fallback)")
        self.engines = []
        for i, g in enumerate(graphs):
            pe = PlainEngine.__new__(PlainEngine)
            prog = programs[i] if programs is not None else Program(g, mode="cta", cta_threads=cta_threads,
                                                                    smem_limit=0)
            pe.dag = _Dag.from_program(prog)
            pe.prog = prog
            pe.n, pe.S = prog.n, prog.S
            pe._ws = None
            pe.launches = 0
            self.engines.append(pe)
        self.n = [e.n for e in self.engines]
        self.S = [e.S for e in self.engines]
        self.launch_count = 0

    def lower(self, boxes, out=None, lb_ibp=None):
        outs = []
        self.launch_count = 0
        for i, (x_L, x_U) in enumerate(boxes):
            e = self.engines[i]
            B = x_L.shape[0]
            o = out[i] if out is not None else None
            ibp = lb_ibp[i] if lb_ibp is not None else None
            if B == 0:
                dev = x_L.device
                outs.append((torch.empty(0, e.S, dtype=torch.float64, device=dev),
                             torch.empty(0, e.S, e.n, dtype=torch.float64, device=dev),
                             torch.empty(0, e.S, dtype=torch.float64, device=dev)))
                continue
            outs.append(e.lower(x_L, x_U, out=o, lb_ibp=ibp))
            self.launch_count += e.launches
        return outs
