"""Autotuner of the CROWN kernel launch: a staged search over execution shapes and tiles, timed on
the caller's own boxes with CUDA events, with the picks cached per program structure, batch-size
class and device.

Search space of one program:

* execution: one box per thread (64 boxes per CTA), or one box per CTA of 64, 128 or 256 threads;
* pass working set (box per CTA): shared memory, or global memory (L1/L2-cached, more CTAs per SM);
* the tensor-core fold of dense nodes on the input (on / off) -- programs with such nodes.

Stages: (1) every execution shape with the fold off; (2) the fold on the best of them. Each
candidate runs once at the full batch (module load, workspace, caches) and is then timed as the
faster of `reps` launches. A candidate that fails to build (a working set beyond shared memory,
say) is skipped. The GEMV tile of the steps through Linear/MatMul nodes is chosen by row shape in
the kernel: forcing 2 x 8, 8 x 1 or 4 x 4 was measured 8-75% slower on dense_q_n200, and reading a
runtime choice raised the kernel's spills and cost 3%, so the tile is not a tuning dimension."""
from __future__ import annotations

import hashlib
from typing import Dict, NamedTuple, Optional

import torch

from . import _lib
from .graph import Graph
from .program import Program


class Config(NamedTuple):
    mode: str = "cta"          # "cta" | "simt"
    threads: int = 128         # threads per CTA (box per CTA)
    smem_global: bool = False  # pass working set in global memory (box per CTA)
    fold_tc: bool = False      # tensor-core fold of dense nodes on the input

    def name(self):
        if self.mode == "simt":
            return "simt"
        s = f"cta{self.threads}" + ("-global" if self.smem_global else "")
        if self.fold_tc:
            s += "-tcfold"
        return s


_CACHE: Dict[tuple, dict] = {}


def structure_key(graph: Graph) -> str:
    """A hash of the compiled program's structure (records and pools), independent of the launch
    shape: programs with equal keys behave alike under every candidate."""
    p = Program(graph, mode="cta")
    h = hashlib.sha1()
    for a in (p.header[:8], p.node_arr, p.step_arr, p.pass_arr, p.op_arr, p.int_pool, p.dbl_pool):
        h.update(a.tobytes())
    return h.hexdigest()


def build(graph: Graph, cfg: Config, spec_rows=None, dense_c=False, tie_rule="reference"):
    """The program of one candidate (ProgramError when it cannot be built)."""
    kw = dict(spec_rows=spec_rows, dense_c=dense_c, tie_rule=tie_rule)
    if cfg.mode == "simt":
        return Program(graph, mode="simt", **kw)
    return Program(graph, mode="cta", cta_threads=cfg.threads, smem_limit=0 if cfg.smem_global else 232448,
                   fold_tc=cfg.fold_tc, **kw)


def _time(dag, x_L, x_U, C, out, reps):
    """Device time (ms) of one launch of an uploaded candidate: the faster of `reps` after one."""
    L = _lib.lib()
    B = x_L.shape[0]
    lb, lA, lbias = out
    ws = torch.empty(max(int(L.gear_crown_workspace_bytes(dag.handle, B)), 8), dtype=torch.uint8,
                     device=x_L.device)
    stream = torch.cuda.current_stream(x_L.device).cuda_stream

    def launch():
        _lib.check(L.gear_crown_lower(dag.handle, x_L.data_ptr(), x_U.data_ptr(), B,
                                      C.data_ptr() if C is not None else None, lb.data_ptr(), lA.data_ptr(),
                                      lbias.data_ptr(), ws.data_ptr(), ws.numel(), stream), "gear_crown_lower")
    launch()
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        launch()
        e1.record()
        torch.cuda.synchronize(x_L.device)
        t = e0.elapsed_time(e1)
        best = t if best is None else min(best, t)
    return best


def tune(graph: Graph, x_L: torch.Tensor, x_U: torch.Tensor, C: Optional[torch.Tensor] = None, spec_rows=None,
         dense_c=False, tie_rule="reference", reps: int = 2, simt_items_max: int = 65536,
         cache: Optional[dict] = None):
    """Search the candidates on these boxes; returns (best Config, {name: ms}). The result is cached
    per (program structure, batch-size class, device, tie rule, spec) in `cache` (module-wide by
    default)."""
    from .engine import _Dag
    cache = _CACHE if cache is None else cache
    B = x_L.shape[0]
    key = (structure_key(graph), max(B - 1, 0).bit_length(), torch.cuda.get_device_name(x_L.device), tie_rule,
           spec_rows, dense_c)
    if key in cache:
        return cache[key]["best"], cache[key]["ms"]
    dev = x_L.device
    probe = Program(graph, mode="cta")
    S, n = probe.S if spec_rows is None else spec_rows, probe.n
    out = (torch.empty(B, S, dtype=torch.float64, device=dev), torch.empty(B, S, n, dtype=torch.float64, device=dev),
           torch.empty(B, S, dtype=torch.float64, device=dev))
    times: Dict[Config, float] = {}

    def trial(cfg):
        if cfg in times:
            return
        try:
            prog = build(graph, cfg, spec_rows, dense_c, tie_rule)
            if cfg.mode == "simt":
                items = 3 * prog.arena_w + prog.plane_w + prog.fold_w + 4 * prog.maxw + prog.simt_buf + \
                    prog.simt_rows
                if items > simt_items_max:
                    return
            dag = _Dag.from_program(prog)
        except Exception:
            return
        times[cfg] = _time(dag, x_L, x_U, C, out, reps)

    # (1) execution shapes
    trial(Config("simt", 0))
    for t in (64, 128, 256):
        for g in (False, True):
            trial(Config("cta", t, g))
    # (2) the tensor-core fold
    best = min(times, key=times.get)
    if best.mode == "cta" and probe.fold_w > 0:
        trial(best._replace(fold_tc=True))
    best = min(times, key=times.get)
    ms = {c.name(): t for c, t in times.items()}
    cache[key] = {"best": best, "ms": ms}
    return best, ms


class TunedEngine:
    """CrownEngine's lower() with the autotuner's pick: the first call of each batch-size class
    tunes on its boxes, later calls reuse the pick (and its uploaded program)."""

    def __init__(self, graph: Graph, spec_rows: Optional[int] = None, dense_c: bool = False,
                 tie_rule: str = "reference"):
        from .engine import CrownEngine
        self.graph, self.spec_rows, self.dense_c, self.tie_rule = graph, spec_rows, dense_c, tie_rule
        self._engines: Dict[Config, "CrownEngine"] = {}
        self._pick: Dict[int, Config] = {}
        self.timings: Dict[int, dict] = {}
        e = self._engine(Config())
        self.n, self.S, self.prog, self.handle = e.n, e.S, e.prog, e.handle
        self.mode = "tune"

    def _engine(self, cfg: Config):
        from .engine import CrownEngine, _Dag
        if cfg not in self._engines:
            eng = CrownEngine.__new__(CrownEngine)
            dag = _Dag.from_program(build(self.graph, cfg, self.spec_rows, self.dense_c, self.tie_rule))
            eng.graph, eng.mode, eng.dense_c = self.graph, "fixed", self.dense_c
            eng._args = (self.graph, self.spec_rows, self.dense_c)
            eng.tie_rule, eng.fold_tc = self.tie_rule, cfg.fold_tc
            eng._dags = {(cfg.mode, cfg.threads): dag}
            eng._fixed = dag
            eng.prog, eng.handle = dag.prog, dag.handle
            eng.n, eng.S = dag.prog.n, dag.prog.S
            eng._choice, eng.timings, eng._ws = {}, {}, None
            self._engines[cfg] = eng
        return self._engines[cfg]

    @staticmethod
    def _bucket(batch):
        return max(int(batch) - 1, 0).bit_length()

    def kernel_name(self, batch: int) -> Optional[str]:
        """The CUDA kernel the pick launches for this batch size."""
        c = self.pick(batch)
        if c is None:
            return None
        if c.mode == "simt":
            return "crown_simt_kernel"
        return f"crown_megakernel<{c.threads}, {int(c.smem_global)}, {int(c.fold_tc)}>"

    def pick(self, batch: int) -> Optional[Config]:
        return self._pick.get(max(int(batch) - 1, 0).bit_length())

    def variant(self, batch: int) -> Optional[str]:
        c = self.pick(batch)
        return None if c is None else c.name()

    def lower(self, x_L, x_U, C=None, return_A=True, out=None, lb_ibp=None):
        B = x_L.shape[0]
        key = max(B - 1, 0).bit_length()
        if key not in self._pick and B > 0:
            xl = x_L.reshape(B, -1).to(torch.float64).contiguous()
            xu = x_U.reshape(B, -1).to(torch.float64).contiguous()
            best, ms = tune(self.graph, xl, xu, C, self.spec_rows, self.dense_c, self.tie_rule)
            self._pick[key] = best
            self.timings[key] = ms
        cfg = self._pick.get(key, Config())
        eng = self._engine(cfg)
        self.prog, self.handle = eng.prog, eng.handle
        return eng.lower(x_L, x_U, C, return_A=return_A, out=out, lb_ibp=lb_ibp)
