"""Drop-in surface of the reference's bound-propagation API for the CROWN hot path.

Mirrors ``auto_LiRPA``'s ``BoundedModule`` / ``BoundedTensor`` / ``PerturbationLpNorm``
(``solver/auto_LiRPA/bound_general.py:87,1275``, ``bounded_tensor.py``,
``perturbations.py:129``) for the calls the solver's bounding step makes
(``complete_verifier/input_split/bounding.py:317``):

    bm = BoundedModule(model, x0, bound_opts=..., device='cuda')
    lb, ub, A = bm.compute_bounds(x=(BoundedTensor(x0, PerturbationLpNorm(x_L=lo, x_U=hi)),),
                                  C=C, method='CROWN', bound_upper=False, return_A=True,
                                  needed_A_dict={bm.output_name[0]: {bm.input_name[0]}})
    A[bm.output_name[0]][bm.input_name[0]] == {'lA': (B, S, n), 'uA': None,
                                               'lbias': (B, S), 'ubias': None,
                                               'unstable_idx': None}

A perturbation carrying linear rows, ``PerturbationLpNorm(x_L=lo, x_U=hi, constraints=(A, b))``
with A (B, K, n) and b (B, K) meaning A x + b <= 0 (perturbations.py:129-199), makes every
concretisation of the call, the intermediate passes' included, the constrained one
(``engine.CutEngine``, C ABI ``gear_crown_lower_cuts``).

Everything runs in float64 on the GPU through ``libgear_b200.so``; there is no CPU path.
Only ``method='CROWN'`` (alias ``'backward'``) and ``'ibp'`` are accepted, with
``bound_upper=False`` for CROWN; other methods raise ``NotImplementedError`` as the
reference does for unsupported combinations.
"""
from __future__ import annotations

from typing import Dict, Optional

import torch

from . import graph as _graph
from .engine import CrownEngine

# The reference's GEAR configuration turns these on (exp_configs/NLP_solver/f3.yaml); the
# engine always behaves as if they were set: an element whose relaxation is undefined (a
# non-finite input interval, log of an interval reaching 0) stops at the node's own interval on
# its undefined sides (backward_bound.py:249-292), and only a row with a non-finite contribution
# is discarded to the output interval (backward_bound.py:826).
HOT_PATH_BOUND_OPTS = {'fp_enclosure': {'affine_backward': True}, 'compare_crown_with_ibp_intermediate': True,
                       'undefined_relaxation_rows': True, 'undefined_relaxation_interval': True}


class PerturbationLpNorm:
    """L-infinity box perturbation given by x_L / x_U (perturbations.py:129)."""

    def __init__(self, eps=0.0, norm=float("inf"), x_L=None, x_U=None, **kwargs):
        if norm != float("inf"):
            raise NotImplementedError("only the L-infinity box perturbation is on the hot path")
        self.eps = eps
        self.norm = norm
        self.x_L = x_L
        self.x_U = x_U
        self.constraints = kwargs.get("constraints")

    def bounds(self, x):
        lo = self.x_L if self.x_L is not None else x - self.eps
        hi = self.x_U if self.x_U is not None else x + self.eps
        return lo, hi


class BoundedTensor(torch.Tensor):
    """A tensor carrying its perturbation (bounded_tensor.py)."""

    @staticmethod
    def __new__(cls, x, ptb=None):
        t = torch.Tensor._make_subclass(cls, x.detach(), False)
        t.ptb = ptb
        return t

    def __init__(self, x, ptb=None):
        self.ptb = ptb


class BoundedModule:
    """CROWN bounds of a traced NLP DAG over batches of boxes on one GPU."""

    def __init__(self, model: torch.nn.Module, global_input: torch.Tensor, bound_opts: Optional[dict] = None,
                 device: str = "cuda", **kwargs):
        self.bound_opts = dict(HOT_PATH_BOUND_OPTS)
        if bound_opts:
            self.bound_opts.update(bound_opts)
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("gear_b200.BoundedModule runs on CUDA only")
        x0 = global_input if global_input.dim() == 2 else global_input.reshape(global_input.shape[0], -1)
        self.graph = _graph.trace(model, x0.detach().to("cpu", torch.float64))
        self.input_name = ["/x"]
        self.output_name = ["/y"]
        self._engines: Dict[tuple, CrownEngine] = {}
        self.model = model

    # ------------------------------------------------------------ engines
    def _engine(self, spec_rows: int, dense_c: bool) -> CrownEngine:
        key = (spec_rows, dense_c)
        eng = self._engines.get(key)
        if eng is None:
            with torch.cuda.device(self.device):
                if self.bound_opts.get("gear_mode", "auto") == "tune":
                    from .autotune import TunedEngine
                    eng = TunedEngine(self.graph, spec_rows=spec_rows, dense_c=dense_c,
                                      tie_rule=self.bound_opts.get("gear_tie_rule", "reference"))
                    self._engines[key] = eng
                    return eng
                eng = CrownEngine(self.graph, spec_rows=spec_rows, dense_c=dense_c,
                                  mode=self.bound_opts.get("gear_mode", "auto"),
                                  cta_threads=int(self.bound_opts.get("gear_cta_threads", 128)),
                                  tie_rule=self.bound_opts.get("gear_tie_rule", "reference"),
                                  fold_tc=self._fold_tc())
            self._engines[key] = eng
        return eng

    def _cut_engine(self, spec_rows: int, dense_c: bool):
        key = ("cuts", spec_rows, dense_c)
        eng = self._engines.get(key)
        if eng is None:
            from .engine import CutEngine
            with torch.cuda.device(self.device):
                eng = CutEngine(self.graph, spec_rows=spec_rows, dense_c=dense_c,
                                cta_threads=int(self.bound_opts.get("gear_cta_threads", 128)),
                                tie_rule=self.bound_opts.get("gear_tie_rule", "reference"))
            self._engines[key] = eng
        return eng

    # "auto" fold placement: dense nodes on the input with at least this many weights in all run
    # their fold products on the tensor cores (measured on B200: 30% off a dense_a_n2048 call with
    # 2 M weights, 4% on dense_q_n200's 50 k, where the fold is a small share of the kernel)
    FOLD_TC_MIN_WEIGHTS = 1 << 20

    def _fold_tc(self) -> bool:
        opt = self.bound_opts.get("gear_fold_tc", "auto")
        if opt != "auto":
            return bool(opt)
        weights = sum(nd.width * self.graph[0].width for nd in self.graph.nodes
                      if nd.kind in ("linear", "matmul") and nd.inputs and nd.inputs[0] == 0)
        return weights >= self.FOLD_TC_MIN_WEIGHTS

    def final_node_width(self) -> int:
        return self.graph[self.graph.output].width

    @staticmethod
    def _is_identity(C: torch.Tensor) -> bool:
        if C.dim() != 3 or C.shape[1] != C.shape[2]:
            return False
        eye = torch.eye(C.shape[1], dtype=C.dtype, device=C.device)
        return bool(torch.equal(C, eye.expand_as(C)))

    # ------------------------------------------------------------ API
    def compute_bounds(self, x=None, C=None, method="CROWN", bound_lower=True, bound_upper=True,
                       return_A=False, needed_A_dict=None, **kwargs):
        if x is None:
            raise ValueError("x is required")
        if isinstance(x, torch.Tensor):
            x = (x,)
        xt = x[0]
        ptb = getattr(xt, "ptb", None)
        if ptb is None:
            raise ValueError("the input must be a BoundedTensor with a PerturbationLpNorm")
        cons = getattr(ptb, "constraints", None)
        lo, hi = ptb.bounds(xt)
        B = lo.shape[0]
        lo = lo.reshape(B, -1).to(self.device, torch.float64)
        hi = hi.reshape(B, -1).to(self.device, torch.float64)
        m = method.lower()
        if m == "ibp":
            raise NotImplementedError("use ibp_bounds() for the interval pre-pass")
        if m not in ("crown", "backward"):
            raise NotImplementedError(f"method {method!r} is not on the GPU hot path")
        if bound_upper or not bound_lower:
            raise NotImplementedError("the final pass computes lower bounds (bound_upper=False)")
        w = self.final_node_width()
        if C is None or self._is_identity(C.to(self.device)):
            eng = self._engine(w, False) if cons is None else None
            Cd = None
        else:
            C = C.to(self.device, torch.float64)
            eng = self._engine(int(C.shape[1]), True) if cons is None else None
            Cd = C
        want_A = bool(return_A)
        if cons is not None:
            # every concretisation over box ∩ rows A x + b <= 0 (PerturbationLpNorm(constraints=
            # (A, b)), perturbations.py:129-199; rows in standard form, (B, K, n) and (B, K))
            ceng = self._cut_engine(int(C.shape[1]) if Cd is not None else w, Cd is not None)
            cA, cb = cons
            lb, lA, lbias = ceng.lower(lo, hi, cA.to(self.device, torch.float64), cb.to(self.device, torch.float64),
                                       Cd, max_rows=int(self.bound_opts.get("concretize_max_constraint_rows", 0)))
        else:
            lb, lA, lbias = eng.lower(lo, hi, Cd, return_A=want_A)
        if not return_A:
            return lb, None
        A = {self.output_name[0]: {self.input_name[0]: {
            "lA": lA, "uA": None, "lbias": lbias, "ubias": None, "unstable_idx": None}}}
        return lb, None, A

    def compute_bounds_host(self, x_L: torch.Tensor, x_U: torch.Tensor, chunk: int = 16384):
        """CROWN lower bounds (identity specification) of boxes held in HOST memory, with the
        copies overlapped with the kernels: chunks of `chunk` boxes go host -> device on one
        stream, are bounded on the current stream and their lb rows come back on a third, through
        two device buffers. Returns lb (B, S) in pinned host memory, complete once the current
        stream has been synchronised. Pinned inputs make the copies asynchronous."""
        B = x_L.shape[0]
        n = self.graph[0].width
        x_L = x_L.reshape(B, n)
        x_U = x_U.reshape(B, n)
        w = self.final_node_width()
        eng = self._engine(w, False)
        dev = self.device
        lb_h = torch.empty(B, w, dtype=torch.float64, pin_memory=True)
        if B == 0:
            return lb_h
        chunk = max(1, min(int(chunk), B))
        cur = torch.cuda.current_stream(dev)
        if getattr(self, "_copy_streams", None) is None or self._copy_streams[0].device != dev:
            self._copy_streams = (torch.cuda.Stream(dev), torch.cuda.Stream(dev))
        s_in, s_out = self._copy_streams
        key = (chunk, n, w)
        if getattr(self, "_host_bufs", None) is None or self._host_bufs[0] != key:
            self._host_bufs = (key, [dict(L=torch.empty(chunk, n, dtype=torch.float64, device=dev),
                                          U=torch.empty(chunk, n, dtype=torch.float64, device=dev),
                                          lb=torch.empty(chunk, w, dtype=torch.float64, device=dev),
                                          lA=torch.empty(chunk, w, n, dtype=torch.float64, device=dev),
                                          lbias=torch.empty(chunk, w, dtype=torch.float64, device=dev))
                                     for _ in range(2)])
        bufs = self._host_bufs[1]
        ins, done, outs = [], [], []
        s_in.wait_stream(cur)
        s_out.wait_stream(cur)
        for k, a in enumerate(range(0, B, chunk)):
            b = min(a + chunk, B)
            m = b - a
            buf = bufs[k % 2]
            with torch.cuda.stream(s_in):
                if k >= 2:
                    s_in.wait_event(done[k - 2])          # the kernel of chunk k-2 has read this buffer
                buf["L"][:m].copy_(x_L[a:b], non_blocking=True)
                buf["U"][:m].copy_(x_U[a:b], non_blocking=True)
                ins.append(torch.cuda.Event())
                ins[-1].record(s_in)
            cur.wait_event(ins[k])
            if k >= 2:
                cur.wait_event(outs[k - 2])               # chunk k-2's lb rows have left this buffer
            eng.lower(buf["L"][:m], buf["U"][:m], None, out=(buf["lb"][:m], buf["lA"][:m], buf["lbias"][:m]))
            done.append(torch.cuda.Event())
            done[-1].record(cur)
            with torch.cuda.stream(s_out):
                s_out.wait_event(done[k])
                lb_h[a:b].copy_(buf["lb"][:m], non_blocking=True)
                outs.append(torch.cuda.Event())
                outs[-1].record(s_out)
        cur.wait_stream(s_out)
        cur.wait_stream(s_in)
        return lb_h

    __call__ = compute_bounds
