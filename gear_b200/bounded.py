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
# engine always behaves as if they were set.
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
                eng = CrownEngine(self.graph, spec_rows=spec_rows, dense_c=dense_c,
                                  mode=self.bound_opts.get("gear_mode", "auto"),
                                  cta_threads=int(self.bound_opts.get("gear_cta_threads", 128)))
            self._engines[key] = eng
        return eng

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
        if getattr(ptb, "constraints", None) is not None:
            raise NotImplementedError("constrained concretisation is not on the GPU path yet")
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
            eng = self._engine(w, False)
            Cd = None
        else:
            C = C.to(self.device, torch.float64)
            eng = self._engine(int(C.shape[1]), True)
            Cd = C
        want_A = bool(return_A)
        lb, lA, lbias = eng.lower(lo, hi, Cd, return_A=want_A)
        if not return_A:
            return lb, None
        A = {self.output_name[0]: {self.input_name[0]: {
            "lA": lA, "uA": None, "lbias": lbias, "ubias": None, "unstable_idx": None}}}
        return lb, None, A

    __call__ = compute_bounds
