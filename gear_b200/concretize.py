"""Constrained concretisation on the GPU: bounds of linear objectives over boxes intersected
with linear rows (the reference's sort_out_constr_batches + constraints_solving,
``auto_LiRPA/concretize_func.py:312-850``, as one device call)."""
from __future__ import annotations

import math
from typing import Optional, Tuple

import torch

from . import _lib


def constraints_solving(x_L: torch.Tensor, x_U: torch.Tensor, objective: torch.Tensor,
                        constraints: Optional[Tuple[torch.Tensor, torch.Tensor]], sign: float = -1.0,
                        max_rows: Optional[int] = None, return_infeasible: bool = False):
    """Bounds (B, H, 1) of objective (B, H, n) . x over {x_L <= x <= x_U, A x + b <= 0}.

    constraints = (A (B, K, n), b (B, K)) in the reference's standard form
    (construct_constraints). sign -1: lower bounds (+inf for a box the rows exclude);
    sign +1: upper bounds (-inf there). max_rows caps the rows each box sweeps
    (the reference's MAX_CONSTRAINT_ROWS / concretize_max_constraint_rows)."""
    if x_L.device.type != "cuda":
        raise _lib.GearError("gear_b200 needs CUDA tensors (no CPU fallback)")
    B = x_L.shape[0]
    dev = x_L.device
    xL = x_L.reshape(B, -1).to(torch.float64).contiguous()
    xU = x_U.reshape(B, -1).to(torch.float64).contiguous()
    n = xL.shape[1]
    obj = objective.to(torch.float64)
    if obj.dim() == 2:
        obj = obj.unsqueeze(0)
    obj = obj.expand(B, -1, -1) if obj.shape[0] == 1 else obj
    if sign == 1.0:
        obj = -obj
    obj = obj.contiguous()
    H = obj.shape[1]
    if constraints is None or constraints[0] is None or constraints[0].numel() == 0:
        A = b = None
        K = 0
    else:
        A = constraints[0].reshape(B, -1, n).to(torch.float64).contiguous()
        b = constraints[1].reshape(B, -1).to(torch.float64).contiguous()
        K = A.shape[1]
    lb = torch.empty(B, H, dtype=torch.float64, device=dev)
    infeasible = torch.empty(B, dtype=torch.uint8, device=dev)
    L = _lib.lib()
    nbytes = int(L.gear_constrained_workspace_bytes(B, K))
    ws = torch.empty(max(nbytes, 8), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = L.gear_constrained_lower(xL.data_ptr(), xU.data_ptr(), B, n, obj.data_ptr(), H,
                                  A.data_ptr() if K else None, b.data_ptr() if K else None, K,
                                  int(max_rows or 0), lb.data_ptr(), infeasible.data_ptr(), ws.data_ptr(),
                                  ws.numel(), stream)
    _lib.check(st, "gear_constrained_lower")
    out = (-lb if sign == 1.0 else lb).unsqueeze(-1)
    if return_infeasible:
        return out, infeasible.bool()
    return out
