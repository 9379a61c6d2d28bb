"""Device engine: a compiled program on the GPU and the launch of the CROWN megakernel."""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _lib
from .graph import Graph
from .program import Program


class CrownEngine:
    """One graph and one specification kind (identity or dense C) on the current device."""

    def __init__(self, graph: Graph, spec_rows: Optional[int] = None, dense_c: bool = False, mode: str = "cta"):
        """mode: "cta" (one box per CTA) or "simt" (one box per thread); both give the same bounds."""
        if not torch.cuda.is_available():
            raise _lib.GearError("gear_b200 needs a CUDA device (no CPU fallback)")
        self.graph = graph
        self.mode = mode
        self.prog = Program(graph, spec_rows=spec_rows, dense_c=dense_c, mode=mode)
        p = self.prog
        L = _lib.lib()
        h = ctypes.c_void_p()
        arrs = [np.ascontiguousarray(a, dtype=np.int32) for a in
                (p.header, p.node_arr, p.step_arr, p.pass_arr, p.op_arr, p.int_pool)]
        dbl = np.ascontiguousarray(p.dbl_pool, dtype=np.float64)
        self._keep = (arrs, dbl)
        st = L.gear_dag_create(_lib.ptr_i32(arrs[0]), arrs[0].size, _lib.ptr_i32(arrs[1]), arrs[1].size,
                               _lib.ptr_i32(arrs[2]), arrs[2].size, _lib.ptr_i32(arrs[3]), arrs[3].size,
                               _lib.ptr_i32(arrs[4]), arrs[4].size, _lib.ptr_i32(arrs[5]), arrs[5].size,
                               _lib.ptr_dbl(dbl), dbl.size, ctypes.byref(h))
        _lib.check(st, "gear_dag_create")
        self.handle = h
        self.n = p.n
        self.S = p.S
        self.dense_c = dense_c
        self._ws = None

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().gear_dag_destroy(h)
            except Exception:
                pass
            self.handle = None

    def workspace(self, batch: int, device) -> torch.Tensor:
        nbytes = int(_lib.lib().gear_crown_workspace_bytes(self.handle, batch))
        if self._ws is None or self._ws.numel() < nbytes or self._ws.device != device:
            self._ws = torch.empty(max(nbytes, 8), dtype=torch.uint8, device=device)
        return self._ws

    def lower(self, x_L: torch.Tensor, x_U: torch.Tensor, C: Optional[torch.Tensor] = None,
              return_A: bool = True, out=None):
        """lb (B, S), lA (B, S, n) or None, lbias (B, S) -- all float64 on x_L's device."""
        B = x_L.shape[0]
        dev = x_L.device
        if dev.type != "cuda":
            raise _lib.GearError("inputs must be CUDA tensors")
        x_L = x_L.reshape(B, -1).to(torch.float64).contiguous()
        x_U = x_U.reshape(B, -1).to(torch.float64).contiguous()
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
        ws = self.workspace(B, dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        st = _lib.lib().gear_crown_lower(self.handle, x_L.data_ptr(), x_U.data_ptr(), B,
                                         C.data_ptr() if self.dense_c else None,
                                         lb.data_ptr(), lA.data_ptr(),
                                         lbias.data_ptr(), ws.data_ptr(), ws.numel(), stream)
        _lib.check(st, "gear_crown_lower")
        return lb, (lA if return_A else None), lbias
