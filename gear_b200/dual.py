"""Rigorous float64 LP dual bounds on the GPU: the reference's Rows / dual_lower_bound /
certify_infeasible (``complete_verifier/nlp_solver/rigorous_dual.py``) over batched LPs
min c^T z + c0 s.t. G z <= h, l <= z <= u, evaluated by gear_dual_lower_bound."""
from __future__ import annotations

import torch

from . import _lib


class Rows:
    """G (m x n) in COO form: a pattern (row, col) shared by the batch, values val (B, nnz) or
    (1, nnz); the column-major (CSC) order the kernel walks is built once per device."""

    def __init__(self, row, col, val, m, n):
        self.row = torch.as_tensor(row).long()
        self.col = torch.as_tensor(col).long()
        self.val = val if val.dim() == 2 else val.unsqueeze(0)
        self.m, self.n = int(m), int(n)
        self._csc = {}

    @classmethod
    def from_dense(cls, G):
        B, m, n = G.shape
        row, col = (G != 0).any(0).nonzero(as_tuple=True)
        return cls(row, col, G[:, row, col], m, n)

    def csc(self, device):
        key = str(device)
        if key not in self._csc:
            order = torch.argsort(self.col, stable=True)
            cnt = torch.bincount(self.col, minlength=self.n)
            colptr = torch.zeros(self.n + 1, dtype=torch.int64)
            colptr[1:] = torch.cumsum(cnt, 0)
            self._csc[key] = (colptr.to(device=device, dtype=torch.int32).contiguous(),
                              self.row[order].to(device=device, dtype=torch.int32).contiguous(),
                              order.to(device=device, dtype=torch.int32).contiguous())
        return self._csc[key]


def _p(t):
    return None if t is None else t.data_ptr()


def _f64(t, dev):
    return None if t is None else torch.as_tensor(t).to(device=dev, dtype=torch.float64).contiguous()


def _run(rows, c, c0, h, l, u, y, tol, c_err, c0_err, infeasibility):
    dev = y.device
    if dev.type != "cuda":
        raise _lib.GearError("gear_b200 needs CUDA tensors (no CPU fallback)")
    for t in (c, c0, h, l, u, y, rows.val):
        if t is not None and t.dtype != torch.float64:
            raise TypeError("rigorous dual: every input must be float64 (the bound is exact for the data as given)")
    B = y.shape[0]
    colptr, rws, perm = rows.csc(dev)
    val = _f64(rows.val, dev)
    tol_t = None if tol is None else torch.as_tensor(tol, dtype=torch.float64, device=dev).expand(B).contiguous()
    lb = torch.empty(B, dtype=torch.float64, device=dev)
    E = torch.empty(B, dtype=torch.float64, device=dev)
    dd = torch.empty(B, dtype=torch.uint8, device=dev)
    args = [_f64(t, dev) for t in (c, c0, h, l, u, y, c_err, c0_err)]
    cc, cc0, hh, ll, uu, yy, ce, c0e = args
    st = torch.cuda.current_stream(dev).cuda_stream
    _lib.check(_lib.lib().gear_dual_lower_bound(_p(colptr), _p(rws), _p(perm), _p(val), 1 if val.shape[0] > 1 else 0,
                                                B, rows.m, rows.n, int(rows.row.numel()), _p(cc), _p(cc0), _p(hh),
                                                _p(ll), _p(uu), _p(yy), _p(tol_t), _p(ce), _p(c0e), infeasibility,
                                                _p(lb), _p(E), _p(dd), st), "gear_dual_lower_bound")
    return lb, E, dd.bool()


def dual_lower_bound(rows: Rows, c, c0, h, l, u, y, tol=None, c_err=None, c0_err=None):
    """(lb (B,), E (B,), dd (B,)): lb <= D(y) exactly on the given floats (rigorous_dual.py:202)."""
    return _run(rows, c, c0, h, l, u, y, tol, c_err, c0_err, 0)


def certify_infeasible(rows: Rows, h, l, u, y):
    """(B,) bool: y >= 0 proves {G z <= h, l <= z <= u} empty (rigorous_dual.py:225)."""
    lb, _, _ = _run(rows, None, None, h, l, u, y, None, None, None, 1)
    return lb > 0
