"""Node-program lowering: the reference's gear compile output into this package's IR.

GEAR's front end (``complete_verifier/gear/lower/emit.py:538``, ``gear/io/torch_direct.py:418``)
turns a float64 model exported with ``torch.export`` into a ``NodeProgram``: ONNX-named nodes
(``onnx::Add``, ``onnx::Gemm``, ``onnx::Slice``, ...) with static batch-1 shapes, parameters and
buffers as program inputs, and one output. ``graph_from_program`` runs that program as a torch
function (one torch op per node) under this package's tracer, so every node lands in the IR with
the same index maps as a directly traced model; the IR is then compiled for the GPU as usual.

The property side: ``parse_vnnlib_subset`` reads the converter's vnnlib subset (input box and
one-variable output rows, ``gear/spec.py:67``) into ``(lower, upper, RowSpec)``, and
``RowSpec.to_dense`` gives the C matrix of ``C y <= rhs`` for ``compute_bounds(C=...)``.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass
from typing import Dict, List, Sequence, Tuple

import numpy as np
import torch

from . import graph as _graph


class LoweringError(ValueError):
    """A node of the program is outside what the IR represents (or the program is malformed)."""


def _field(n, key):
    return n[key] if isinstance(n, dict) else getattr(n, key)


def _ints(t) -> List[int]:
    return [int(v) for v in torch.as_tensor(t).reshape(-1).tolist()]


def _slice(x, starts, ends, axes, steps):
    idx = [slice(None)] * x.dim()
    for s, e, a, st in zip(starts, ends, axes, steps):
        a = a % x.dim()
        if a == 0:
            raise LoweringError("onnx::Slice along the batch axis")
        idx[a] = slice(s, None if e >= 2 ** 62 else e, st)
    return x[tuple(idx)]


def _gather(x, index, axis):
    axis = axis % x.dim()
    if axis == 0:
        raise LoweringError("onnx::Gather along the batch axis")
    idx = [slice(None)] * axis + [index.long() if index.dim() else int(index)]
    return x[tuple(idx)]


def _gemm(attr, a, b, c=None):
    if float(attr.get("alpha", 1.0)) != 1.0 or int(attr.get("transA", 0)):
        raise LoweringError("onnx::Gemm with alpha != 1 or transA")
    W = b if int(attr.get("transB", 0)) else b.t()
    bias = None
    if c is not None:
        beta = float(attr.get("beta", 1.0))
        bias = c if beta == 1.0 else beta * c
    return torch.nn.functional.linear(a, W, bias)


def _reshape(x, shape):
    s = _ints(shape)
    s[0] = -1                        # the leading axis is the batch (the program is static at batch 1)
    return x.reshape(s)


def _cast(attr, x):
    if int(attr.get("to", 11)) != 11:
        raise LoweringError("onnx::Cast to a type other than float64")
    return x.to(torch.float64)


# ONNX op -> torch evaluation (args: the node's inputs in order; attr: its attributes)
_OPS = {
    "onnx::Add": lambda attr, a, b: a + b,
    "onnx::Sub": lambda attr, a, b: a - b,
    "onnx::Mul": lambda attr, a, b: a * b,
    "onnx::Neg": lambda attr, a: -a,
    "onnx::Pow": lambda attr, a, e: a ** float(e),
    "onnx::Exp": lambda attr, a: torch.exp(a),
    "onnx::Log": lambda attr, a: torch.log(a),
    "onnx::Sin": lambda attr, a: torch.sin(a),
    "onnx::Cos": lambda attr, a: torch.cos(a),
    "onnx::Gemm": _gemm,
    "onnx::MatMul": lambda attr, a, b: torch.matmul(a, b),
    "onnx::Transpose": lambda attr, a: a.permute(*attr.get("perm", list(range(a.dim()))[::-1])),
    "onnx::Gather": lambda attr, a, i: _gather(a, i, int(attr.get("axis", 0))),
    "onnx::Slice": lambda attr, x, s, e, a=None, st=None: _slice(
        x, _ints(s), _ints(e), _ints(a) if a is not None else list(range(len(_ints(s)))),
        _ints(st) if st is not None else [1] * len(_ints(s))),
    "onnx::Concat": lambda attr, *xs: torch.cat(list(xs), dim=int(attr.get("axis", 0))),
    "onnx::Reshape": lambda attr, x, shape: _reshape(x, shape),
    "onnx::Flatten": lambda attr, x: torch.flatten(x, int(attr.get("axis", 1))),
    "onnx::Unsqueeze": lambda attr, x, axes: _unsqueeze(x, _ints(axes)),
    "onnx::Squeeze": lambda attr, x, axes=None: _squeeze(x, None if axes is None else _ints(axes)),
    "onnx::ReduceSum": lambda attr, x, axes: torch.sum(x, dim=_ints(axes), keepdim=bool(int(attr.get("keepdims", 1)))),
    "onnx::Cast": _cast,
}


def _unsqueeze(x, axes):
    for a in sorted(a % (x.dim() + len(axes)) for a in axes):
        x = x.unsqueeze(a)
    return x


def _squeeze(x, axes):
    if axes is None:
        raise LoweringError("onnx::Squeeze without axes")
    for a in sorted((a % x.dim() for a in axes), reverse=True):
        x = x.squeeze(a)
    return x


class ProgramModule(torch.nn.Module):
    """A NodeProgram (nodes_op, nodes_in, nodes_out) as a torch module of x (batch, n)."""

    def __init__(self, nodes_op: Sequence, nodes_in: Sequence, nodes_out: Sequence[str]):
        super().__init__()
        if len(nodes_out) != 1:
            raise LoweringError("the program must have exactly one output")
        self.nodes_op = list(nodes_op)
        self.out = nodes_out[0]
        self.input_name = None
        self.consts: Dict[str, torch.Tensor] = {}
        for n in nodes_in:
            if _field(n, "model_input_index") == 0:
                if self.input_name is not None:
                    raise LoweringError("the program must have exactly one perturbed input")
                self.input_name = _field(n, "name")
            else:
                p = _field(n, "param")
                if p is None:
                    raise LoweringError(f"program input {_field(n, 'name')} has no value")
                self.consts[_field(n, "name")] = torch.as_tensor(p).detach()
        if self.input_name is None:
            raise LoweringError("the program has no model input")
        for n in self.nodes_op:
            op = _field(n, "op")
            if op != "onnx::Constant" and op not in _OPS:
                raise LoweringError(f"{op} is not supported by the IR")

    def forward(self, x):
        env = dict(self.consts)
        env[self.input_name] = x
        for n in self.nodes_op:
            op, attr = _field(n, "op"), _field(n, "attr") or {}
            if op == "onnx::Constant":
                env[_field(n, "name")] = torch.as_tensor(attr["value"])
                continue
            args = [env[i] for i in _field(n, "inputs")]
            env[_field(n, "name")] = _OPS[op](attr, *args)
        return env[self.out]


def graph_from_program(nodes_op: Sequence, nodes_in: Sequence, nodes_out: Sequence[str], n: int,
                       x0: torch.Tensor = None) -> _graph.Graph:
    """The IR of a NodeProgram whose input has n variables (x0: an example point, default 0)."""
    mod = ProgramModule(nodes_op, nodes_in, nodes_out)
    if x0 is None:
        x0 = torch.zeros(2, n, dtype=torch.float64)
    return _graph.trace(mod, x0.reshape(-1, n).to(torch.float64))


# ---------------------------------------------------------------- output rows (vnnlib subset)
@dataclass(frozen=True)
class RowSpec:
    """Output rows C y <= rhs in CSR form; C is (nrows, num_outputs)."""
    num_outputs: int
    indptr: np.ndarray
    indices: np.ndarray
    data: np.ndarray
    rhs: np.ndarray

    @property
    def nrows(self) -> int:
        return int(self.rhs.shape[0])

    def to_dense(self) -> np.ndarray:
        C = np.zeros((self.nrows, self.num_outputs), dtype=np.float64)
        r = np.repeat(np.arange(self.nrows), np.diff(self.indptr))
        C[r, self.indices] = self.data
        return C


_NUMBER = r"[+-]?(?:\d+(?:\.\d*)?|\.\d+)(?:[eE][+-]?\d+)?"
_DECLARE = re.compile(r"\(declare-const ([XY])_(0|[1-9]\d*) Real\)")
_BOUND = re.compile(r"\(assert \((<=|>=) ([XY])_(0|[1-9]\d*) (" + _NUMBER + r")\)\)")


def parse_vnnlib_subset(text: str, name: str = "<vnnlib>") -> Tuple[np.ndarray, np.ndarray, RowSpec]:
    """(lower, upper, rows) of the converter's vnnlib subset: declarations of X_i / Y_i and single
    bounds (<= or >=) on one variable per assertion. Input bounds intersect; the box is returned as
    mean -/+ half-width (the reference reader's rewrite); a ">= Y_k c" row is -Y_k <= -c. Anything
    else raises LoweringError."""
    decl = {"X": set(), "Y": set()}
    bounds = []
    for k, raw in enumerate(text.splitlines(), 1):
        line = raw.split(";", 1)[0].strip()
        if not line:
            continue
        m = _DECLARE.fullmatch(line)
        if m:
            i = int(m.group(2))
            if i in decl[m.group(1)]:
                raise LoweringError(f"{name}:{k}: {m.group(1)}_{i} declared twice")
            decl[m.group(1)].add(i)
            continue
        m = _BOUND.fullmatch(line)
        if not m:
            raise LoweringError(f"{name}:{k}: not in the supported subset: {line[:80]!r}")
        bounds.append((k, m.group(1), m.group(2), int(m.group(3)), m.group(4)))
    nx, ny = len(decl["X"]), len(decl["Y"])
    if nx == 0:
        raise LoweringError(f"{name}: no input variable")
    if decl["X"] != set(range(nx)) or decl["Y"] != set(range(ny)):
        raise LoweringError(f"{name}: variable indices are not 0..k-1")
    lo, hi = np.full(nx, -np.inf), np.full(nx, np.inf)
    cols, data, rhs = [], [], []
    for k, op, kind, i, tok in bounds:
        v = float(tok)
        if not math.isfinite(v):
            raise LoweringError(f"{name}:{k}: non-finite constant")
        if kind == "X":
            if i >= nx:
                raise LoweringError(f"{name}:{k}: X_{i} not declared")
            if op == "<=":
                hi[i] = min(hi[i], v)
            else:
                lo[i] = max(lo[i], v)
        else:
            if i >= ny:
                raise LoweringError(f"{name}:{k}: Y_{i} not declared")
            cols.append(i)
            data.append(1.0 if op == "<=" else -1.0)
            rhs.append(v if op == "<=" else -1 * v)
    if not (np.isfinite(lo).all() and np.isfinite(hi).all()):
        raise LoweringError(f"{name}: an input variable has no bound")
    if not (lo <= hi).all():
        raise LoweringError(f"{name}: an input range is empty")
    mid, half = (lo + hi) / 2, (hi - lo) / 2 * 1.0
    m = len(cols)
    spec = RowSpec(ny, np.arange(m + 1, dtype=np.int64), np.asarray(cols, dtype=np.int64),
                   np.asarray(data, dtype=np.float64), np.asarray(rhs, dtype=np.float64))
    return mid - half, mid + half, spec
