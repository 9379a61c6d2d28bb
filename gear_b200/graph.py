"""Expression-DAG IR for the bound-propagation hot path, and a tracer that builds it
from a ``torch.nn.Module``.

The reference builds its DAG by exporting the module through ONNX and wrapping every
ONNX node in a ``Bound*`` operator (``auto_LiRPA/bound_general.py:803-1001``,
``auto_LiRPA/parse_graph.py:295``), then rewrites it (``auto_LiRPA/optimize_graph.py:34``).
CROWN bounds depend on that structure (which products are one node, which constants are
merged), so the IR mirrors the reference's node granularity:

* one IR node per perturbed ``Bound*`` node, with the reference operator name in ``kind``;
* constants are attributes (the reference keeps them as unperturbed ``BoundConstant``
  nodes whose backward contribution is ``A @ value``, ``backward_bound.py:1604``);
* every per-box shape is flattened row-major; shape-only operators (Slice, Gather,
  Unsqueeze, Reshape, Concat, broadcasting) carry explicit element index maps.

The rewrites mirrored from ``optimize_graph.py:34-66``: ``merge_identical_gather``
(``:470``), ``merge_common_subexpressions`` (``:529``), ``merge_identical_act`` (``:573``),
``convert_sqr`` (``:124``, Mul(x, x) and Pow(x, 2) become Sqr; the new node is not merged
by the second CSE pass because it has no forward value there) and dead-node removal.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch
from torch.overrides import TorchFunctionMode

# Operator kinds (names follow the reference's Bound* classes).
UNARY_RELAX = ("sqr", "exp", "log", "sin", "cos", "pow")
# kind -> (ibp_intermediate flag of the reference class, requires_input_bounds)
#   ibp_intermediate: operators/base.py:210 default False; set True by Slice/Concat
#   (slice_concat.py:30,156), Neg (linear.py:1176), Transpose (reshape.py:440),
#   Sin/Cos (trigonometric.py:33, s_shaped.py:39); Pow resets it to False (s_shaped.py:590).
KIND_FLAGS = {
    "input": (False, ()),
    "linear": (False, ()),
    "matmul": (False, ()),
    "mul": (False, (0, 1)),
    "mulc": (False, ()),
    "add": (False, ()),
    "sub": (False, ()),
    "addc": (False, ()),
    "subc": (False, ()),
    "rsubc": (False, ()),
    "neg": (True, ()),
    "sqr": (False, (0,)),
    "exp": (False, (0,)),
    "log": (False, (0,)),
    "sin": (True, (0,)),
    "cos": (True, (0,)),
    "pow": (False, (0,)),
    "reducesum": (False, ()),
    "gather": (False, ()),
    "slice": (True, ()),
    "concat": (True, ()),
    "reshape": (False, ()),
    "unsqueeze": (False, ()),
    "squeeze": (False, ()),
    "flatten": (False, ()),
    "transpose": (True, ()),
}
CONSTRAINT_KINDS = ("exp", "pow")
# Shape-only operators: out[j] = in[map[j]].
MAP_KINDS = ("gather", "slice", "reshape", "unsqueeze", "squeeze", "flatten", "transpose")


class GraphError(ValueError):
    """The module uses an operator or a form outside the supported set."""


@dataclass
class Node:
    id: int
    kind: str
    inputs: List[int]
    shape: Tuple[int, ...]
    attrs: Dict[str, object] = field(default_factory=dict)
    from_rewrite: bool = False

    @property
    def width(self) -> int:
        return int(np.prod(self.shape)) if len(self.shape) else 1

    @property
    def ibp_intermediate(self) -> bool:
        return KIND_FLAGS[self.kind][0]

    @property
    def requires_input_bounds(self) -> Tuple[int, ...]:
        return KIND_FLAGS[self.kind][1]

    @property
    def has_constraint(self) -> bool:
        """Exp and Pow register as layers with a constraint (convex_concave.py:409,
        s_shaped.py:591; edit_graph.py:42): every consumer then asks for their bounds."""
        return self.kind in CONSTRAINT_KINDS

    def __repr__(self):
        return f"Node({self.id}:{self.kind} in={self.inputs} shape={self.shape})"


class Graph:
    """A DAG of perturbed nodes; node 0 is the input, ``output`` the final node."""

    def __init__(self):
        self.nodes: List[Node] = []
        self.output: int = -1

    def add(self, kind, inputs, shape, from_rewrite=False, **attrs) -> int:
        if kind not in KIND_FLAGS:
            raise GraphError(f"unsupported operator kind {kind}")
        nid = len(self.nodes)
        self.nodes.append(Node(nid, kind, list(inputs), tuple(int(s) for s in shape),
                               dict(attrs), from_rewrite))
        return nid

    def __getitem__(self, i) -> Node:
        return self.nodes[i]

    def __len__(self):
        return len(self.nodes)

    @property
    def n_inputs(self) -> int:
        return self.nodes[0].width

    def consumers(self) -> Dict[int, List[int]]:
        out = {n.id: [] for n in self.nodes}
        for n in self.nodes:
            for i in n.inputs:
                out[i].append(n.id)
        return out

    def summary(self) -> str:
        return "\n".join(repr(n) for n in self.nodes)

    # ------------------------------------------------------------------ rewrites
    def _replace(self, old: int, new: int):
        for n in self.nodes:
            n.inputs = [new if i == old else i for i in n.inputs]
        if self.output == old:
            self.output = new

    def _topo_from_output(self) -> List[int]:
        order, seen = [], set()
        stack = [(self.output, False)]
        while stack:
            nid, done = stack.pop()
            if done:
                order.append(nid)
                continue
            if nid in seen:
                continue
            seen.add(nid)
            stack.append((nid, True))
            for i in self.nodes[nid].inputs:
                if i not in seen:
                    stack.append((i, False))
        return order

    @staticmethod
    def _attr_key(attrs):
        key = []
        for k in sorted(attrs):
            v = attrs[k]
            if isinstance(v, np.ndarray):
                key.append((k, str(v.dtype), v.shape, v.tobytes()))
            elif isinstance(v, (list, tuple)):
                key.append((k, tuple(v)))
            else:
                key.append((k, repr(v)))
        return tuple(key)

    def optimize(self):
        """Mirror of the default rewrites in ``optimize_graph.py:34-66``."""
        # merge_identical_gather (optimize_graph.py:470): same input, same constant index.
        seen = {}
        for n in list(self.nodes):
            if n.kind != "gather" or n.id not in self._alive():
                continue
            key = (n.inputs[0], n.attrs["axis"], n.attrs["index"].tobytes(), n.attrs["index"].shape)
            if key in seen:
                self._replace(n.id, seen[key])
            else:
                seen[key] = n.id
        self._cse()
        # merge_identical_act (optimize_graph.py:573): single-input activations only
        # (Pow has a second, exponent input in the reference and is not merged).
        alive = self._alive()
        acts = [n for n in self.nodes if n.id in alive and n.kind in ("sqr", "exp", "log", "sin", "cos")]
        merged = set()
        for i, a in enumerate(acts):
            if a.id in merged:
                continue
            for b in acts[i + 1:]:
                if b.id not in merged and b.kind == a.kind and b.inputs[0] == a.inputs[0]:
                    self._replace(b.id, a.id)
                    merged.add(b.id)
        # convert_sqr (optimize_graph.py:124): Mul(x, x) and Pow(x, 2) -> Sqr (a new node).
        for n in list(self.nodes):
            if n.id not in self._alive():
                continue
            if (n.kind == "mul" and n.inputs[0] == n.inputs[1]) or (
                    n.kind == "pow" and float(n.attrs["exponent"]) == 2.0):
                new = self.add("sqr", [n.inputs[0]], n.shape, from_rewrite=True)
                self._replace(n.id, new)
        self._cse()
        self._compact()

    def _alive(self):
        return set(self._topo_from_output())

    def _cse(self):
        canon = {}
        for nid in self._topo_from_output():
            n = self.nodes[nid]
            if n.kind == "input" or n.from_rewrite:
                continue
            key = (n.kind, tuple(n.inputs), self._attr_key(n.attrs), n.shape)
            other = canon.get(key)
            if other is None or other == nid:
                canon[key] = nid
                continue
            self._replace(nid, other)

    def _compact(self):
        """Drop dead nodes and renumber in a topological order that keeps node 0 = input.

        The order follows the reference's node list order (creation order, rewritten
        nodes appended), restricted to the live set."""
        alive = self._alive()
        alive.add(0)
        keep = [n for n in self.nodes if n.id in alive]
        # creation order is topological for traced nodes; rewritten nodes are appended
        # after their consumers, so re-sort topologically (stable w.r.t. creation order).
        order, placed = [], set()
        pending = list(keep)
        while pending:
            progressed = False
            rest = []
            for n in pending:
                if all(i in placed for i in n.inputs):
                    order.append(n)
                    placed.add(n.id)
                    progressed = True
                else:
                    rest.append(n)
            pending = rest
            if not progressed:
                raise GraphError("cycle in graph")
        remap = {n.id: k for k, n in enumerate(order)}
        for n in order:
            n.inputs = [remap[i] for i in n.inputs]
            n.id = remap[n.id]
        self.output = remap[self.output]
        self.nodes = order

    # ------------------------------------------------------------------ evaluation
    def forward_numpy(self, x: np.ndarray) -> np.ndarray:
        """Evaluate the DAG on points x (P, n) in float64; returns (P, w_out)."""
        vals = {}
        P = x.shape[0]
        for n in self.nodes:
            k = n.kind
            if k == "input":
                v = x.reshape(P, -1).astype(np.float64)
            else:
                ins = [vals[i] for i in n.inputs]
                v = eval_node(n, ins)
            vals[n.id] = v
        return vals[self.output]


def eval_node(n: Node, ins: List[np.ndarray]) -> np.ndarray:
    """Point evaluation of one node on flattened per-box values (P, w)."""
    k, a = n.kind, n.attrs
    if k == "linear":
        out = ins[0] @ a["W"].T
        if a.get("b") is not None:
            out = out + a["b"]
        return out
    if k == "matmul":
        return ins[0] @ a["W"]
    if k == "mul":
        return ins[0][:, a["map0"]] * ins[1][:, a["map1"]]
    if k == "mulc":
        return ins[0][:, a["map0"]] * a["c"]
    if k == "add":
        return ins[0][:, a["map0"]] + ins[1][:, a["map1"]]
    if k == "sub":
        return ins[0][:, a["map0"]] - ins[1][:, a["map1"]]
    if k == "addc":
        return ins[0][:, a["map0"]] + a["c"]
    if k == "subc":
        return ins[0][:, a["map0"]] - a["c"]
    if k == "rsubc":
        return a["c"] - ins[0][:, a["map0"]]
    if k == "neg":
        return -ins[0]
    if k == "sqr":
        return ins[0] ** 2
    if k == "exp":
        return np.exp(ins[0])
    if k == "log":
        with np.errstate(divide="ignore", invalid="ignore"):
            return np.log(ins[0])
    if k == "sin":
        return np.sin(ins[0])
    if k == "cos":
        return np.cos(ins[0])
    if k == "pow":
        return np.power(ins[0], a["exponent"])
    if k == "reducesum":
        out = np.zeros((ins[0].shape[0], n.width))
        np.add.at(out.T, a["rmap"], ins[0].T)
        return out
    if k in MAP_KINDS:
        return ins[0][:, a["map"]]
    if k == "concat":
        return np.concatenate([ins[j][:, :] for j in range(len(ins))], axis=1)[:, a["cmap"]]
    raise GraphError(k)


# ---------------------------------------------------------------------- tracing
class _Tracked:
    __slots__ = ("nid", "tensor")

    def __init__(self, nid, tensor):
        self.nid, self.tensor = nid, tensor


_F = torch.nn.functional


def _is_tensor(v):
    return isinstance(v, torch.Tensor)


class _TraceMode(TorchFunctionMode):
    """Records every torch call that touches a tensor derived from the input."""

    def __init__(self, graph: Graph, batch: int):
        super().__init__()
        self.g = graph
        self.B = batch
        self.track: Dict[int, _Tracked] = {}
        self.keep = []

    # -- helpers
    def nid(self, t):
        if _is_tensor(t):
            tr = self.track.get(id(t))
            if tr is not None and tr.tensor is t:
                return tr.nid
        return None

    def register(self, t, nid):
        self.track[id(t)] = _Tracked(nid, t)
        self.keep.append(t)

    def per_box_shape(self, t):
        if t.dim() == 0 or t.shape[0] != self.B:
            raise GraphError("a perturbed value lost its batch dimension")
        return tuple(t.shape[1:])

    def bmap(self, src_shape_full, out_full, is_node):
        """Element map of a broadcast operand into the per-box output."""
        if is_node:
            w = int(np.prod(src_shape_full[1:])) if len(src_shape_full) > 1 else 1
            ar = np.arange(w).reshape((1,) + tuple(src_shape_full[1:]))
        else:
            w = int(np.prod(src_shape_full)) if len(src_shape_full) else 1
            ar = np.arange(w).reshape(tuple(src_shape_full)) if len(src_shape_full) else np.array(0)
        full = np.broadcast_to(ar, out_full)
        if is_node:
            return np.ascontiguousarray(full[0].reshape(-1)).astype(np.int64)
        if full.shape[0] != 1 and len(src_shape_full) == len(out_full) and src_shape_full[0] != 1:
            raise GraphError("a constant operand varies along the batch dimension")
        return np.ascontiguousarray(full[0].reshape(-1)).astype(np.int64)

    def const_values(self, c, out_full):
        arr = c.detach().to(torch.float64).cpu().numpy() if _is_tensor(c) else np.asarray(c, dtype=np.float64)
        full = np.broadcast_to(arr, out_full)
        return np.ascontiguousarray(full[0].reshape(-1)).astype(np.float64)

    def binary(self, kind, a, b, out):
        na, nb = self.nid(a), self.nid(b)
        out_full = tuple(out.shape)
        shape = self.per_box_shape(out)
        if na is not None and nb is not None:
            m0 = self.bmap(tuple(a.shape), out_full, True)
            m1 = self.bmap(tuple(b.shape), out_full, True)
            return self.g.add(kind, [na, nb], shape, map0=m0, map1=m1)
        node, const, node_first = (na, b, True) if na is not None else (nb, a, False)
        src = a if node_first else b
        m0 = self.bmap(tuple(src.shape), out_full, True)
        c = self.const_values(const, out_full)
        if kind == "mul":
            return self.g.add("mulc", [node], shape, map0=m0, c=c, node_first=node_first)
        if kind == "add":
            return self.g.add("addc", [node], shape, map0=m0, c=c, node_first=node_first)
        if kind == "sub":
            return self.g.add("subc" if node_first else "rsubc", [node], shape, map0=m0, c=c)
        raise GraphError(kind)

    def index_map(self, x, fn):
        """Apply a shape-only function to an index tensor shaped like x."""
        w = int(np.prod(x.shape[1:])) if x.dim() > 1 else 1
        ar = torch.arange(w, dtype=torch.int64).reshape((1,) + tuple(x.shape[1:]))
        ar = ar.expand((self.B,) + tuple(x.shape[1:]))
        res = fn(ar)
        if res.dim() == 0 or res.shape[0] != self.B:
            raise GraphError("shape operator changed the batch dimension")
        return res[0].reshape(-1).numpy().astype(np.int64), tuple(res.shape[1:])

    # -- dispatcher
    def __torch_function__(self, func, types, args=(), kwargs=None):
        kwargs = kwargs or {}
        out = func(*args, **kwargs)
        flat = list(args) + list(kwargs.values())
        ins = []
        for a in flat:
            if isinstance(a, (list, tuple)):
                ins += [self.nid(t) for t in a]
            else:
                ins.append(self.nid(a))
        if all(i is None for i in ins):
            return out
        nid = self.handle(func, args, kwargs, out)
        if nid is not None:
            self.register(out, nid)
        return out

    def handle(self, func, args, kwargs, out):
        T = torch.Tensor
        name = getattr(func, "__name__", str(func))
        g = self.g
        if not _is_tensor(out):
            # size(), dim(), shape, etc.
            return None
        if func in (T.__mul__, T.__rmul__, torch.mul, T.mul):
            a, b = args[0], args[1]
            if func is T.__rmul__:
                a, b = b, a
            return self.binary("mul", a, b, out)
        if func in (T.__add__, T.__radd__, torch.add, T.add):
            if kwargs.get("alpha", 1) != 1:
                raise GraphError("add with alpha")
            a, b = args[0], args[1]
            if func is T.__radd__:
                a, b = b, a
            return self.binary("add", a, b, out)
        if func in (T.__sub__, torch.sub, T.sub):
            return self.binary("sub", args[0], args[1], out)
        if func is T.__rsub__:
            return self.binary("sub", args[1], args[0], out)
        if func in (T.__truediv__, torch.div, T.div):
            a, b = args[0], args[1]
            if self.nid(b) is not None:
                raise GraphError("division by a perturbed value (reciprocal) is not supported")
            recip = 1.0 / (b.detach().to(torch.float64) if _is_tensor(b) else torch.tensor(float(b), dtype=torch.float64))
            return self.binary("mul", a, recip, out)
        if func in (T.__neg__, torch.neg, T.neg):
            return g.add("neg", [self.nid(args[0])], self.per_box_shape(out))
        if func in (torch.exp, T.exp):
            return g.add("exp", [self.nid(args[0])], self.per_box_shape(out))
        if func in (torch.log, T.log):
            return g.add("log", [self.nid(args[0])], self.per_box_shape(out))
        if func in (torch.sin, T.sin):
            return g.add("sin", [self.nid(args[0])], self.per_box_shape(out))
        if func in (torch.cos, T.cos):
            return g.add("cos", [self.nid(args[0])], self.per_box_shape(out))
        if func in (torch.square, T.square):
            return g.add("pow", [self.nid(args[0])], self.per_box_shape(out), exponent=2.0)
        if func in (T.__pow__, torch.pow, T.pow):
            if self.nid(args[1]) is not None if len(args) > 1 else False:
                raise GraphError("variable exponent")
            p = args[1]
            p = float(p.item()) if _is_tensor(p) else float(p)
            if p == 1.0:
                return self.nid(args[0])             # x ** 1 is x (BoundPow passes A through)
            if not (p > 0) or math.isinf(p):
                raise GraphError(f"pow with exponent {p}: only positive finite exponents are supported")
            return g.add("pow", [self.nid(args[0])], self.per_box_shape(out), exponent=p)
        if func in (T.sum, torch.sum):
            x = args[0]
            dim = kwargs.get("dim", args[1] if len(args) > 1 else None)
            keepdim = kwargs.get("keepdim", args[2] if len(args) > 2 else False)
            if dim is None:
                raise GraphError("sum over the batch dimension")
            dims = [dim] if isinstance(dim, int) else list(dim)
            dims = [d % x.dim() for d in dims]
            if 0 in dims:
                raise GraphError("sum over the batch dimension")
            in_shape = tuple(x.shape[1:])
            out_keep = tuple(1 if (i + 1) in dims else s for i, s in enumerate(in_shape))
            wo = int(np.prod(out_keep)) if out_keep else 1
            rmap = np.broadcast_to(np.arange(wo).reshape(out_keep), in_shape).reshape(-1).astype(np.int64)
            return g.add("reducesum", [self.nid(x)], self.per_box_shape(out), rmap=np.ascontiguousarray(rmap),
                         keepdim=bool(keepdim))
        if func is T.__getitem__:
            x, idx = args[0], args[1]
            kind = self.getitem_kind(idx)
            m, shape = self.index_map(x, lambda ar: ar[idx])
            if kind == "gather":
                return g.add("gather", [self.nid(x)], shape, map=m, axis=1, index=m.copy())
            return g.add("slice", [self.nid(x)], shape, map=m)
        if func in (T.reshape, torch.reshape, T.view):
            x = args[0]
            rest = args[1:]
            m, shape = self.index_map(x, lambda ar: func(ar, *rest, **kwargs))
            return g.add("reshape", [self.nid(x)], shape, map=m)
        if func in (T.flatten, torch.flatten):
            x = args[0]
            m, shape = self.index_map(x, lambda ar: func(ar, *args[1:], **kwargs))
            return g.add("flatten", [self.nid(x)], shape, map=m)
        if func in (T.unsqueeze, torch.unsqueeze):
            x = args[0]
            m, shape = self.index_map(x, lambda ar: func(ar, *args[1:], **kwargs))
            return g.add("unsqueeze", [self.nid(x)], shape, map=m)
        if func in (T.squeeze, torch.squeeze):
            x = args[0]
            m, shape = self.index_map(x, lambda ar: func(ar, *args[1:], **kwargs))
            return g.add("squeeze", [self.nid(x)], shape, map=m)
        if func in (torch.cat, torch.concat, torch.concatenate):
            tensors = list(args[0])
            dim = kwargs.get("dim", args[1] if len(args) > 1 else 0) % out.dim()
            if dim == 0:
                raise GraphError("concatenation along the batch dimension")
            nodes, pieces, offset = [], [], 0
            for t in tensors:
                nid = self.nid(t)
                if nid is None:
                    raise GraphError("concatenation with a constant is not supported")
                nodes.append(nid)
                w = int(np.prod(t.shape[1:]))
                pieces.append(torch.arange(offset, offset + w, dtype=torch.int64).reshape((1,) + tuple(t.shape[1:])))
                offset += w
            cm = torch.cat(pieces, dim=dim)[0].reshape(-1).numpy().astype(np.int64)
            return g.add("concat", nodes, self.per_box_shape(out), cmap=cm, axis=dim)
        if func in (torch.matmul, T.__matmul__, T.matmul):
            a, b = args[0], args[1]
            if self.nid(b) is not None or a.dim() != 2 or b.dim() != 2:
                raise GraphError("matmul must be (perturbed batch x n) @ (constant n x m)")
            W = b.detach().to(torch.float64).cpu().numpy()
            return g.add("matmul", [self.nid(a)], self.per_box_shape(out), W=np.ascontiguousarray(W))
        if func is _F.linear:
            x, W = args[0], args[1]
            b = kwargs.get("bias", args[2] if len(args) > 2 else None)
            if self.nid(W) is not None or (b is not None and self.nid(b) is not None) or x.dim() != 2:
                raise GraphError("linear must have a constant weight and a 2-D input")
            Wn = W.detach().to(torch.float64).cpu().numpy()
            if b is None:
                # exported as MatMul(x, Transpose(W)) (no Gemm without a bias)
                return g.add("matmul", [self.nid(x)], self.per_box_shape(out), W=np.ascontiguousarray(Wn.T))
            bn = b.detach().to(torch.float64).cpu().numpy()
            return g.add("linear", [self.nid(x)], self.per_box_shape(out), W=np.ascontiguousarray(Wn), b=bn)
        if name in ("__get__",) or func in (T.size, T.dim):
            return None
        if func in (T.contiguous, T.clone, T.detach):
            self.register(out, self.nid(args[0]))
            return None
        if func in (T.to, T.double, T.float):
            if out.dtype != torch.float64:
                raise GraphError("perturbed values must stay float64")
            self.register(out, self.nid(args[0]))
            return None
        raise GraphError(f"operator {name} on a perturbed value is not supported")

    @staticmethod
    def getitem_kind(idx):
        idx = idx if isinstance(idx, tuple) else (idx,)
        if not idx or not (isinstance(idx[0], slice) and idx[0] == slice(None)):
            raise GraphError("indexing must keep the batch dimension")
        for k in idx[1:]:
            if isinstance(k, slice):
                if k.step not in (None, 1):
                    return "gather"
                continue
            if k is None or k is Ellipsis:
                continue
            return "gather"
        return "slice"


def trace(model: torch.nn.Module, x0: torch.Tensor, optimize: bool = True) -> Graph:
    """Trace ``model`` at the example input ``x0`` (batch, n) into a ``Graph``."""
    if x0.dim() != 2:
        raise GraphError("the input must be (batch, n)")
    x0 = x0.detach().to(torch.float64)
    B = x0.shape[0]
    if B < 2:
        # a batch of 2 keeps the batch axis distinguishable from broadcast axes
        x0 = torch.cat([x0, x0], 0)
        B = 2
    g = Graph()
    mode = _TraceMode(g, B)
    xin = x0.clone()
    g.add("input", [], tuple(x0.shape[1:]))
    mode.register(xin, 0)
    with torch.no_grad(), mode:
        y = model(xin)
    out = mode.nid(y)
    if out is None:
        raise GraphError("the output does not depend on the input")
    if y.dim() != 2:
        raise GraphError("the output must be (batch, 1 + m)")
    g.output = out
    if optimize:
        g.optimize()
    else:
        g._compact()
    return g
