"""Seeded synthetic bounded NLP instances (the benchmark workloads).

Each instance is a ``torch.nn.Module`` mapping x (B, n) to y (B, 1 + m): row 0 is the
objective, rows 1..m are constraints g_k(x) <= 0, the GEAR problem form
(``benchmarks/README.md:36-62`` of the reference). Generation is float64 with a CPU
``torch.Generator``; seed = workload index * 1000 + instance index. Sub-boxes follow
lo = max(L, c - w/2), hi = min(U, c + w/2) with centres uniform in the box.

Workloads:
  quad_exp_n10     n=10, box [-2, 2]^10, f = sum a_i x_i x_{i+1} + b_i exp(c_i x_i) + d_i x_i^2,
                   two constraints of four bilinear terms each (<= 1); 256 sub-boxes of
                   widths U(0.05, 1).
  dense_q_n200     n=200, box [-1, 1]^200, f = x^T Q x + sum sin(w_i x_i) + log(1 + x_i^2),
                   Q = V diag(lambda) V^T; 50 constraints of five bilinear terms plus L x,
                   <= U(0.5, 2); sub-boxes of half-widths U(0, 0.1).
  dense_a_n2048    n=2048, box [-1, 1]^2048, y = A x with A (1024 x 2048) ~ N(0, 1/2048),
                   f = sum alpha_j y_j^2 + beta_j y_j y_{j+1}; no constraints.
"""
from __future__ import annotations

import math
from typing import Tuple

import torch

F64 = torch.float64


def _gen(seed):
    return torch.Generator().manual_seed(int(seed))


class QuadExpN10(torch.nn.Module):
    """f = sum_i a_i x_i x_{i+1} + b_i exp(c_i x_i) + d_i x_i^2, two bilinear rows."""

    def __init__(self, n=10, m=2, terms=4, seed=1000):
        super().__init__()
        g = _gen(seed)
        self.n, self.m, self.terms = n, m, terms
        self.register_buffer("a", torch.randn(n - 1, generator=g, dtype=F64))
        self.register_buffer("b", torch.randn(n, generator=g, dtype=F64))
        self.register_buffer("c", torch.rand(n, generator=g, dtype=F64) * 2 - 1)
        self.register_buffer("d", torch.randn(n, generator=g, dtype=F64))
        self.register_buffer("P", torch.randint(0, n, (m * terms,), generator=g))
        self.register_buffer("R", torch.randint(0, n, (m * terms,), generator=g))
        self.register_buffer("W", torch.randn(m * terms, generator=g, dtype=F64))
        self.box = (-2.0, 2.0)

    def forward(self, x):
        f = ((self.a * x[:, :-1] * x[:, 1:]).sum(1, keepdim=True)
             + (self.b * torch.exp(self.c * x)).sum(1, keepdim=True)
             + (self.d * x ** 2).sum(1, keepdim=True))
        bil = (self.W * x[:, self.P] * x[:, self.R]).reshape(-1, self.m, self.terms).sum(2)
        return torch.cat([f, bil - 1.0], 1)


class DenseQN200(torch.nn.Module):
    """f = x^T Q x + sum sin(w_i x_i) + log(1 + x_i^2); rows: 5 bilinears + L x - u."""

    def __init__(self, n=200, m=50, terms=5, seed=2000):
        super().__init__()
        g = _gen(seed)
        self.n, self.m, self.terms = n, m, terms
        lam = torch.randn(n, generator=g, dtype=F64)
        V, _ = torch.linalg.qr(torch.randn(n, n, generator=g, dtype=F64))
        Q = (V * lam) @ V.T
        self.register_buffer("Q", (Q + Q.T) / 2)
        self.register_buffer("w", torch.rand(n, generator=g, dtype=F64) * 2.5 + 0.5)
        self.register_buffer("P", torch.randint(0, n, (m * terms,), generator=g))
        self.register_buffer("R", torch.randint(0, n, (m * terms,), generator=g))
        self.register_buffer("Wb", torch.randn(m * terms, generator=g, dtype=F64))
        self.register_buffer("L", torch.randn(m, n, generator=g, dtype=F64))
        self.register_buffer("u", torch.rand(m, generator=g, dtype=F64) * 1.5 + 0.5)
        self.box = (-1.0, 1.0)

    def forward(self, x):
        f = ((x * torch.nn.functional.linear(x, self.Q)).sum(1, keepdim=True)
             + torch.sin(self.w * x).sum(1, keepdim=True)
             + torch.log(1 + x * x).sum(1, keepdim=True))
        bil = (self.Wb * x[:, self.P] * x[:, self.R]).reshape(-1, self.m, self.terms).sum(2)
        return torch.cat([f, bil + torch.nn.functional.linear(x, self.L) - self.u], 1)


class DenseAN2048(torch.nn.Module):
    """y = A x; f = sum alpha_j y_j^2 + beta_j y_j y_{j+1}."""

    def __init__(self, n=2048, k=1024, seed=3000):
        super().__init__()
        g = _gen(seed)
        self.n, self.k = n, k
        self.register_buffer("A", torch.randn(k, n, generator=g, dtype=F64) / math.sqrt(n))
        self.register_buffer("alpha", torch.randn(k, generator=g, dtype=F64))
        self.register_buffer("beta", torch.randn(k - 1, generator=g, dtype=F64))
        self.box = (-1.0, 1.0)

    def forward(self, x):
        y = torch.nn.functional.linear(x, self.A)
        return ((self.alpha * y * y).sum(1, keepdim=True)
                + (self.beta * y[:, :-1] * y[:, 1:]).sum(1, keepdim=True))


class MixedFamily(torch.nn.Module):
    """One instance of the uneven-batch family (the quad-exp family at many sizes and depths).

    n = round(exp(U(ln 5, ln 500))) variables in [-2, 2]^n and depth d ~ U{3..12}: the input
    passes through d stages cycling Mul (z <- z * z[perm] / 2), Exp (z <- exp(c z) - 1,
    c ~ U(-1/2, 1/2)) and Sqr (z <- z^2 / 2), each mapping [-2, 2] into itself; the objective is
    the quad-exp form on the staged vector, f = sum a_i z_i z_{i+1} + b_i exp(c_i z_i) + d_i z_i^2,
    and m = n // 4 constraints are sums of four bilinear terms of x minus 1."""

    STAGES = ("mul", "exp", "sqr")

    def __init__(self, seed=4000, n=None, depth=None, terms=4):
        super().__init__()
        g = _gen(seed)
        u = float(torch.rand(1, generator=g, dtype=F64))
        dd = int(torch.randint(3, 13, (1,), generator=g))
        self.n = n if n is not None else int(round(math.exp(math.log(5) + (math.log(500) - math.log(5)) * u)))
        self.depth = depth if depth is not None else dd
        n = self.n
        self.m, self.terms = n // 4, terms
        self.register_buffer("perm", torch.stack([torch.randperm(n, generator=g) for _ in range(self.depth)]))
        self.register_buffer("cs", torch.rand(self.depth, n, generator=g, dtype=F64) - 0.5)
        self.register_buffer("a", torch.randn(n - 1, generator=g, dtype=F64))
        self.register_buffer("b", torch.randn(n, generator=g, dtype=F64))
        self.register_buffer("c", torch.rand(n, generator=g, dtype=F64) * 2 - 1)
        self.register_buffer("d", torch.randn(n, generator=g, dtype=F64))
        self.register_buffer("P", torch.randint(0, n, (self.m * terms,), generator=g))
        self.register_buffer("R", torch.randint(0, n, (self.m * terms,), generator=g))
        self.register_buffer("W", torch.randn(self.m * terms, generator=g, dtype=F64))
        self.box = (-2.0, 2.0)

    def forward(self, x):
        z = x
        for t in range(self.depth):
            kind = self.STAGES[t % 3]
            if kind == "mul":
                z = 0.5 * (z * z[:, self.perm[t]])
            elif kind == "exp":
                z = torch.exp(self.cs[t] * z) - 1.0
            else:
                z = 0.5 * z ** 2
        f = ((self.a * z[:, :-1] * z[:, 1:]).sum(1, keepdim=True)
             + (self.b * torch.exp(self.c * z)).sum(1, keepdim=True)
             + (self.d * z ** 2).sum(1, keepdim=True))
        if self.m == 0:
            return f
        bil = (self.W * x[:, self.P] * x[:, self.R]).reshape(-1, self.m, self.terms).sum(2)
        return torch.cat([f, bil - 1.0], 1)


def mixed_instance(k: int, **kw) -> MixedFamily:
    """Instance k of the uneven-batch family (seed 4000 + k)."""
    return MixedFamily(seed=4000 + k, **kw)


def mixed_boxes(inst: MixedFamily, batch: int, k: int, seed_offset: int = 500):
    """Sub-boxes of [-2, 2]^n for instance k: centres uniform, widths U(0.05, 1)."""
    g = _gen(4000 + k + seed_offset)
    n = inst.n
    c = -2.0 + 4.0 * torch.rand(batch, n, generator=g, dtype=F64)
    w = 0.05 + 0.95 * torch.rand(batch, n, generator=g, dtype=F64)
    return torch.clamp(c - w / 2, min=-2.0), torch.clamp(c + w / 2, max=2.0)


WORKLOADS = {
    "quad_exp_n10": dict(cls=QuadExpN10, index=1, n=10, width=(0.05, 1.0), kind="width", boxes=256),
    "dense_q_n200": dict(cls=DenseQN200, index=2, n=200, width=(0.0, 0.1), kind="half", boxes=4096),
    "dense_a_n2048": dict(cls=DenseAN2048, index=3, n=2048, width=(0.0, 0.1), kind="half", boxes=8192),
}


def make_instance(workload: str, instance: int = 0, **kw) -> torch.nn.Module:
    spec = WORKLOADS[workload]
    return spec["cls"](seed=spec["index"] * 1000 + instance, **kw)


def make_boxes(workload: str, batch: int, instance: int = 0, n: int = None,
               box: Tuple[float, float] = None, seed_offset: int = 500) -> Tuple[torch.Tensor, torch.Tensor]:
    """Sub-boxes (lo, hi) of shape (batch, n), float64, seeded."""
    spec = WORKLOADS[workload]
    n = spec["n"] if n is None else n
    L, U = box if box is not None else (-2.0, 2.0) if workload == "quad_exp_n10" else (-1.0, 1.0)
    g = _gen(spec["index"] * 1000 + instance + seed_offset)
    c = L + (U - L) * torch.rand(batch, n, generator=g, dtype=F64)
    a, b = spec["width"]
    w = a + (b - a) * torch.rand(batch, n, generator=g, dtype=F64)
    if spec["kind"] == "half":
        w = 2 * w
    lo = torch.clamp(c - w / 2, min=L)
    hi = torch.clamp(c + w / 2, max=U)
    return lo, hi


def root_box(workload: str, n: int = None):
    spec = WORKLOADS[workload]
    n = spec["n"] if n is None else n
    L, U = (-2.0, 2.0) if workload == "quad_exp_n10" else (-1.0, 1.0)
    return torch.full((1, n), L, dtype=F64), torch.full((1, n), U, dtype=F64)


def cut_rows(batch: int, n: int, rows: int, objectives: int = 1, seed: int = 7000, t_lo: float = -1.1,
             t_hi: float = 0.6):
    """A constrained-concretisation workload: boxes (batch, n) of half-widths U(0.05, 0.95) around
    centres U(-2, 2), objectives (batch, objectives, n) ~ N(0, 1) and rows A x + b <= 0 (A (batch,
    rows, n) ~ N(0, 1)) whose plane sits at t ~ U(t_lo, t_hi) half-ranges of the row over its box
    (t < -1: the row never binds; t > 1: it excludes the box; between: it cuts). float64, seeded."""
    g = _gen(seed)
    c = torch.rand(batch, n, generator=g, dtype=F64) * 4 - 2
    w = torch.rand(batch, n, generator=g, dtype=F64) * 0.9 + 0.05
    xl, xu = c - w, c + w
    obj = torch.randn(batch, objectives, n, generator=g, dtype=F64)
    A = torch.randn(batch, rows, n, generator=g, dtype=F64)
    t = torch.rand(batch, rows, generator=g, dtype=F64) * (t_hi - t_lo) + t_lo
    b = -(A * c[:, None]).sum(-1) + t * (A.abs() * w[:, None]).sum(-1)
    return xl, xu, obj, A, b
