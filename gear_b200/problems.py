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
