"""Tangent-point tables of odd integer powers, restated with torch float64 on the CPU.

TEST INFRASTRUCTURE: part of the CPU oracle (only tests, the smoke check and the benchmark's
CPU-baseline leg use it). Follows BoundPow.precompute_relaxation
(auto_LiRPA/operators/s_shaped.py:695-764): grid step 0.01 up to x_limit 500, doubling then
100-step bisection for d_upper (tangent point <= 0 whose line stays above x**p up to the grid
point) and d_lower (tangent point >= 0 whose line stays below x**p down to minus the grid point).
"""
import functools

import torch

STEP_PRE = 0.01
X_LIMIT = 500


@functools.lru_cache(maxsize=8)
@torch.no_grad()
def tables(p):
    f = lambda x: torch.pow(x, p)
    df = lambda x: p * torch.pow(x, p - 1)
    n = int(X_LIMIT / STEP_PRE)
    grid = STEP_PRE * torch.arange(0, n + 5, dtype=torch.float64)
    lo_side, hi_side = torch.zeros_like(grid), -torch.ones_like(grid)
    while True:
        ok = (df(hi_side) * (grid - hi_side) + f(hi_side) >= f(grid)).int()
        hi_side = ok * hi_side + (1 - ok) * (hi_side * 2)
        if ok.sum() == grid.numel():
            break
    a, b = hi_side, lo_side
    for _ in range(100):
        m = (a + b) / 2
        ok = (df(m) * (grid - m) + f(m) >= f(grid)).int()
        a = ok * m + (1 - ok) * a
        b = ok * b + (1 - ok) * m
    d_upper = a.clone()
    neg = -grid
    a, b = torch.zeros_like(grid), torch.ones_like(grid)
    while True:
        ok = (df(b) * (neg - b) + f(b) <= f(neg)).int()
        b = ok * b + (1 - ok) * (b * 2)
        if ok.sum() == grid.numel():
            break
    for _ in range(100):
        m = (a + b) / 2
        ok = (df(m) * (neg - m) + f(m) <= f(neg)).int()
        a = (1 - ok) * m + ok * a
        b = (1 - ok) * b + ok * m
    return b.clone().numpy(), d_upper.numpy()
