"""Tangent-point tables of the periodic sin/cos relaxation, built once on the host.

Same construction as the reference (``auto_LiRPA/operators/s_shaped.py:125-202``
``precompute_relaxation`` with x_limit = pi/2 and step 0.01, and
``auto_LiRPA/operators/trigonometric.py:49-66, 228-320``: four 1001-entry tables of global
tangent points over [0, 2 pi], 20-step bisections), computed with torch float64 on the CPU
and uploaded to the device next to the program constants.
"""
import math

import numpy as np
import torch

STEP_PRE = 0.01
N_TABLE = 1001
PI = math.pi


@torch.no_grad()
def _precompute_d(x_limit=PI / 2, max_iter=100):
    func, dfunc = torch.sin, torch.cos
    n = int(x_limit / STEP_PRE)
    upper = STEP_PRE * torch.arange(0, n + 5, dtype=torch.float64)
    r = torch.zeros_like(upper)
    l = -torch.ones_like(upper)

    def check_lower(up, d):
        return dfunc(d) * (up - d) + func(d) <= func(up)

    def check_upper(lo, d):
        return dfunc(d) * (lo - d) + func(d) >= func(lo)

    while True:
        c = check_lower(upper, l).int()
        l = c * l + (1 - c) * (l * 2)
        if c.sum() == l.numel():
            break
    for _ in range(max_iter):
        m = (l + r) / 2
        c = check_lower(upper, m).int()
        l = c * m + (1 - c) * l
        r = c * r + (1 - c) * m
    d_lower = l.clone()
    lower = -STEP_PRE * torch.arange(0, n + 5, dtype=torch.float64)
    l = torch.zeros_like(upper)
    r = torch.ones_like(upper)
    while True:
        c = check_upper(lower, r).int()
        r = c * r + (1 - c) * (r * 2)
        if c.sum() == l.numel():
            break
    for _ in range(max_iter):
        m = (l + r) / 2
        c = check_upper(lower, m).int()
        l = (1 - c) * m + c * l
        r = (1 - c) * r + c * m
    return d_lower, r.clone()


def _check(tp, x):
    return torch.sin(x) - (torch.cos(tp) * (x - tp) + torch.sin(tp))


def _lower_left(xl, steps=20):
    cycles = torch.floor((xl + 0.5 * PI) / (2 * PI)) * (2 * PI)
    xl = xl - cycles
    use = (xl >= PI).to(xl.dtype)
    left = PI * torch.ones_like(xl)
    right = 1.5 * PI * torch.ones_like(xl)
    last = right.clone()
    for _ in range(steps):
        mid = (left + right) / 2.
        pos = (_check(mid, xl) > 0).to(xl.dtype)
        neg = 1.0 - pos
        right = mid * pos + right * neg
        last = mid * pos + last * neg
        left = mid * neg + left * pos
    return xl * use + last * (1. - use), cycles


def _upper_left(xl, steps=20):
    cycles = torch.floor((xl - 0.5 * PI) / (2 * PI)) * (2 * PI)
    xl = xl - cycles
    use = (xl >= 2.0 * PI).to(xl.dtype)
    left = 2.0 * PI * torch.ones_like(xl)
    right = 2.5 * PI * torch.ones_like(xl)
    last = right.clone()
    for _ in range(steps):
        mid = (left + right) / 2.
        pos = (_check(mid, xl) > 0).to(xl.dtype)
        neg = 1.0 - pos
        right = mid * neg + right * pos
        last = mid * neg + last * pos
        left = mid * pos + left * neg
    return xl * use + last * (1. - use), cycles


@torch.no_grad()
def build():
    """Tables in the device layout order (see SIN_TABLE_ORDER)."""
    x = torch.linspace(0, 2 * PI, N_TABLE, dtype=torch.float64)
    d_lower, d_upper = _precompute_d()
    xl_lower = _lower_left(x)
    xl_upper = _upper_left(x)
    c = torch.floor((x + 0.5 * PI) / (2 * PI)) * (2 * PI)
    d, _ = _lower_left(PI - (x - c))
    xu_lower = (3 * PI - d, c - 2 * PI)
    c = torch.floor((x - 0.5 * PI) / (2 * PI)) * (2 * PI)
    d, _ = _upper_left(3 * PI - (x - c))
    xu_upper = (5 * PI - d, c - 2 * PI)
    out = {"d_lower": d_lower, "d_upper": d_upper,
           "xl_lower_d": xl_lower[0], "xl_lower_c": xl_lower[1],
           "xl_upper_d": xl_upper[0], "xl_upper_c": xl_upper[1],
           "xu_lower_d": xu_lower[0], "xu_lower_c": xu_lower[1],
           "xu_upper_d": xu_upper[0], "xu_upper_c": xu_upper[1]}
    return {k: v.numpy().astype(np.float64) for k, v in out.items()}


_SIN_CACHE = {}


def build_cached():
    """build(), computed once per process (the tables depend on nothing)."""
    if "t" not in _SIN_CACHE:
        _SIN_CACHE["t"] = build()
    return _SIN_CACHE["t"]


SIN_TABLE_ORDER = ("d_lower", "d_upper", "xl_lower_d", "xl_lower_c", "xl_upper_d", "xl_upper_c",
                   "xu_lower_d", "xu_lower_c", "xu_upper_d", "xu_upper_c")


# ---------------------------------------------------------------- odd integer powers
POW_X_LIMIT = 500.0
_POW_CACHE = {}


def pow_tables_cached(p: int):
    """pow_tables(p), built once per process."""
    if p not in _POW_CACHE:
        _POW_CACHE[p] = pow_tables(p)
    return _POW_CACHE[p]


@torch.no_grad()
def pow_tables(p: int, max_iter: int = 100):
    """Tangent-point tables of an odd power x**p on the grid 0.01 * [0, 50005) (the reference's
    BoundPow.precompute_relaxation, auto_LiRPA/operators/s_shaped.py:695-764, x_limit 500):
    d_upper[i] <= 0 is the tangent point whose tangent stays above the curve up to 0.01 i, and
    d_lower[i] >= 0 the one whose tangent stays below it down to -0.01 i. 100-step bisections in
    float64 on the CPU. Returns (d_lower, d_upper) as float64 numpy arrays."""
    func = lambda x: torch.pow(x, p)
    dfunc = lambda x: p * torch.pow(x, p - 1)
    n = int(POW_X_LIMIT / STEP_PRE)

    def below(up, d):        # the tangent at d lower-bounds the curve at up
        return dfunc(d) * (up - d) + func(d) <= func(up)

    def above(lo, d):        # the tangent at d upper-bounds the curve at lo
        return dfunc(d) * (lo - d) + func(d) >= func(lo)

    upper = STEP_PRE * torch.arange(0, n + 5, dtype=torch.float64)
    r = torch.zeros_like(upper)
    l = -torch.ones_like(upper)
    while True:
        c = above(upper, l).int()
        l = c * l + (1 - c) * (l * 2)
        if c.sum() == l.numel():
            break
    for _ in range(max_iter):
        m = (l + r) / 2
        c = above(upper, m).int()
        l = c * m + (1 - c) * l
        r = c * r + (1 - c) * m
    d_upper = l.clone()
    lower = -STEP_PRE * torch.arange(0, n + 5, dtype=torch.float64)
    l = torch.zeros_like(upper)
    r = torch.ones_like(upper)
    while True:
        c = below(lower, r).int()
        r = c * r + (1 - c) * (r * 2)
        if c.sum() == l.numel():
            break
    for _ in range(max_iter):
        m = (l + r) / 2
        c = below(lower, m).int()
        l = (1 - c) * m + c * l
        r = (1 - c) * r + c * m
    return r.clone().numpy(), d_upper.numpy()
