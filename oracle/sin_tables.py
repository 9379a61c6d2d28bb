"""Tangent-point tables of the periodic S-shaped sin/cos relaxation, restated in numpy.

TEST INFRASTRUCTURE: part of the CPU oracle; only tests, the smoke check and the
benchmark's CPU-baseline leg use it.

Follows ``auto_LiRPA/operators/s_shaped.py:125-202`` (``precompute_relaxation``: bisection
for the tangent points d_lower / d_upper on the grid step 0.01 up to x_limit = pi/2) and
``auto_LiRPA/operators/trigonometric.py:49-66, 228-320`` (the 1001-entry global tangent
tables over [0, 2 pi], 20-step bisections).
"""
import math

import numpy as np

STEP_PRE = 0.01
N_TABLE = 1001
PI = math.pi


def precompute_d(x_limit=PI / 2, max_iter=100):
    """d_lower / d_upper for sin (func) with derivative cos (s_shaped.py:125-202)."""
    func, dfunc = np.sin, np.cos
    num_points_pre = int(x_limit / STEP_PRE)
    upper = STEP_PRE * np.arange(0, num_points_pre + 5, dtype=np.float64)
    r = np.zeros_like(upper)
    l = -np.ones_like(upper)

    def check_lower(up, d):
        k = dfunc(d)
        return k * (up - d) + func(d) <= func(up)

    def check_upper(lo, d):
        k = dfunc(d)
        return k * (lo - d) + func(d) >= func(lo)

    while True:
        checked = check_lower(upper, l).astype(np.int64)
        l = checked * l + (1 - checked) * (l * 2)
        if checked.sum() == l.size:
            break
    for _ in range(max_iter):
        m = (l + r) / 2
        checked = check_lower(upper, m).astype(np.int64)
        l = checked * m + (1 - checked) * l
        r = checked * r + (1 - checked) * m
    d_lower = l.copy()

    lower = -STEP_PRE * np.arange(0, num_points_pre + 5, dtype=np.float64)
    l = np.zeros_like(upper)
    r = np.ones_like(upper)
    while True:
        checked = check_upper(lower, r).astype(np.int64)
        r = checked * r + (1 - checked) * (r * 2)
        if checked.sum() == l.size:
            break
    for _ in range(max_iter):
        m = (l + r) / 2
        checked = check_upper(lower, m).astype(np.int64)
        l = (1 - checked) * m + checked * l
        r = (1 - checked) * r + checked * m
    d_upper = r.copy()
    return d_lower, d_upper


def _check_bound(tp, x):
    d = np.cos(tp)
    val = d * (x - tp) + np.sin(tp)
    return np.sin(x) - val


def get_lower_left_bound(xl, steps=20):
    cycles = np.floor((xl + 0.5 * PI) / (2 * PI)) * (2 * PI)
    xl = xl - cycles
    use_tangent_line = (xl >= PI).astype(np.float64)
    left = PI * np.ones_like(xl)
    right = (1.5 * PI) * np.ones_like(xl)
    last_right = right.copy()
    for _ in range(steps):
        mid = (left + right) / 2.
        margin = _check_bound(mid, xl)
        pos = (margin > 0).astype(np.float64)
        neg = 1.0 - pos
        right = mid * pos + right * neg
        last_right = mid * pos + last_right * neg
        left = mid * neg + left * pos
    d = xl * use_tangent_line + last_right * (1. - use_tangent_line)
    return d, cycles


def get_upper_left_bound(xl, steps=20):
    cycles = np.floor((xl - 0.5 * PI) / (2 * PI)) * (2 * PI)
    xl = xl - cycles
    use_tangent_line = (xl >= 2.0 * PI).astype(np.float64)
    left = (2.0 * PI) * np.ones_like(xl)
    right = (2.5 * PI) * np.ones_like(xl)
    last_right = right.copy()
    for _ in range(steps):
        mid = (left + right) / 2.
        margin = _check_bound(mid, xl)
        pos = (margin > 0).astype(np.float64)
        neg = 1.0 - pos
        right = mid * neg + right * pos
        last_right = mid * neg + last_right * pos
        left = mid * pos + left * neg
    d = xl * use_tangent_line + last_right * (1. - use_tangent_line)
    return d, cycles


def get_lower_right_bound(xu, steps=20):
    cycles = np.floor((xu + 0.5 * PI) / (2 * PI)) * (2 * PI)
    xu = xu - cycles
    d, _ = get_lower_left_bound(PI - xu, steps)
    return 3 * PI - d, cycles - 2 * PI


def get_upper_right_bound(xu, steps=20):
    cycles = np.floor((xu - 0.5 * PI) / (2 * PI)) * (2 * PI)
    xu = xu - cycles
    d, _ = get_upper_left_bound(3 * PI - xu, steps)
    return 5 * PI - d, cycles - 2 * PI


def build():
    """All tables: dict of float64 arrays."""
    x = np.linspace(0, 2 * PI, N_TABLE, dtype=np.float64)
    d_lower, d_upper = precompute_d()
    xl_lower = get_lower_left_bound(x)
    xl_upper = get_upper_left_bound(x)
    xu_lower = get_lower_right_bound(x)
    xu_upper = get_upper_right_bound(x)
    return dict(d_lower=d_lower, d_upper=d_upper,
                xl_lower_d=xl_lower[0], xl_lower_c=xl_lower[1],
                xl_upper_d=xl_upper[0], xl_upper_c=xl_upper[1],
                xu_lower_d=xu_lower[0], xu_lower_c=xu_lower[1],
                xu_upper_d=xu_upper[0], xu_upper_c=xu_upper[1])
