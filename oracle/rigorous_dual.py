"""CPU oracle of the rigorous float64 weak-duality bound (numpy).

TEST INFRASTRUCTURE ONLY: the device kernel (gear_b200/csrc/dual_kernels.cuh) is checked
against it by tests/. It restates dual_lower_bound and certify_infeasible
(solver/complete_verifier/nlp_solver/rigorous_dual.py:1-240) and is pinned to the reference
by tests/golden/make_dual_golden.py.

For min c^T z + c0 s.t. G z <= h, l <= z <= u and y >= 0, D(y) = c0 - h^T y +
sum_j min(r_j l_j, r_j u_j), r = c + G^T y, bounds the LP optimum from below; the returned lb
<= D(y) in exact arithmetic on the given floats (Higham's rounding model, with a double-double
(Dot2) recomputation of r where the first error term is large).
"""
import numpy as np

U = 2.0 ** -53
ETA = 2.0 ** -1074
BIG = 2.0 ** 400


def gamma(k):
    return k * U / (1.0 - k * U)


def _two_sum(a, b):
    s = a + b
    bb = s - a
    return s, (a - (s - bb)) + (b - bb)


def _two_prod(a, b):
    p = a * b
    t = 134217729.0 * a
    ah = t - (t - a)
    al = a - ah
    t = 134217729.0 * b
    bh = t - (t - b)
    bl = b - bh
    return p, ((ah * bh - p) + ah * bl + al * bh) + al * bl


def reduced_float(row, col, val, c, y):
    """_reduced_float (rigorous_dual.py:118-127): column sums in entry order, then + c."""
    B, n = c.shape
    r = np.zeros((B, n))
    rho = np.zeros((B, n))
    k = np.zeros((B, n))
    vals = np.broadcast_to(val, (B, len(row)))
    for e in range(len(row)):
        ya = y[:, row[e]]
        act = (ya != 0) & (vals[:, e] != 0)
        p = np.where(act, vals[:, e] * ya, 0.0)
        r[:, col[e]] += p
        rho[:, col[e]] += np.abs(p)
        k[:, col[e]] += act
    return r + c, rho + np.abs(c), k


def reduced_dd(row, col, val, c, y):
    """_reduced_dd (rigorous_dual.py:130-142): Dot2 per column in entry order."""
    B, n = c.shape
    hi, lo = c.copy(), np.zeros_like(c)
    vals = np.broadcast_to(val, (B, len(row)))
    order = np.argsort(col, kind="stable")            # entries of each column in their order
    for e in order:
        j = col[e]
        ya = y[:, row[e]]
        a = np.where(ya != 0, vals[:, e], 0.0)
        p, pe = _two_prod(a, ya)
        s, se = _two_sum(hi[:, j], p)
        hi[:, j] = s
        lo[:, j] = lo[:, j] + (se + pe)
    return hi + lo


def _bound(c0, h, l, u, y, r, rho, k, dd, infl, c_err, c0_err):
    """_bound (rigorous_dual.py:146-170)."""
    kk = np.where(k > 0, gamma(k + 1.0), 0.0)
    eps = (kk * kk * rho + 2 * U * np.abs(r) if dd else kk * rho) + 4 * ETA * (k + 2) + c_err
    eps_sign = eps * infl
    fl, fu = np.isfinite(l), np.isfinite(u)
    both = fl & fu
    l0, u0 = np.where(fl, l, 0.0), np.where(fu, u, 0.0)
    pos, neg = (r > eps_sign) & fl, (r < -eps_sign) & fu
    zero = (rho == 0) & (k == 0) & (c_err == 0)
    ok_col = both | zero | pos | neg
    with np.errstate(invalid="ignore", over="ignore"):
        t = np.where(both, np.minimum(r * l0, r * u0), np.where(pos, r * l0, np.where(neg, r * u0, 0.0)))
        M = np.where(both, np.maximum(np.abs(l0), np.abs(u0)),
                     np.where(pos, np.abs(l0), np.where(neg, np.abs(u0), 0.0)))
        hy = np.where(y > 0, h * y, 0.0)
        val = c0 - hy.sum(1) + t.sum(1)
        N = 1.0 + (y > 0).sum(1) + (t != 0).sum(1)
        under = (h.shape[1] + l.shape[1] + 3) * ETA
        E = gamma(N + 2) * (np.abs(c0) + np.abs(hy).sum(1) + np.abs(t).sum(1)) + (M * eps).sum(1) + under + c0_err
        E = E * infl
        E = E + 4 * U * (np.abs(val) + E)
        lb = val - E
    good = ok_col.all(1) & np.isfinite(lb)
    return val, E, np.where(good, lb, -np.inf)


def _evaluate(row, col, val, m, n, c, c0, h, l, u, y, need, c_err, c0_err):
    """_evaluate (rigorous_dual.py:173-199)."""
    y = np.where(np.isnan(y), y, np.maximum(y, 0.0))
    infl = 1.0 + gamma(2 * (m + n) + 16)
    valid = (np.isfinite(c).all(1) & np.isfinite(y).all(1) & np.isfinite(c0) & ~np.isnan(l).any(1)
             & ~np.isnan(u).any(1))
    r, rho, k = reduced_float(row, col, val, c, y)
    v, E, lb = _bound(c0, h, l, u, y, r, rho, k, False, infl, c_err, c0_err)
    flag = (valid & need(v, E, lb)) if len(row) else np.zeros_like(valid)
    dd = np.zeros_like(valid)
    for b in np.nonzero(flag)[0]:
        vb = val if val.shape[0] == 1 else val[b:b + 1]
        if not (np.abs(vb).max(initial=0.0) < BIG and y[b].max(initial=0.0) < BIG and np.abs(c[b]).max(initial=0.0) < BIG):
            continue
        sl = slice(b, b + 1)
        r2 = reduced_dd(row, col, vb, c[sl], y[sl])
        v2, E2, lb2 = _bound(c0[sl], h[sl], l[sl], u[sl], y[sl], r2, rho[sl], k[sl], True, infl, c_err[sl], c0_err[sl])
        dd[b] = True
        if lb2[0] > lb[b]:
            lb[b], E[b], v[b] = lb2[0], E2[0], v2[0]
    return lb, E, v, dd


def dual_lower_bound(row, col, val, m, n, c, c0, h, l, u, y, tol=None):
    """dual_lower_bound (rigorous_dual.py:202-222) without caller error terms: (lb, E, dd)."""
    def need(v, E, lb):
        t = np.maximum(np.abs(v) * 1e-4, 1e-5) if tol is None else tol
        return ~(E <= t / 10) | ~np.isfinite(lb)
    c_err = np.zeros_like(c)
    c0_err = np.zeros_like(c0)
    lb, E, _, dd = _evaluate(row, col, val, m, n, c, c0, h, l, u, y, need, c_err, c0_err)
    return lb, E, dd


def certify_infeasible(row, col, val, m, n, h, l, u, y):
    """certify_infeasible (rigorous_dual.py:225-238)."""
    B = y.shape[0]
    zc, zc0 = np.zeros((B, n)), np.zeros(B)
    ray = (y > 0).any(1)

    def need(v, E, lb):
        return (v + E > 0) & (lb <= 0) & ray
    lb, _, _, _ = _evaluate(row, col, val, m, n, zc, zc0, h, l, u, y, need, zc, zc0)
    return lb > 0
