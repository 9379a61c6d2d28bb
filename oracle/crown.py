"""CPU oracle: a float64 numpy restatement of the reference's CROWN bound propagation.

TEST INFRASTRUCTURE ONLY. Nothing in the product imports this module; the GPU path
(``gear_b200``) is checked against it by ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py``.

What it restates (reference paths are relative to ``solver/auto_LiRPA``):

* ``BoundedModule.compute_bounds(method='CROWN')`` / ``_compute_bounds_main``
  (``bound_general.py:1275-1722``): roots, C = I default, ``check_prior_bounds``
  (``:1032-1079``) and ``compute_intermediate_bounds`` (``:1081-1222``) with the IBP
  shortcuts ``check_IBP_intermediate`` / ``check_IBP_first_linear``
  (``interval_bound.py:310-390``), NaN sanitising (``bound_general.py:1164-1173``) and
  ``compare_with_IBP`` (``interval_bound.py:393-406``) under
  ``compare_crown_with_ibp_intermediate``.
* ``backward_general`` (``backward_bound.py:880-1206``): the degree-counted BFS
  (``get_degrees`` ``:1498``), per-node ``bound_backward`` and ``add_bound`` accumulation.
* Operator relaxations: McCormick with the coefficient-aware plane pick
  (``operators/bivariate.py:38-77, 206-247, 401-488``), generic sign-split backward
  (``operators/activation_base.py:137-183``, ``operators/clampmult.py:31-77``),
  Sqr (``operators/activations.py:186-210``), Exp (``operators/convex_concave.py:569-626``),
  Log (``operators/convex_concave.py:64-92``), Sin/Cos (``operators/s_shaped.py:325-550``,
  ``operators/trigonometric.py:27-527``).
* Box concretisation (``concretize_bounds.py:160-321``, ``perturbations.py:241-275``,
  ``concretize_func.py:553-569``) with ``box_rounding_error`` (``fp_enclosure.py:60-82``).

Rounding enclosure. The reference charges outward rounding terms of order eps * magnitude
(``fp_enclosure.py``, ``backward_bound.py:529-823``). This oracle charges the same
categories with the formulas shared by the GPU engine (see ``charge_*`` below): affine
steps through Linear/MatMul (gamma_k <|A|, |W| m>), inexact constant products (u <|A'|, m>),
Add/Sub output rounding (72 eps <|A|, |m_x| + |m_y|>), A merges (u <|A_sum|, m>), bias
accumulation and the box concretisation term. Node magnitudes m are max(|lo|, |hi|) of the
node's stored bounds, else of its interval from plain IBP over the input box. All charges
are O(1e-14) relative in float64, far below the 1e-5 parity tolerance; they keep the bounds
outward-rounded, not bit-identical to the reference.

Undefined relaxations (a non-finite input interval of a relaxing node, log of a
non-positive interval) discard the rows that touch the element (-inf lower / +inf upper,
the ``undefined_relaxation_rows`` semantics of ``backward_bound.py:295-418``), and those
rows fall back to interval bounds (``_interval_fallback_rows``, ``:826``). The reference's
finer ``undefined_relaxation_interval`` stop is not restated.
"""
from __future__ import annotations

import math
from collections import deque
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import sin_tables

EPS = float(np.finfo(np.float64).eps)
U = EPS / 2
PI = math.pi
EPSILON = 1e-12  # operators/base.py:32


def rounding_error(mag, n):
    """fp_enclosure.py:34-48: magnitude * (n + 16) * 4 eps."""
    return mag * ((n + 16) * EPS * 4)


def finite_abs(v):
    return np.where(np.isfinite(v), np.abs(v), 0.0)


def widen(bound, err, sign):
    """fp_enclosure.py:51-57."""
    out = np.where(np.isfinite(bound), bound + sign * err, bound)
    return np.where(np.isposinf(err), sign * np.inf, out)


def gamma(k):
    """Higham gamma_k as used by backward_bound.py:_higham: (k + 1) u (1 + 1e-6)."""
    return (k + 1) * U * (1 + 1e-6)


def two_product_error(a, b):
    """a * b - fl(a * b) exactly (Dekker's TwoProduct with Veltkamp's split); +inf where the product
    is not finite or a split could overflow."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    with np.errstate(all="ignore"):
        p = a * b
        f = 2.0 ** 27 + 1.0

        def split(x):
            t = f * x
            h = t - (t - x)
            return h, x - h
        ah, al = split(a)
        bh, bl = split(b)
        e = ((ah * bh - p) + ah * bl + al * bh) + al * bl
    lim = np.finfo(np.float64).max / 2.0 ** 28
    ok = np.isfinite(p) & (np.abs(a) < lim) & (np.abs(b) < lim)
    return np.where(ok, e, np.inf)


def abs_dot(absA, m):
    """<|A|, m> per row with 0 * inf = 0 and inf where |A| > 0 meets m = inf."""
    mf = np.where(np.isinf(m), 0.0, m)
    tot = (absA * mf).sum(-1)
    hit = ((absA > 0) & np.isinf(m)).any(-1)
    return np.where(hit, np.inf, tot)


# ============================================================ relaxations
def relax_sqr(l, u):
    """operators/activations.py:186-210."""
    uk = l + u
    ub = -l * uk + l * l
    mid = np.maximum(l, 0) - np.maximum(-u, 0)
    lk = 2 * mid
    lb = -mid * lk + mid * mid
    return lk, lb, uk, ub


def relax_exp(l, u):
    """operators/convex_concave.py:569-626 (plain CROWN, no alpha)."""
    with np.errstate(all="ignore"):
        du = u - l
        neg_expm1 = -np.expm1(l - u)
        m_par = u + np.log(np.maximum(neg_expm1, EPSILON)) - np.log(np.maximum(du, EPSILON))
        m_mid = (l + u) / 2
        m = np.where(du > 1e-6, m_par, m_mid)
        m = np.minimum(np.maximum(m, l), u)
        exp_l, exp_m, exp_u = np.exp(l), np.exp(m), np.exp(u)
        lower_k = np.where(np.isfinite(exp_m), exp_m, 0.0)
        lower_x0 = np.where(np.isfinite(m), m, 0.0)
        lower_b = -lower_x0 * lower_k + lower_k
        lsafe = np.isfinite(lower_k) & np.isfinite(lower_b)
        lw = np.where(lsafe, lower_k, 0.0)
        lb = np.where(lsafe, lower_b, 0.0)
        d = u - l
        k = np.where(d < 1,
                     exp_l * np.where(d > 0, np.expm1(np.minimum(d, 1)) / np.maximum(d, 1e-300), 1.0),
                     (exp_u - exp_l) / np.maximum(d, 1))
        upper_b = -l * k + exp_l
        usafe = np.isfinite(k) & np.isfinite(upper_b)
        uw = np.where(usafe, k, 0.0)
        ub = np.where(usafe, upper_b, np.inf)
    return lw, lb, uw, ub


def _pw(x, p):
    """x ** p as the reference evaluates it (torch.pow on float64 tensors)."""
    import torch
    return torch.pow(torch.as_tensor(np.asarray(x, np.float64)), p).numpy()


def _retrieve(table, bound, default):
    """retrieve_from_precompute (s_shaped.py:223-245): index trunc(bound / 0.01) + 1."""
    with np.errstate(invalid="ignore"):
        idx = np.maximum(np.trunc(bound / 0.01), 0)
    idx = np.where(np.isfinite(idx), idx, len(table)).astype(np.float64) + 1
    inside = idx < len(table)
    return np.where(inside, table[np.minimum(idx, len(table) - 1).astype(np.int64)], default)


def relax_pow(l, u, p):
    """BoundPow.bound_relax (operators/s_shaped.py:881-1035), plain CROWN, for an exponent p that
    is an integer >= 3 (odd: inverse-S relaxation with tangent tables, even: convex with the 1e-6
    relative widening) or a non-integer > 0 (x >= 0: convex / concave tangent and secant). The
    input upper bound is first raised to lower + 1e-8 (bound_backward, :791/:801)."""
    u = np.maximum(u, l + 1e-8)
    if p == int(p) and int(p) % 2 == 1:
        from .pow_tables import tables
        p = int(p)
        f = lambda x: _pw(x, p)
        df = lambda x: p * _pw(x, p - 1)
        d2 = lambda x: p * (p - 1) * _pw(x, p - 2)
        y_l, y_u = f(l), f(u)
        width = u - l
        k_dir = (y_u - y_l) / np.maximum(width, 1e-8)
        k_dir = np.where(width < 1e-8, df(l), k_dir)
        conv = d2(l) >= 0
        mneg = (d2(l) >= 0) & (d2(u) >= 0)
        mpos = (d2(l) < 0) & (d2(u) < 0)
        mboth = ~(mneg | mpos)
        lw, lb, uw, ub = [np.zeros_like(l) for _ in range(4)]

        def put(mask, kind, k, x0, y0):
            nonlocal lw, lb, uw, ub
            k = np.broadcast_to(k, l.shape)
            b = -x0 * k + y0
            if kind == "lower":
                lw, lb = np.where(mask, k, lw), np.where(mask, b, lb)
            else:
                uw, ub = np.where(mask, k, uw), np.where(mask, b, ub)
        put(mneg, "upper", k_dir, l, y_l)
        put(mpos, "lower", k_dir, l, y_l)
        d_lo_t, d_up_t = tables(p)
        d_upper = _retrieve(d_up_t, u, l)
        d_lower = _retrieve(d_lo_t, -l, u)
        dl_dir = np.where(conv, k_dir < df(l), k_dir > df(u)) & mboth
        du_dir = np.where(conv, k_dir < df(u), k_dir > df(l)) & mboth
        m = (l + u) / 2
        y_m, k_m = f(m), df(m)
        put(mneg, "lower", k_m, m, y_m)
        put(mpos, "upper", k_m, m, y_m)
        put(dl_dir, "lower", k_dir, l, y_l)
        put(mboth & ~dl_dir, "lower", df(d_lower), d_lower, f(d_lower))
        put(du_dir, "upper", k_dir, l, y_l)
        put(mboth & ~du_dir, "upper", df(d_upper), d_upper, f(d_upper))
        put(mboth & (d_lower < m), "lower", k_m, m, y_m)
        put(mboth & (d_upper >= m), "upper", k_m, m, y_m)
        return lw, lb, uw, ub
    if p == int(p):
        p = int(p)
        y_l, y_u = _pw(l, p), _pw(u, p)
        eps = np.maximum(np.abs(y_l), np.abs(y_u)) * 1e-6 + 1e-12
        uk = (y_u - y_l) / np.maximum(u - l, 1e-8)
        ub = -l * uk + (y_l + eps)
        mid = np.where(l >= 0, l, np.where(u <= 0, u, 0.0))
        lk = p * _pw(mid, p - 1)
        lb = -mid * lk + (_pw(mid, p) - eps)
        return lk, lb, uk, ub
    # non-integer exponent on x >= 0
    l_t = np.maximum(l, 1e-9) if p < 1 else l
    if p < 1:
        zl = l == 0
        f_l = np.where(zl, 0.0, _pw(np.where(zl, 1.0, l), p))
    else:
        f_l = _pw(l, p)
    f_u = _pw(u, p)
    k_s = (f_u - f_l) / np.maximum(u - l, 1e-8)
    m = (l_t + u) / 2
    if p > 1:
        z = m == 0
        ms = np.where(z, 1.0, m)
        k_t = np.where(z, 0.0, p * _pw(ms, p - 1))
        f_m = np.where(z, 0.0, _pw(ms, p))
    else:
        k_t = p * _pw(m, p - 1)
        f_m = _pw(m, p)
    if p < 1:
        return k_s, -l * k_s + f_l, k_t, -m * k_t + f_m
    return k_t, -m * k_t + f_m, k_s, -l * k_s + f_l


def pow_domain(l, u, p):
    """The interval BoundPow relaxes: a non-integer exponent restricts the base to x >= 0
    (domain_aware_ops); an interval entirely below 0 has no relaxation (undefined)."""
    if p == int(p):
        return l, u, np.zeros(np.shape(l), bool)
    return np.maximum(l, 0.0), u, ~(u >= 0)


def relax_log(l, u):
    """operators/convex_concave.py:64-92 (input already known to be > 0)."""
    with np.errstate(all="ignore"):
        rl, ru = np.log(l), np.log(u)
        du = u - l
        ku = (ru - rl) / np.maximum(du, EPSILON)
        lw, lb = ku, -l * ku + rl
        dlog = np.maximum(ru - rl, EPSILON)
        m_par = du / dlog
        m_mid = (l + u) / 2
        m = np.where(du > 1e-6, m_par, m_mid)
        m = np.minimum(np.maximum(m, l), u)
        k = 1.0 / m
        uw, ub = k, -m * k + np.log(m)
    return lw, lb, uw, ub


class SinRelax:
    """BoundSin / BoundCos relaxation (s_shaped.py:325-550, trigonometric.py:27-527)."""

    def __init__(self):
        t = sin_tables.build()
        self.t = t
        self.num_points_pre = len(t["d_lower"]) - 5

    @staticmethod
    def _masks(lb, ub):
        twopi = 2 * PI
        lbc = lb - np.floor(lb / twopi) * twopi
        ubc = ub - np.floor(ub / twopi) * twopi
        m_lb = [(lbc >= 0) & (lbc < PI / 2), (lbc >= PI / 2) & (lbc < PI),
                (lbc >= PI) & (lbc < 3 * PI / 2), (lbc >= 3 * PI / 2) & (lbc < 2 * PI)]
        m_ub = [(ubc >= 0) & (ubc < PI / 2), (ubc >= PI / 2) & (ubc < PI),
                (ubc >= PI) & (ubc < 3 * PI / 2), (ubc >= 3 * PI / 2) & (ubc < 2 * PI)]
        sig = (ub - lb <= PI) & ((((m_lb[1] | m_lb[2]) & (m_ub[1] | m_ub[2]))) |
                                 ((m_lb[0] | m_lb[3]) & (m_ub[0] | m_ub[3])))
        mneg = (m_lb[2] | m_lb[3]) & ((m_ub[2] | m_ub[3]) & sig)
        mpos = (m_lb[0] | m_lb[1]) & ((m_ub[0] | m_ub[1]) & sig)
        mboth = sig ^ (mneg | mpos)
        convex_concave = (-np.sin(lb)) >= 0
        return sig, mneg, mpos, mboth, convex_concave

    def _gen_d(self, lower, upper):
        """trigonometric.py:generate_d_lower_upper."""
        t, sp = self.t, sin_tables.STEP_PRE
        twopi = 2 * PI
        k = np.floor(upper / twopi)
        uc = upper - k * twopi
        c1 = (uc >= 0) & (uc <= PI / 2)
        ucn = np.clip(uc, 0, PI / 2)
        idx = np.maximum(0, (ucn / sp).astype(np.int64)) + 1
        d_lower = (t["d_lower"][idx] + k * 2 * PI) * c1
        c2 = (uc >= PI) & (uc <= 3 * PI / 2)
        ucn = np.clip(uc, PI, 3 * PI / 2)
        idx = np.maximum(0, ((PI - ucn) / -sp).astype(np.int64)) + 1
        d_upper = (PI - t["d_upper"][idx] + k * 2 * PI) * c2
        k = np.floor(lower / twopi)
        lc = lower - k * twopi
        c3 = (lc >= 3 * PI / 2) & (lc <= 2 * PI)
        lcn = np.clip(lc, 3 * PI / 2, 2 * PI)
        idx = np.maximum(0, ((lcn - 2 * PI) / -sp).astype(np.int64)) + 1
        d_upper = d_upper + (t["d_upper"][idx] + (k + 1) * 2 * PI) * c3
        c4 = (lc >= PI / 2) & (lc <= PI)
        lcn = np.clip(lc, PI / 2, 3 * PI)
        idx = np.maximum(0, ((PI - lcn) / sp).astype(np.int64)) + 1
        d_lower = d_lower + (PI - t["d_lower"][idx] + k * 2 * PI) * c4
        return d_lower, d_upper

    def _bound_tb(self, lb, ub):
        """trigonometric.py:get_bound_tb (non-optimised branch)."""
        t = self.t
        lower, upper = lb, ub
        step = 2 * PI / (sin_tables.N_TABLE - 1)
        lb_cyc = np.floor(lb / (2 * PI)) * (2 * PI)
        lbm = np.clip(lb - lb_cyc, 0, 2 * PI)
        ub_cyc = np.floor(ub / (2 * PI)) * (2 * PI)
        ubm = np.clip(ub - ub_cyc, 0, 2 * PI)
        il = (lbm / step).astype(np.int64)
        iu = np.minimum(np.ceil(ubm / step).astype(np.int64), sin_tables.N_TABLE - 1)
        tll, tlu = t["xl_lower_d"][il], t["xl_upper_d"][il]
        trl, tru = t["xu_lower_d"][iu], t["xu_upper_d"][iu]
        cll, clu = t["xl_lower_c"][il], t["xl_upper_c"][il]
        crl, cru = t["xu_lower_c"][iu], t["xu_upper_c"][iu]
        mid = (lower + upper) / 2

        def pick(tl, tr, cl, cr, base):
            unf_l = tl + cl + lb_cyc
            l_ends = base + cl + lb_cyc
            unf_r = tr + cr + ub_cyc
            r_ends = base + cr + ub_cyc
            leftmost = (mid < unf_l) & (unf_l <= upper)
            left_range = (mid >= unf_l) & (mid < l_ends)
            inbetween = (mid >= l_ends) & (mid < r_ends)
            rightmost = (mid >= unf_r) & (unf_r >= lower)
            right_range = (~left_range) & ((mid >= r_ends) & (mid < unf_r))
            tp = (leftmost * tl + left_range * (mid - cl - lb_cyc) + inbetween.astype(np.float64) * base
                  + rightmost * tr + right_range * (mid - cr - ub_cyc))
            any_ = leftmost | left_range | inbetween | rightmost | right_range
            return np.where(any_, tp, tl)

        tp_l = pick(tll, trl, cll, crl, 1.5 * PI)
        tp_u = pick(tlu, tru, clu, cru, 2.5 * PI)
        d_l = np.cos(tp_l)
        b_l = np.sin(tp_l) - d_l * (tp_l + np.where(tp_l <= 1.5 * PI, cll + lb_cyc, crl + ub_cyc))
        d_u = np.cos(tp_u)
        b_u = np.sin(tp_u) - d_u * (tp_u + np.where(tp_u <= 2.5 * PI, clu + lb_cyc, cru + ub_cyc))
        return d_l, b_l, d_u, b_u

    @staticmethod
    def _n_crossing(start, end, s):
        cycles = np.floor((end - start) / (2 * PI))
        dist = np.floor((s - start) / (2 * PI))
        real_s = s - dist * 2 * PI
        real_end = end - cycles * 2 * PI
        return (real_s >= start).astype(np.float64) * (real_s <= real_end).astype(np.float64) + cycles

    def _branch(self, lb, ub):
        """trigonometric.py:bound_relax_branch."""
        ub = np.maximum(ub, lb + 1e-8)
        sub, slb = np.sin(ub), np.sin(lb)
        mid = (sub + slb) / 2.
        smid = np.sin((ub + lb) / 2)
        gap = smid - mid
        slope = (sub - slb) / np.maximum(ub - lb, 1e-10)
        bias = slb - slope * lb
        # get_intersection(lb, ub, slope, theta = pi/2)
        c = slope
        with np.errstate(invalid="ignore"):
            # BoundSin.arcsin: |c| > 1 (a rounded secant slope) gives NaN, no crossing
            cr1 = np.where(c == -1, -PI / 2, np.where(c == 1, PI / 2, np.arcsin(c))) - 0.5 * PI
        cr2 = PI - cr1 - 2 * 0.5 * PI
        crossings = self._n_crossing(lb, ub, cr1) + self._n_crossing(lb, ub, cr2)
        use_line = crossings == 1
        upper_line = (gap < 0) & use_line
        lower_line = (gap >= 0) & use_line
        d_l, b_l, d_u, b_u = self._bound_tb(lb, ub)
        ll = lower_line.astype(np.float64)
        ul = upper_line.astype(np.float64)
        return (ll * slope + (1 - ll) * d_l, ll * bias + (1 - ll) * b_l,
                ul * slope + (1 - ul) * d_u, ul * bias + (1 - ul) * b_u)

    def relax_sin(self, l, u):
        """BoundSin.bound_relax incl. the 8 eps (1 + max|l|,|u|) widening."""
        func, dfunc = np.sin, np.cos
        lower, upper = l, u
        lw = np.zeros_like(l); lb = np.zeros_like(l); uw = np.zeros_like(l); ub = np.zeros_like(l)
        sig, mneg, mpos, mboth, cc = self._masks(l, u)

        def add(mask, side, k, x0, y0):
            nonlocal lw, lb, uw, ub
            b = -x0 * k + y0
            if side == "lower":
                lw = np.where(mask, k, lw); lb = np.where(mask, b, lb)
            else:
                uw = np.where(mask, k, uw); ub = np.where(mask, b, ub)

        with np.errstate(all="ignore"):
            y_l, y_u = func(lower), func(upper)
            width = upper - lower
            k_direct = (y_u - y_l) / np.maximum(width, 1e-8)
            k_direct = np.where(width < 1e-8, dfunc(lower), k_direct)
            add(mneg, "upper", k_direct, lower, y_l)
            add(mpos, "lower", k_direct, lower, y_l)
            d_lower, d_upper = self._gen_d(lower, upper)
            mdl = np.where(cc, k_direct < dfunc(lower), k_direct > dfunc(upper)) & mboth
            mdu = np.where(cc, k_direct < dfunc(upper), k_direct > dfunc(lower)) & mboth
            m = (lower + upper) / 2
            y_m, k_m = func(m), dfunc(m)
            add(mneg, "lower", k_m, m, y_m)
            add(mpos, "upper", k_m, m, y_m)
            add(mdl, "lower", k_direct, lower, y_l)
            add(mboth ^ mdl, "lower", dfunc(d_lower), d_lower, func(d_lower))
            add(mdu, "upper", k_direct, lower, y_l)
            add(mboth ^ mdu, "upper", dfunc(d_upper), d_upper, func(d_upper))
            y_l, y_u = func(lower), func(upper)
            add(sig & (y_l < y_u) & (d_lower >= m), "lower", k_m, m, y_m)
            add(sig & (y_l < y_u) & (d_upper < m), "upper", k_m, m, y_m)
            add(sig & (y_l >= y_u) & (d_lower < m), "lower", k_m, m, y_m)
            add(sig & (y_l >= y_u) & (d_upper >= m), "upper", k_m, m, y_m)
            bl_s, bl_b, bu_s, bu_b = self._branch(l, u)
        lw = np.where(sig, lw, bl_s); lb = np.where(sig, lb, bl_b)
        uw = np.where(sig, uw, bu_s); ub = np.where(sig, ub, bu_b)
        ro = 8 * EPS * (1 + np.maximum(np.abs(l), np.abs(u)))
        return lw, lb - ro, uw, ub + ro

    def relax_cos(self, l, u):
        hp = 0.5 * PI
        lw, lb, uw, ub = self.relax_sin(l + hp, u + hp)
        return lw, lb + lw * hp, uw, ub + uw * hp


# tie tolerance of the "exact" McCormick tie rule (the reference's rule is tie_tol = 0)
EXACT_TIE_TOL = 1e-12


def relax_mul(xl, xu, yl, yu, tie_tol=0.0):
    """McCormick with the coefficient-aware pick (bivariate.py:206-247, 38-77).

    Where both candidate planes have the same box minimum (maximum) in exact arithmetic --
    x entirely negative and y entirely positive, or the reverse, or a degenerate interval --
    the reference's float comparison is decided by rounding noise in its intermediate
    bounds. With tie_tol > 0 a relative difference below tie_tol counts as a tie and picks
    plane 1, the outcome of the reference's >= / <= comparisons in exact arithmetic.
    tie_tol = 0 is the reference's plain float comparison."""
    # lower candidates
    def amin(a, b, c):
        return a * np.where(a >= 0, xl, xu) + b * np.where(b >= 0, yl, yu) + c

    def amax(a, b, c):
        return a * np.where(a >= 0, xu, xl) + b * np.where(b >= 0, yu, yl) + c

    m1, m2 = amin(yl, xl, -xl * yl), amin(yu, xu, -xu * yu)
    M1, M2 = amax(yu, xl, -yu * xl), amax(yl, xu, -yl * xu)
    r_l = (m1 >= m2 - tie_tol * (np.abs(m1) + np.abs(m2))).astype(np.float64)
    r_u = (M1 <= M2 + tie_tol * (np.abs(M1) + np.abs(M2))).astype(np.float64)
    al = (yl - yu) * r_l + yu
    bl = (xl - xu) * r_l + xu
    gl = (yu * xu - yl * xl) * r_l - yu * xu
    au = (yu - yl) * r_u + yl
    bu = (xl - xu) * r_u + xu
    gu = (yl * xu - yu * xl) * r_u - yl * xu
    return al, bl, gl, au, bu, gu


# ============================================================ interval propagation
def ibp_sin(l, u, max_point, min_point, func=np.sin):
    """trigonometric.py:BoundSin.interval_propagate (BoundCos: cos, extrema at 0 and pi)."""
    def crossing(ll, uu, point):
        lc = (ll - point) / (2 * PI)
        uc = (uu - point) / (2 * PI)
        ro = 2 * EPS * (1 + np.maximum(np.abs(lc), np.abs(uc)))
        return (uu - ll >= 2 * PI) | (np.floor(uc + ro) > np.floor(lc - ro))

    with np.errstate(invalid="ignore"):
        fl, fu = func(l), func(u)
    hi = np.where(crossing(l, u, max_point), 1.0, np.maximum(fl, fu))
    lo = np.where(crossing(l, u, min_point), -1.0, np.minimum(fl, fu))
    return lo, hi


def ibp_node(n, ivs):
    """Interval of node n from its inputs' intervals ivs[i] = (lo, hi), each (B, w)."""
    k, a = n.kind, n.attrs
    with np.errstate(all="ignore"):
        if k in ("linear", "matmul"):
            lo, hi = ivs[0]
            W = a["W"].T if k == "linear" else a["W"]     # (in, out)
            bias = a.get("b") if k == "linear" else None
            mid = (lo + hi) / 2
            diff = (hi - lo) / 2
            center = mid @ W
            dev = diff @ np.abs(W)
            l_out, u_out = center - dev, center + dev
            if not (np.isfinite(lo).all() and np.isfinite(hi).all()):
                Wp, Wn = np.where(W > 0, W, 0), np.where(W < 0, W, 0)
                l_out = np.nan_to_num(lo @ Wp, nan=-np.inf) + np.nan_to_num(hi @ Wn, nan=-np.inf)
                u_out = np.nan_to_num(hi @ Wp, nan=np.inf) + np.nan_to_num(lo @ Wn, nan=np.inf)
            if bias is not None:
                l_out, u_out = l_out + bias, u_out + bias
            mag = finite_abs(np.maximum(np.abs(lo), np.abs(hi))) @ np.abs(W)
            nterm = W.shape[0]
            bmag = np.abs(bias) if bias is not None else 0.0
            err = rounding_error(mag + bmag, nterm)
            return widen(l_out, err, -1), widen(u_out, err, 1)
        if k == "mul":
            (xl, xu), (yl, yu) = ivs
            xl, xu = xl[:, a["map0"]], xu[:, a["map0"]]
            yl, yu = yl[:, a["map1"]], yu[:, a["map1"]]
            r = [xl * yl, xl * yu, xu * yl, xu * yu]
            nan = np.isnan(r[0]) | np.isnan(r[1]) | np.isnan(r[2]) | np.isnan(r[3])
            lo = np.fmin(np.fmin(r[0], r[1]), np.fmin(r[2], r[3]))
            hi = np.fmax(np.fmax(r[0], r[1]), np.fmax(r[2], r[3]))
            return np.where(nan, -np.inf, lo), np.where(nan, np.inf, hi)
        if k == "mulc":
            lo, hi = ivs[0]
            lo, hi = lo[:, a["map0"]], hi[:, a["map0"]]
            c = a["c"]
            lo2 = np.where(c > 0, lo * c, np.where(c < 0, hi * c, 0.0))
            hi2 = np.where(c > 0, hi * c, np.where(c < 0, lo * c, 0.0))
            return lo2, hi2
        if k in ("add", "sub", "addc", "subc", "rsubc"):
            if k in ("add", "sub"):
                (xl, xu), (yl, yu) = ivs
                xl, xu = xl[:, a["map0"]], xu[:, a["map0"]]
                yl, yu = yl[:, a["map1"]], yu[:, a["map1"]]
            else:
                xl, xu = ivs[0]
                xl, xu = xl[:, a["map0"]], xu[:, a["map0"]]
                yl = yu = np.broadcast_to(a["c"], xl.shape)
                if k == "rsubc":
                    xl, xu, yl, yu = yl, yu, xl, xu
            if k in ("add", "addc"):
                lo, hi = xl + yl, xu + yu
            else:
                lo, hi = xl - yu, xu - yl
            # _enclose_affine_interval (interval_bound.py:80-94)
            return (widen(lo, rounding_error(finite_abs(lo), 1), -1),
                    widen(hi, rounding_error(finite_abs(hi), 1), 1))
        if k == "neg":
            lo, hi = ivs[0]
            return -hi, -lo
        if k == "sqr":
            lo, hi = ivs[0]
            l2 = np.where(hi < 0, hi ** 2, np.where(lo > 0, lo ** 2, 0.0))
            return l2, np.maximum(lo ** 2, hi ** 2)
        if k == "pow":
            lo, hi = ivs[0]
            p = float(a["exponent"])
            if p == int(p):
                pl, pu = _pw(lo, int(p)), _pw(hi, int(p))
                if int(p) % 2 == 1:
                    return pl, pu
                cross = (lo < 0) & (hi > 0)
                return np.where(cross, 0.0, np.minimum(pl, pu)), np.maximum(pl, pu)
            return _pw(np.maximum(lo, 0.0), p), _pw(hi, p)
        if k == "exp":
            lo, hi = ivs[0]
            return np.exp(lo), np.exp(hi)
        if k == "log":
            lo, hi = ivs[0]
            lo = np.where(lo <= 0, 0.0, lo)
            return np.log(lo), np.log(hi)
        if k == "sin":
            lo, hi = ivs[0]
            return ibp_sin(lo, hi, PI / 2, PI * 3 / 2)
        if k == "cos":
            lo, hi = ivs[0]
            return ibp_sin(lo, hi, 0.0, PI, np.cos)
        if k == "reducesum":
            lo, hi = ivs[0]
            B = lo.shape[0]
            ol = np.zeros((B, n.width)); oh = np.zeros((B, n.width))
            np.add.at(ol.T, a["rmap"], lo.T)
            np.add.at(oh.T, a["rmap"], hi.T)
            return ol, oh
        if k in ("gather", "slice", "reshape", "unsqueeze", "squeeze", "flatten", "transpose"):
            lo, hi = ivs[0]
            return lo[:, a["map"]], hi[:, a["map"]]
        if k == "concat":
            lo = np.concatenate([v[0] for v in ivs], 1)[:, a["cmap"]]
            hi = np.concatenate([v[1] for v in ivs], 1)[:, a["cmap"]]
            return lo, hi
    raise NotImplementedError(k)


def _nan_to_inf(lo, hi):
    return np.where(np.isnan(lo), -np.inf, lo), np.where(np.isnan(hi), np.inf, hi)


# ============================================================ the oracle
class CrownOracle:
    """compute_bounds(method='CROWN') over a batch of boxes for a ``gear_b200.graph.Graph``."""

    def __init__(self, graph, tie_tol=0.0, inject=None):
        """inject: {node id: (lo, hi)} replaces the computed bounds of those nodes (used to
        check the restatement against recorded reference intermediates)."""
        self.tie_tol = tie_tol
        self.inject = inject or {}
        self.cuts = None
        self.g = graph
        self.sin = SinRelax()
        self.consumers = graph.consumers()
        self.anc = self._ancestors(graph.output)

    def _ancestors(self, t):
        seen, stack = set(), [t]
        while stack:
            v = stack.pop()
            if v in seen:
                continue
            seen.add(v)
            stack += self.g[v].inputs
        return seen

    # -------------------------------------------------------------- intervals
    def _interval(self, v, transient):
        """Current interval: stored bounds, else IBP from inputs (not stored)."""
        if v in self.bounds:
            return self.bounds[v]
        if v in transient:
            return transient[v]
        n = self.g[v]
        ivs = [self._interval(i, transient) for i in n.inputs]
        iv = _nan_to_inf(*ibp_node(n, ivs))
        transient[v] = iv
        return iv

    def _ibp_store(self, v):
        """IBP_general(v) with delete_bounds_after_use=False: inputs lacking bounds are stored too."""
        n = self.g[v]
        for i in n.inputs:
            if i not in self.bounds:
                self._ibp_store(i)
        self.bounds[v] = self.inject.get(v, _nan_to_inf(*ibp_node(n, [self.bounds[i] for i in n.inputs])))
        self.log.append(("ibp", v))

    def magnitude(self, v):
        lo, hi = self.bounds[v] if v in self.bounds else self.ibp0[v]
        return np.where(lo > hi, np.inf, np.maximum(-lo, hi))

    # -------------------------------------------------------------- relaxation cache
    def planes(self, v):
        if v in self.plane_cache:
            return self.plane_cache[v]
        n = self.g[v]
        k = n.kind
        if k == "mul":
            (xl, xu), (yl, yu) = self.bounds[n.inputs[0]], self.bounds[n.inputs[1]]
            xl, xu = xl[:, n.attrs["map0"]], xu[:, n.attrs["map0"]]
            yl, yu = yl[:, n.attrs["map1"]], yu[:, n.attrs["map1"]]
            bad = ~(np.isfinite(xl) & np.isfinite(xu) & np.isfinite(yl) & np.isfinite(yu))
            with np.errstate(all="ignore"):
                p = relax_mul(xl, xu, yl, yu, self.tie_tol)
            p = tuple(np.where(bad, 0.0, q) for q in p)
            res = ("mul", p, bad)
        else:
            l, u = self.bounds[n.inputs[0]]
            bad = ~(np.isfinite(l) & np.isfinite(u))
            if k == "log":
                bad = bad | ~(l > 0)
            off = np.zeros_like(bad)
            if k == "pow":
                # BoundPow.bound_backward raises the input node's stored upper bound to
                # lower + 1e-8 before relaxing (s_shaped.py:791, :801); the change persists
                i0 = n.inputs[0]
                with np.errstate(invalid="ignore"):
                    u = np.maximum(u, l + 1e-8)
                self.bounds[i0] = (self.bounds[i0][0], u)
                if i0 in self.computed:
                    c_l, c_u = self.computed[i0]
                    with np.errstate(invalid="ignore"):
                        self.computed[i0] = (c_l, np.maximum(c_u, c_l + 1e-8))
                l, u, off = pow_domain(l, u, float(n.attrs["exponent"]))
                bad = bad | off
            ls, us = np.where(bad, 0.0, l), np.where(bad, 1.0, u)
            if k == "sqr":
                p = relax_sqr(ls, us)
            elif k == "exp":
                p = relax_exp(ls, us)
            elif k == "log":
                p = relax_log(ls, us)
            elif k == "sin":
                p = self.sin.relax_sin(ls, us)
            elif k == "cos":
                p = self.sin.relax_cos(ls, us)
            elif k == "pow":
                with np.errstate(all="ignore"):
                    p = relax_pow(ls, us, float(n.attrs["exponent"]))
            else:
                raise NotImplementedError(k)
            p = tuple(np.where(bad, 0.0, q) for q in p)
            if bad.any():
                p, bad = self._stop_undefined(v, k, l, u, p, bad, off)
            res = ("unary", p, bad)
        self.plane_cache[v] = res
        return res

    def _stop_undefined(self, v, k, l, u, p, bad, off):
        """_stop_undefined_interval (backward_bound.py:249-292) on the elements whose relaxation is
        undefined (a non-finite input interval, log of an interval reaching 0): a coefficient that
        selects an undefined side uses the node's own interval (_node_interval: its stored bounds,
        else interval arithmetic from its inputs) as a constant plane, and only a non-finite
        constant still discards the row. The square is convex with a tangent below
        (require_finite_relaxation_bounds(convex_tangent_lower=True), operators/base.py:318-340):
        only its upper side is undefined and the lower tangent is built on the substitute interval
        (the finite endpoint, or 0 -/+ 1 when both are unbounded), unless the node's interval lies
        above the hull's lower end (backward_bound.py:384-392), where the lower side stops too.
        Off-domain pow elements (a fractional power entirely below 0) keep discarding their rows.
        No element stops when some element's interval is NaN or inverted. Returns (planes, the
        elements that still discard every row using them)."""
        lo_v, hi_v = self.bounds[v] if v in self.bounds else self._interval(v, {})
        if np.any(np.isnan(lo_v) | np.isnan(hi_v) | (lo_v > hi_v)):
            return p, bad
        lw, lb, uw, ub = p
        stop = bad & ~off
        no_lower, no_upper = stop.copy(), stop.copy()
        if k == "sqr":
            fl, fu = np.isfinite(l), np.isfinite(u)
            lf, uf = np.where(fl, l, 0.0), np.where(fu, u, 0.0)
            sl = np.where(fl, l, np.minimum(uf, 0.0) - 1.0)
            su = np.where(fu, u, np.maximum(lf, 0.0) + 1.0)
            tk, tb, _, _ = relax_sqr(sl, su)
            with np.errstate(invalid="ignore"):
                hull = np.where(u < 0, u * u, np.where(l > 0, l * l, 0.0))
            no_lower = stop & (lo_v > hull)
            tangent = stop & ~no_lower
            lw, lb = np.where(tangent, tk, lw), np.where(tangent, tb, lb)
        lw, lb = np.where(no_lower, 0.0, lw), np.where(no_lower, lo_v, lb)
        uw, ub = np.where(no_upper, 0.0, uw), np.where(no_upper, hi_v, ub)
        return (lw, lb, uw, ub), bad & off

    # -------------------------------------------------------------- backward
    def backward(self, t, C, lower=True, upper=True):
        """backward_general(t, C). C: (S, B, w_t). Returns lb, ub (B, S), lA (B, S, n), lbias."""
        g = self.g
        S, B = C.shape[0], C.shape[1]
        # get_degrees
        deg, added, q = {}, {t}, deque([t])
        while q:
            l = q.popleft()
            for p in g[l].inputs:
                deg[p] = deg.get(p, 0) + 1
                if p not in added:
                    q.append(p)
                    added.add(p)
        A = {t: [C.copy() if lower else None, C.copy() if upper else None]}
        bias = [np.zeros((S, B)), np.zeros((S, B))]
        bias_mag = [np.zeros((S, B)), np.zeros((S, B))]
        err = [np.zeros((S, B)), np.zeros((S, B))]
        undef = [np.zeros((S, B), bool), np.zeros((S, B), bool)]
        # contributions into each node in this pass (merge-rounding factor K_p)
        reach, K = {t}, {}
        q2, deg2 = deque([t]), dict(deg)
        while q2:
            l = q2.popleft()
            if l == 0:
                continue
            for p in g[l].inputs:
                deg2[p] -= 1
                if deg2[p] == 0:
                    q2.append(p)
            if l in reach:
                for p in g[l].inputs:
                    reach.add(p)
                    K[p] = K.get(p, 0) + 1
        queue = deque([t])
        nvisit = 0
        while queue:
            l = queue.popleft()
            if l == 0:
                continue
            n = g[l]
            for p in n.inputs:
                deg[p] -= 1
                if deg[p] == 0:
                    queue.append(p)
            if l not in A:
                continue
            nvisit += 1
            lA, uA = A.pop(l)
            outs = self._node_backward(n, lA, uA, bias, bias_mag, err, undef)
            for side in (0, 1):
                if (lA, uA)[side] is None:
                    continue
                for i, p in enumerate(n.inputs):
                    new = outs[i][side]
                    if new is None:
                        continue
                    if p not in A:
                        A[p] = [None, None]
                    old = A[p][side]
                    if K.get(p, 0) >= 2:
                        # merge rounding: the K_p additions into A_p err by at most
                        # gamma(K_p) sum_i |contribution_i| (charged per contribution) on the
                        # finite magnitudes; on an unbounded entry only an addition that rounded
                        # costs (+inf), by TwoSum (_merge_charge, backward_bound.py:740-752)
                        m = self.magnitude(p)
                        unb = np.isinf(m)
                        err[side] += gamma(K[p]) * abs_dot(np.abs(new), np.where(unb, 0.0, m)[None])
                        if old is not None and unb.any():
                            with np.errstate(all="ignore"):
                                tot_ = old + new
                                bv = tot_ - old
                                e2 = (old - (tot_ - bv)) + (new - bv)
                            e2 = np.where(np.isfinite(tot_), e2, np.inf)
                            err[side] += np.where(((e2 != 0) & unb[None]).any(-1), np.inf, 0.0)
                    A[p][side] = new if old is None else old + new
        # concretisation at the input
        xL, xU = self.xL, self.xU
        x0 = (xU + xL) / 2.0
        eps = (xU - xL) / 2.0
        maxabs = finite_abs(np.maximum(np.abs(xL), np.abs(xU)))
        nin = g[0].width
        res, resA = [None, None], [None, None]
        for side, sign in ((0, -1.0), (1, 1.0)):
            if not (lower, upper)[side]:
                continue
            Ax = A.get(0, [None, None])[side]
            if Ax is None:
                Ax = np.zeros((S, B, nin))
            # combined outward rounding: every magnitude is scaled by its rounding factor and
            # added to one error term (bias sums over visits + n terms, the box dot over n terms)
            f_bias = (max(nvisit, 1) + nin + 16) * EPS * 4
            f_box = (nin + 16) * EPS * 4
            if self.cuts is not None:
                # concretisation over box ∩ cut rows (PerturbationLpNorm(constraints=...):
                # constraints_solving, concretize_func.py:431-850, with its own rounding and the
                # box bound as floor); an upper bound is minus the lower bound of -A
                from .concretize import constrained_lower
                cA, cb, cmax = self.cuts
                with np.errstate(all="ignore"):
                    obj = np.ascontiguousarray((Ax if side == 0 else -Ax).transpose(1, 0, 2))
                    v = constrained_lower(xL, xU, obj, cA, cb, cmax).T
                base = v if side == 0 else -v
                dev = np.zeros_like(base)
                val = bias[side] + base
                errt = err[side] + bias_mag[side] * f_bias
            else:
                base = np.einsum("sbx,bx->sb", Ax, x0)
                dev = np.einsum("sbx,bx->sb", np.abs(Ax), eps)
                bmag = np.einsum("sbx,bx->sb", finite_abs(Ax), maxabs)
                val = bias[side] + base
                errt = err[side] + bias_mag[side] * f_bias + bmag * f_box + dev
            with np.errstate(invalid="ignore"):
                tot = val + sign * (errt + (np.abs(val) + errt) * (17 * EPS * 4))
            bad = undef[side] | np.isnan(tot) | (tot == -sign * np.inf)
            tot = np.where(bad, sign * np.inf, tot)
            undef[side] = bad
            res[side] = tot.T.copy()
            root = base + sign * dev
            Ax = np.where(bad[:, :, None], 0.0, Ax)
            # save_root_A (backward_bound.py:1629): lbias = bound minus the root's term
            with np.errstate(invalid="ignore"):
                lbias = np.where(bad, sign * np.inf, tot - root)
            resA[side] = (Ax.transpose(1, 0, 2).copy(), lbias.T.copy())
        return res[0], res[1], resA, (undef[0].T.copy(), undef[1].T.copy())

    def _node_backward(self, n, lA, uA, bias, bias_mag, err, undef):
        """bound_backward of node n for both sides; returns [(lA_in, uA_in) per input]."""
        k, a = n.kind, n.attrs
        g = self.g
        outs = [[None, None] for _ in n.inputs]
        sides = [(0, lA), (1, uA)]

        def scatter(Aout, m, w_in):
            S, B, _ = Aout.shape
            res = np.zeros((S, B, w_in))
            np.add.at(res.transpose(2, 0, 1), m, Aout.transpose(2, 0, 1))
            return res

        for side, Am in sides:
            if Am is None:
                continue
            S, B, w = Am.shape
            if k in ("linear", "matmul"):
                Wt = a["W"] if k == "linear" else a["W"].T     # (out, in)
                outs[0][side] = Am @ Wt
                if k == "linear" and a.get("b") is not None:
                    bt = Am @ a["b"]
                    bias[side] += bt
                    bias_mag[side] += np.abs(Am) @ np.abs(a["b"])
                m_in = self.magnitude(n.inputs[0])
                t = np.nan_to_num(np.abs(Wt) @ np.where(np.isinf(m_in), 0.0, m_in).T, nan=0.0)  # (out, B)
                err[side] += gamma(w) * np.einsum("sbo,ob->sb", np.abs(Am), t)
            elif k == "mulc":
                c = a["c"]
                newA = Am * c
                outs[0][side] = scatter(newA, a["map0"], g[n.inputs[0]].width)
                m_in = self.magnitude(n.inputs[0])[:, a["map0"]]
                exact = (c == 0) | (np.abs(np.frexp(c)[0]) == 0.5)
                # on unbounded inputs only a product that rounded costs (+inf): the exact error of
                # A * c by TwoProduct (_affine_backward_terms, backward_bound.py:611-640)
                unb = np.isinf(m_in)
                m_fin = np.where(unb, 0.0, m_in)
                e = U * abs_dot(np.abs(np.where(exact, 0.0, newA)), m_fin[None])
                rounded = (two_product_error(Am, np.broadcast_to(c, Am.shape)) != 0) & unb[None]
                err[side] += np.where(rounded.any(-1), np.inf, e)
            elif k in ("add", "sub", "addc", "subc", "rsubc"):
                mx = self.magnitude(n.inputs[0])[:, a["map0"]]
                if k in ("add", "sub"):
                    outs[0][side] = scatter(Am, a["map0"], g[n.inputs[0]].width)
                    sgn = 1.0 if k == "add" else -1.0
                    outs[1][side] = scatter(sgn * Am, a["map1"], g[n.inputs[1]].width)
                    my = self.magnitude(n.inputs[1])[:, a["map1"]]
                else:
                    sgn = -1.0 if k == "rsubc" else 1.0
                    outs[0][side] = scatter(sgn * Am, a["map0"], g[n.inputs[0]].width)
                    cval = a["c"] if k != "subc" else -a["c"]
                    cb = Am @ cval
                    bias[side] += cb
                    bias_mag[side] += np.abs(Am) @ np.abs(cval)
                    my = np.abs(a["c"])[None, :]
                # Add/Sub output rounding (_affine_output_error, interval_bound.py:71-77); an
                # unbounded output entry adds nothing (its magnitude counts as 0, as in the
                # deferred charge of _enclose_affine_backward, backward_bound.py:780-787)
                with np.errstate(invalid="ignore"):
                    e = rounding_error(mx + my, 2)
                e = np.where(np.isinf(e), 0.0, e)
                err[side] += abs_dot(finite_abs(Am), e[None])
            elif k == "neg":
                outs[0][side] = -Am
            elif k == "reducesum":
                outs[0][side] = Am[:, :, a["rmap"]]
            elif k in ("gather", "slice", "reshape", "unsqueeze", "squeeze", "flatten", "transpose"):
                outs[0][side] = scatter(Am, a["map"], g[n.inputs[0]].width)
            elif k == "concat":
                off = 0
                inv = np.argsort(a["cmap"], kind="stable")     # concat-position -> output element
                for i, p in enumerate(n.inputs):
                    w_i = g[p].width
                    outs[i][side] = Am[:, :, inv[off:off + w_i]]
                    off += w_i
            elif k == "mul":
                _, (al, bl, gl, au, bu, gu), bad = self.planes(n.id)
                Ap, An = np.maximum(Am, 0), np.minimum(Am, 0)
                if side == 0:
                    px, py, pg, nx, ny, ng = al, bl, gl, au, bu, gu
                else:
                    px, py, pg, nx, ny, ng = au, bu, gu, al, bl, gl
                Ax = np.where(Ap == 0, 0.0, px * Ap) + np.where(An == 0, 0.0, nx * An)
                Ay = np.where(Ap == 0, 0.0, py * Ap) + np.where(An == 0, 0.0, ny * An)
                bt = (np.where(Ap == 0, 0.0, Ap * pg) + np.where(An == 0, 0.0, An * ng))
                bias[side] += bt.sum(-1)
                bias_mag[side] += np.abs(bt).sum(-1)
                undef[side] |= ((Am != 0) & bad[None]).any(-1)
                outs[0][side] = scatter(Ax, a["map0"], g[n.inputs[0]].width)
                outs[1][side] = scatter(Ay, a["map1"], g[n.inputs[1]].width)
            else:
                _, (lw, lb, uw, ub), bad = self.planes(n.id)
                Ap, An = np.maximum(Am, 0), np.minimum(Am, 0)
                if side == 0:
                    wp, bp, wn, bn = lw, lb, uw, ub
                else:
                    wp, bp, wn, bn = uw, ub, lw, lb
                with np.errstate(invalid="ignore"):
                    newA = np.where(Ap == 0, 0.0, wp * Ap) + np.where(An == 0, 0.0, wn * An)
                    bt = np.where(Ap == 0, 0.0, Ap * bp) + np.where(An == 0, 0.0, An * bn)
                rowbad = ((Am != 0) & bad[None]).any(-1) | ~np.isfinite(bt).all(-1) | ~np.isfinite(newA).all(-1)
                undef[side] |= rowbad
                bt = np.where(np.isfinite(bt), bt, 0.0)
                newA = np.where(np.isfinite(newA), newA, 0.0)
                bias[side] += bt.sum(-1)
                bias_mag[side] += np.abs(bt).sum(-1)
                outs[0][side] = newA
        return outs

    # -------------------------------------------------------------- driver
    def compute_bounds(self, xL, xU, C=None, bound_upper=False, constraints=None, max_rows=0):
        """lb (B, S), ub or None, A = (lA (B, S, n), lbias (B, S)). constraints = (A (B, K, n),
        b (B, K)): rows A x + b <= 0 that every concretisation, intermediate passes included,
        intersects with the box (PerturbationLpNorm(constraints=...)); max_rows caps the rows a
        box sweeps (MAX_CONSTRAINT_ROWS)."""
        g = self.g
        self.cuts = None if constraints is None else (np.asarray(constraints[0], np.float64),
                                                      np.asarray(constraints[1], np.float64), int(max_rows))
        self.xL = np.asarray(xL, dtype=np.float64).reshape(xL.shape[0], -1)
        self.xU = np.asarray(xU, dtype=np.float64).reshape(xU.shape[0], -1)
        B = self.xL.shape[0]
        self.bounds: Dict[int, Tuple[np.ndarray, np.ndarray]] = {0: (self.xL, self.xU)}
        self.plane_cache = {}
        self.computed = {}
        self.log: List[tuple] = []
        # plain IBP over the input box: magnitudes of non-bounded nodes
        self.ibp0 = {0: (self.xL, self.xU)}
        for n in g.nodes[1:]:
            self.ibp0[n.id] = _nan_to_inf(*ibp_node(n, [self.ibp0[i] for i in n.inputs]))
        t = g.output
        wt = g[t].width
        if C is None:
            C = np.broadcast_to(np.eye(wt), (B, wt, wt))
        C = np.asarray(C, dtype=np.float64)
        self.prior_checked = set()
        self._check_prior_bounds(t, C)
        Cs = C.transpose(1, 0, 2)
        lb, ub, A, und = self.backward(t, Cs, lower=True, upper=bound_upper)
        lb, ub = self._interval_fallback(t, C, lb, ub, und)
        self.log.append(("final", t))
        return lb, ub, A[0][0], A[0][1]

    def _interval_fallback(self, t, C, lb, ub, und):
        """_interval_fallback_rows (backward_bound.py:826): discarded rows of a dense C."""
        if not (und[0].any() or (ub is not None and und[1].any())):
            return lb, ub
        lo, hi = self._interval(t, {})
        val_l = (np.where(C > 0, C * lo[:, None, :], 0.0) + np.where(C < 0, C * hi[:, None, :], 0.0)).sum(-1)
        lb = np.where(und[0], np.fmax(lb, val_l), lb)
        if ub is not None:
            val_u = (np.where(C > 0, C * hi[:, None, :], 0.0) + np.where(C < 0, C * lo[:, None, :], 0.0)).sum(-1)
            ub = np.where(und[1], np.fmin(ub, val_u), ub)
        return lb, ub

    def _check_prior_bounds(self, v, C=None):
        """bound_general.py:1032-1079."""
        n = self.g[v]
        if v in self.prior_checked or v not in self.anc or n.kind == "input":
            return
        if C is not None and n.kind == "concat":
            Cs = np.abs(C).sum(axis=(0, 1))
            inv = np.argsort(n.attrs["cmap"], kind="stable")
            off = 0
            for p in n.inputs:
                w = self.g[p].width
                if (Cs[inv[off:off + w]].sum() != 0):
                    self._check_prior_bounds(p)
                off += w
        else:
            for p in n.inputs:
                self._check_prior_bounds(p)
        for i, p in enumerate(n.inputs):
            if i in n.requires_input_bounds or self.g[p].has_constraint:
                self._compute_intermediate(p)
        self.prior_checked.add(v)

    def _compute_intermediate(self, v):
        """bound_general.py:1081-1222 for an intermediate node."""
        if v in self.bounds:
            return
        n = self.g[v]
        # check_IBP_intermediate (interval_bound.py:310-354)
        if n.kind == "reshape" and n.inputs[0] in self.bounds:
            lo, hi = self.bounds[n.inputs[0]]
            self.bounds[v] = self.inject.get(v, (lo[:, n.attrs["map"]], hi[:, n.attrs["map"]]))
            self.log.append(("ibp", v))
            return
        chain, cur, ok = [], v, True
        while cur not in self.bounds:
            if not self.g[cur].ibp_intermediate:
                ok = False
                break
            chain.append(cur)
            cur = self.g[cur].inputs[0]
        if ok:
            for c in reversed(chain):
                self._ibp_store(c)
            return
        # check_IBP_first_linear (interval_bound.py:357-390): BoundLinear on the input
        if n.kind == "linear" and n.inputs[0] == 0:
            self._ibp_store(v)
            return
        B = self.xL.shape[0]
        w = n.width
        C = np.broadcast_to(np.eye(w)[:, None, :], (w, B, w))
        lb, ub, _, und = self.backward(v, C, lower=True, upper=True)
        lb, ub = _nan_to_inf(lb, ub)
        if und[0].any() or und[1].any():
            Cb = np.broadcast_to(np.eye(w), (B, w, w))
            lb, ub = self._interval_fallback(v, Cb, lb, ub, und)
        self.log.append(("crown", v))
        # compare_with_IBP: IBP of v from its inputs' current intervals
        trans = {}
        ilo, ihi = _nan_to_inf(*ibp_node(n, [self._interval(p, trans) for p in n.inputs]))
        self.computed[v] = (np.fmax(lb, ilo), np.fmin(ub, ihi))
        self.bounds[v] = self.inject.get(v, self.computed[v])


def ibp_output(graph, xL, xU, C=None):
    """IBP_general(final, C) on plain IBP intervals: the IBP pre-pass of
    get_lower_bound_with_ibp_enhancement (complete_verifier/input_split/bounding.py:789)."""
    iv = {0: (np.asarray(xL, np.float64), np.asarray(xU, np.float64))}
    for n in graph.nodes[1:]:
        iv[n.id] = _nan_to_inf(*ibp_node(n, [iv[i] for i in n.inputs]))
    lo, hi = iv[graph.output]
    if C is None:
        return lo, hi
    # BoundLinear._bound_box (operators/linear.py:621-653)
    if np.isfinite(lo).all() and np.isfinite(hi).all():
        mid, rad = (lo + hi) / 2, (hi - lo) / 2
        center = np.einsum("bsw,bw->bs", C, mid)
        dev = np.einsum("bsw,bw->bs", np.abs(C), rad)
        low, up = center - dev, center + dev
    else:
        with np.errstate(invalid="ignore"):
            low = (np.where(C > 0, C * lo[:, None], 0.0) + np.where(C < 0, C * hi[:, None], 0.0)).sum(-1)
            up = (np.where(C > 0, C * hi[:, None], 0.0) + np.where(C < 0, C * lo[:, None], 0.0)).sum(-1)
    mag = np.einsum("bsw,bw->bs", finite_abs(C), finite_abs(np.maximum(np.abs(lo), np.abs(hi))))
    err = rounding_error(mag, C.shape[-1])
    return _nan_to_inf(widen(low, err, -1), widen(up, err, 1))
