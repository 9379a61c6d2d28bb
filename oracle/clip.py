"""CPU oracle of domain clipping (numpy, float64): shrink boxes along each coordinate to the
part where every plane lA_s x + lbias_s can still be <= thr_s.

TEST INFRASTRUCTURE ONLY: the device kernel (clip_kernel in gear_b200/csrc/bab_kernels.cuh)
is checked against it by tests/. It restates clip_domains / _clip_main_fn
(solver/complete_verifier/input_split/clip.py:138-470, lower-bound planes, no base input rows)
and is pinned to the reference by tests/golden/make_clip_golden.py.
"""
import numpy as np

EPS = float(np.finfo(np.float64).eps)
TINY = float(np.finfo(np.float64).tiny)


def finite_abs(v):
    return np.where(np.isfinite(v), np.abs(v), 0.0)


def underflow(n):
    """_underflow (clip.py:131-135)."""
    return (n + 16) * TINY * EPS


def box_rounding_error(lA, xl, xu, lbias):
    """fp_enclosure.box_rounding_error with a bias: (|A| max|x| + |bias|) (n + 16) 4 eps."""
    m = finite_abs(np.maximum(np.abs(xl), np.abs(xu)))
    mag = np.einsum("bsn,bn->bs", finite_abs(lA), m) + finite_abs(lbias)
    return mag * ((lA.shape[-1] + 16) * EPS * 4)


def concretize(xl, xu, lA, lbias):
    """concretize_bounds (clip.py:472-486), lower planes."""
    xhat, eps = (xu + xl) / 2, (xu - xl) / 2
    return np.einsum("bsn,bn->bs", lA, xhat) - np.einsum("bsn,bn->bs", np.abs(lA), eps) + lbias


def concretize_error(lA, xl, xu, lbias):
    """_concretize_error (clip.py:138-144)."""
    n = lA.shape[-1]
    return box_rounding_error(lA, xl, xu, lbias) * ((n + 4) / (4 * (n + 16))) + underflow(n)


def clip_main(xl, xu, lA, lbias, thr, dm_lb, num_iters, dm_lb_err):
    """_clip_main_fn (clip.py:147-198), is_lower."""
    n = lA.shape[-1]
    thr = thr[:, :, None]
    dm_lb = dm_lb[:, :, None]
    for it in range(num_iters):
        xhat, eps = (xu + xl) / 2, (xu - xl) / 2
        if it > 0:
            dm_lb = concretize(xl, xu, lA, lbias)[:, :, None]
            dm_lb_err = concretize_error(lA, xl, xu, lbias)
        ax = lA * xhat[:, None, :]
        ae = np.abs(lA) * eps[:, None, :]
        cmo = dm_lb - ax + ae
        num = thr - cmo
        mag = finite_abs(thr) + finite_abs(dm_lb) + finite_abs(ax) + finite_abs(ae)
        err = mag * (4 * EPS) + underflow(n) + dm_lb_err[:, :, None]
        fin = np.isfinite(num)
        lo_n = np.where(fin, num - err, num)
        hi_n = np.where(fin, num + err, num)
        with np.errstate(divide="ignore", invalid="ignore"):
            q_lo, q_hi = lo_n / lA, hi_n / lA
        cu = np.nextafter(np.maximum(q_lo, q_hi), np.inf)
        cl = np.nextafter(np.minimum(q_lo, q_hi), -np.inf)
        cand_u = np.where(lA > 0, cu, np.inf)
        cand_l = np.where(lA < 0, cl, -np.inf)
        xu = np.minimum(cand_u.min(1), xu)
        xl = np.maximum(cand_l.max(1), xl)
    return xl, xu


def clip_domains(xl, xu, thr, lA, lbias, num_iters=1):
    """clip_domains (clip.py:237-470) for lower planes without base input rows: boxes whose
    data are not finite stay as they are; a box some plane already proves done becomes empty
    (x_L[0] = next double above x_U[0]); the others are clipped."""
    xl = np.array(xl, np.float64, copy=True)
    xu = np.array(xu, np.float64, copy=True)
    lA = np.asarray(lA, np.float64)
    lbias = np.asarray(lbias, np.float64)
    thr = np.asarray(thr, np.float64)
    ok = (np.isfinite(lA).all((1, 2)) & (np.isfinite(thr) | np.isposinf(thr)).all(1) & np.isfinite(lbias).all(1))
    idx = np.nonzero(ok)[0]
    if idx.size == 0:
        return xl, xu
    l, u, A, bb, t = xl[idx], xu[idx], lA[idx], lbias[idx], thr[idx]
    dm_lb = concretize(l, u, A, bb)
    cert_lb = dm_lb - box_rounding_error(A, l, u, bb) - underflow(A.shape[-1])
    err = concretize_error(A, l, u, bb)
    cert = (cert_lb > t).any(1)
    l[cert, 0] = np.nextafter(u[cert, 0], np.inf)
    un = ~cert
    if un.any():
        l2, u2 = clip_main(l[un], u[un], A[un], bb[un], t[un], dm_lb[un], num_iters, err[un])
        l[un], u[un] = l2, u2
    xl[idx], xu[idx] = l, u
    return xl, xu
