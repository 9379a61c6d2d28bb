"""CPU oracle of constrained concretisation (numpy, float64): the box-plus-linear-rows lower
bound of an objective by the reference's sequential dual sweep.

TEST INFRASTRUCTURE ONLY: the device kernels (gear_b200/csrc/concretize_kernels.cuh) are
checked against these functions by tests/. Reference paths are relative to
solver/auto_LiRPA; the reference's own functions pin this restatement through
tests/golden/make_concretize_golden.py.

Problem: for every box b and objective row h, a lower bound of min c_h^T x over
{x_L <= x <= x_U, A_k^T x + b_k <= 0 for every row k}. Rows are in standard form
(construct_constraints, concretize_func.py:51-97).
"""
import numpy as np

EPS = float(np.finfo(np.float64).eps)


def finite_abs(v):
    """fp_enclosure.py:8-10."""
    v = np.asarray(v, np.float64)
    return np.where(np.isfinite(v), np.abs(v), 0.0)


def rounding_error(mag, n, bias=0.0):
    """fp_enclosure.py:37-52: (|dot| + |bias|) (n + 16) 4 eps."""
    return (mag + finite_abs(bias)) * ((n + 16) * EPS * 4)


def widen(bound, err, sign):
    """fp_enclosure.py:55-61."""
    out = np.where(np.isfinite(bound), bound + sign * err, bound)
    return np.where(np.isposinf(err), sign * np.inf, out)


def box_rounding_error(A, xl, xu, bias=0.0):
    """fp_enclosure.py:64-84 for a dense A (..., N, X) and boxes (B, X)."""
    m = finite_abs(np.maximum(np.abs(xl), np.abs(xu)))           # (B, X)
    mag = np.einsum("bnx,bx->bn", finite_abs(A), m)
    return rounding_error(mag, A.shape[-1], bias)


def finite_rows(A, b):
    """_finite_constraints (concretize_func.py:100-103): a row with a non-finite entry
    becomes 0 x - 1 <= 0."""
    valid = np.isfinite(A).all(-1) & np.isfinite(b)
    return np.where(valid[..., None], A, 0.0), np.where(valid, b, -1.0)


def sort_out(xl, xu, A, b):
    """sort_out_constr_batches (concretize_func.py:312-412) without rearrangement.

    Returns (all_covered, infeasible (B,), covered (B,), A (B,K,X), d (B,K)): d is the centred
    offset A x0 + b rounded down by box_rounding_error(A, x0, x0, b)."""
    x0 = (xl + xu) / 2
    eps = (xu - xl) / 2
    sA, sb = finite_rows(A, b)
    # _sort_out_constraints (concretize_func.py:106-136)
    x0_term = np.einsum("bkx,bx->bk", sA, x0) + sb
    eps_term = np.einsum("bkx,bx->bk", np.abs(sA), eps)
    err = box_rounding_error(sA, x0 - eps, x0 + eps, sb)
    lo_v = widen(x0_term - eps_term, err, -1)
    hi_v = widen(x0_term + eps_term, err, 1)
    infeasible = (lo_v > 0).any(1)
    covered = (hi_v <= 0).all(1)
    if covered.all():
        return True, infeasible, covered, None, None
    d = np.einsum("bkx,bx->bk", A, x0) + b
    d = widen(d, box_rounding_error(A, x0, x0, b), -1)
    A2, d2 = finite_rows(A, d)
    return False, infeasible, covered, A2, d2


def kept_rows(A, d, eps, max_rows=0):
    """drop_redundant_constraints (concretize_func.py:269-309) for one batch.

    Returns (row lists per box, K): each box's non-redundant rows in their original order
    (at most max_rows of them, the largest worst-case values, when the batch maximum exceeds
    max_rows), and K, the row count the reference's sweep iterates (the batch maximum, at
    least 1; rows a box lacks are inert padding)."""
    max_val = d + np.einsum("bkx,bx->bk", np.abs(A), eps)
    redundant = max_val <= 0
    n_keep = max(int((~redundant).sum(1).max()), 1)
    rows = []
    if max_rows and n_keep > max_rows:
        score = np.where(redundant, -np.inf, np.nan_to_num(max_val, nan=np.inf))
        for b in range(A.shape[0]):
            order = np.lexsort((np.arange(A.shape[1]), -score[b]))[:max_rows]
            keep = sorted(int(k) for k in order if not redundant[b, k])
            rows.append(keep)
        return rows, max_rows
    for b in range(A.shape[0]):
        rows.append([k for k in range(A.shape[1]) if not redundant[b, k]])
    return rows, n_keep


def solve_dual_var(a, c, d, e):
    """_solve_dual_var (concretize_func.py:168-247) for one objective row: the multiplier
    beta >= 0 maximising -|c + beta a|^T e + beta d, at the first breakpoint -c_i / a_i (in
    ascending order) where the slope turns non-positive; +inf when it never does."""
    with np.errstate(divide="ignore", invalid="ignore"):
        q = -(c / a)
    order = np.argsort(q, kind="stable")
    w = np.abs(a * e)[order]
    P = np.concatenate([[0.0], np.cumsum(w)])            # sequential prefix sums
    grad = (P - P[-1]) + P - d
    j = int(np.searchsorted(grad, 0.0, side="left"))
    qn = np.concatenate([[0.0], q[order], [np.inf]])
    return max(qn[j], 0.0) if not np.isnan(qn[j]) else qn[j]


def constrained_lower(xl, xu, obj, A, b, max_rows=0):
    """sort_out_constr_batches + constraints_solving(sign=-1, no_return_inf=False)
    (concretize_func.py:415-850): lower bounds (B, H) of obj (B, H, X) . x over the boxes
    intersected with the rows A (B, K, X) x + b (B, K) <= 0. An infeasible box gets +inf."""
    xl = np.asarray(xl, np.float64)
    xu = np.asarray(xu, np.float64)
    obj = np.asarray(obj, np.float64)
    B, H, X = obj.shape
    x0 = (xu + xl) / 2.0
    eps = (xu - xl) / 2.0
    # naive (box) bound and the objective's own rounding (concretize_func.py:596-619)
    obj_err = box_rounding_error(obj, xl, xu)                      # (B, H)
    base = np.einsum("bhx,bx->bh", obj, x0)
    naive = widen(base - np.einsum("bhx,bx->bh", np.abs(obj), eps), obj_err, -1)
    naive = np.where(np.isfinite(naive), naive, -np.inf)
    if A is None or np.asarray(A).size == 0:
        return naive
    all_cov, infeasible, covered, Ac, dc = sort_out(xl, xu, np.asarray(A, np.float64), np.asarray(b, np.float64))
    if all_cov:
        return naive
    out = naive.copy()
    act = np.nonzero(~covered)[0]
    rows, K = kept_rows(Ac[act], dc[act], eps[act], max_rows)
    for ai, bi in enumerate(act):
        e = eps[bi]
        for h in range(H):
            c = obj[bi, h].copy()
            cmag = finite_abs(np.abs(c))
            dual = 0.0
            dmag = 0.0
            for k in rows[ai]:
                a = Ac[bi, k]
                beta = solve_dual_var(a, c, dc[bi, k], e)
                upd = beta * a
                c = c + upd
                cmag = cmag + finite_abs(upd)
                dual += beta * dc[bi, k]
                dmag = dmag + float(finite_abs(beta * dc[bi, k]))
            eps_term = float(np.abs(c) @ e)
            dual -= eps_term
            dmag = dmag + float(finite_abs(eps_term)) + float(cmag @ finite_abs(e))
            val = base[bi, h] + dual
            err = obj_err[bi, h] + rounding_error(dmag, X + K, base[bi, h])
            val = float(widen(np.float64(val), np.float64(err), -1))
            out[bi, h] = val if np.isfinite(val) else naive[bi, h]
    out = np.maximum(out, naive)
    return np.where(infeasible[:, None], np.inf, out)
