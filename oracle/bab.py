"""CPU oracle of the branch-and-bound select / prune / branch / split step (numpy).

TEST INFRASTRUCTURE ONLY: the product's device kernels (gear_b200/csrc/bab_kernels.cuh)
are checked against these functions by tests/. Reference paths are relative to
solver/complete_verifier/input_split.
"""
import math

import numpy as np

EPS = float(np.finfo(np.float64).eps)


def prune_mask(lb, thr):
    """get_remaining_index (branching_domains.py:412-558), solving mode, check_dm_lbs.

    Returns (keep (B,) bool, discarded threshold minimum or +inf)."""
    lb = np.asarray(lb, np.float64)
    thr = np.asarray(thr, np.float64)
    fin = np.isfinite(lb) & np.isfinite(thr)
    gt = fin & (lb > thr)
    gt[:, 0] |= fin[:, 0] & (lb[:, 0] >= thr[:, 0])
    verified = gt.any(1) | (np.isposinf(lb[:, 0]) & np.isfinite(thr[:, 0]))
    disc = thr[verified][:, 0]
    disc = disc[np.isfinite(disc)]
    return ~verified, (float(disc.min()) if disc.size else math.inf)


def sb_branch(lA, lo, hi, lb, thr, root_width=None, coeff_thresh=1e-3, min_width_ratio=0.001):
    """input_split_branching with method 'sb', sb_sum (branching_heuristics.py:25-125,
    :176-202). Ties pick the lowest index."""
    lA = np.asarray(lA, np.float64)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    thr = np.where(np.isposinf(thr), lb, thr)
    width = hi - lo
    nonfinite = not (np.isfinite(lA).all() and np.isfinite(lb).all() and np.isfinite(thr).all())
    if nonfinite:
        return np.argmax(width, axis=1).astype(np.int64)
    raw = np.maximum(np.abs(lA), coeff_thresh) * width[:, None, :] / 2
    score = np.zeros(width.shape)
    for s in range(lA.shape[1]):            # sequential over the specification rows
        score = score + raw[:, s, :]
    idx = np.argmax(score, axis=1)          # first maximal index
    if root_width is not None and min_width_ratio > 0:
        rw = np.asarray(root_width, np.float64).reshape(1, -1)
        rel = np.where(rw > 0, width / np.maximum(rw, 1e-300), 0.0)
        rel_max = rel.max(1)
        widest = np.argmax(rel, axis=1)
        chosen = rel[np.arange(len(idx)), idx]
        idx = np.where(chosen < min_width_ratio * rel_max, widest, idx)
    return idx.astype(np.int64)


def split(lo, hi, kept, idx):
    """input_split_parallel (split.py:26-122) of the kept boxes: [upper halves; lower halves]."""
    lo = np.asarray(lo, np.float64)[kept]
    hi = np.asarray(hi, np.float64)[kept]
    i = np.asarray(idx)[kept]
    K = len(kept)
    out_l, out_u = [], []
    for part in range(2):
        l2, u2 = lo.copy(), hi.copy()
        a, b = lo[np.arange(K), i], hi[np.arange(K), i]
        l2[np.arange(K), i] = ((part + 1) * a + (2 - part - 1) * b) / 2
        u2[np.arange(K), i] = (part * a + (2 - part) * b) / 2
        out_l.append(l2)
        out_u.append(u2)
    return np.concatenate(out_l), np.concatenate(out_u)


def child_keys(lb, lA, lbias, child_lo, child_hi, kept):
    """_raise_child_keys / _plane_minimum_down (batch_branch_and_bound.py:189-225) with the
    parents' rows repeated for both children."""
    kept = np.asarray(kept)
    par = np.concatenate([kept, kept])
    keys = np.asarray(lb, np.float64)[par].copy()
    a = np.asarray(lA, np.float64)[par][:, 0, :]
    b = np.asarray(lbias, np.float64)[par][:, 0]
    c, r = (child_lo + child_hi) / 2, (child_hi - child_lo) / 2
    plane = (a * c - np.abs(a) * r).sum(1) + b
    n = child_lo.shape[1]
    margin = (n + 4) * EPS / 2 * ((np.abs(a) * (np.abs(c) + r)).sum(1) + np.abs(b))
    pmin = np.nextafter(plane - margin, -np.inf)
    usable = (child_lo <= child_hi).all(1) & np.isfinite(pmin)
    keys[:, 0] = np.where(usable, np.maximum(keys[:, 0], pmin), keys[:, 0])
    return keys


def queue_order(key, ids):
    """Descending key, stable by insertion id (the reference's lb sort, branching_domains.py:1171,
    with stable tie-breaking); the batch is popped from the end of this order."""
    key = np.asarray(key, np.float64)
    ids = np.asarray(ids)
    return np.lexsort((ids, -key))
