"""The domain-clipping oracle against the reference's clip_domains (fixtures recorded by
tests/golden/make_clip_golden.py): the same boxes become empty, and the other boxes' bounds
agree to 1e-13 (the reference's einsum and the oracle sum in different orders)."""
import os

import numpy as np
import pytest

from oracle.clip import clip_domains

GOLD = os.path.join(os.path.dirname(__file__), "golden", "clip.npz")
CASES = sorted({k.rsplit("_", 1)[0] for k in np.load(GOLD).files})


def compare(cl, cu, rl, ru, xl, xu, tol=1e-13):
    emp_r = (rl > ru).any(1)
    assert np.array_equal(emp_r, (cl > cu).any(1))
    ne = ~emp_r
    scale = np.maximum(1.0, np.abs(xu - xl))[ne]
    assert np.max(np.abs(cl - rl)[ne] / scale) <= tol
    assert np.max(np.abs(cu - ru)[ne] / scale) <= tol


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference(case):
    d = np.load(GOLD)
    it = int(case.split("it")[1])
    cl, cu = clip_domains(d[case + "_xl"], d[case + "_xu"], d[case + "_thr"], d[case + "_lA"], d[case + "_lbias"],
                          num_iters=it)
    compare(cl, cu, d[case + "_cl"], d[case + "_cu"], d[case + "_xl"], d[case + "_xu"])


def test_clipping_keeps_every_point_a_plane_allows():
    """Sampled points of the original box where every plane is <= its threshold stay inside."""
    d = np.load(GOLD)
    case = "small_it1"
    xl, xu, thr, lA, lb = (d[case + s] for s in ("_xl", "_xu", "_thr", "_lA", "_lbias"))
    cl, cu = d[case + "_cl"], d[case + "_cu"]
    rng = np.random.default_rng(1)
    for b in range(xl.shape[0]):
        if not np.isfinite(lA[b]).all():
            continue
        x = xl[b] + (xu[b] - xl[b]) * rng.random((3000, xl.shape[1]))
        ok = ((x @ lA[b].T + lb[b]) <= thr[b]).all(1)
        if ok.any():
            assert np.all(x[ok] >= cl[b]) and np.all(x[ok] <= cu[b])
