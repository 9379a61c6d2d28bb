"""The BaB step oracle (oracle/bab.py) against the reference's own functions (fixtures)."""
import os

import numpy as np
import pytest

from oracle import bab

D = np.load(os.path.join(os.path.dirname(__file__), "golden", "bab_steps.npz"))
CASES = sorted({k.split("_")[0] for k in D.files})


def g(c, k):
    return D[f"{c}_{k}"]


@pytest.mark.parametrize("c", CASES)
def test_prune_mask_matches_reference(c):
    keep, _ = bab.prune_mask(g(c, "lb"), g(c, "thr"))
    assert np.array_equal(keep, g(c, "keep"))


@pytest.mark.parametrize("c", CASES)
def test_sb_branch_matches_reference(c):
    idx = bab.sb_branch(g(c, "lA"), g(c, "lo"), g(c, "hi"), g(c, "lb_f"), g(c, "thr"), root_width=g(c, "root_w"))
    assert np.array_equal(idx, g(c, "idx"))


@pytest.mark.parametrize("c", CASES)
def test_split_matches_reference(c):
    cl, cu = bab.split(g(c, "lo"), g(c, "hi"), g(c, "kept"), g(c, "idx"))
    assert np.array_equal(cl, g(c, "child_lo")) and np.array_equal(cu, g(c, "child_hi"))


@pytest.mark.parametrize("c", CASES)
def test_child_keys_match_reference(c):
    # the key is a rounded-down plane minimum; its last bits depend on the order of the sum
    # over the inputs (numpy vs torch), so the match is to 1e-14 relative
    k = bab.child_keys(g(c, "lb_f"), g(c, "lA"), g(c, "lbias"), g(c, "child_lo"), g(c, "child_hi"), g(c, "kept"))
    ref = g(c, "child_key")
    assert np.all(np.abs(k - ref) <= 1e-14 * np.maximum(1.0, np.abs(ref)))


@pytest.mark.parametrize("c", CASES)
def test_queue_order_matches_stable_reference_sort(c):
    key = g(c, "qkey")
    assert np.array_equal(bab.queue_order(key, np.arange(len(key))), g(c, "order"))
