"""The IBP pass of the bounding glue (get_lower_bound_with_ibp_enhancement,
input_split/bounding.py:789): the oracle's ibp_output against the reference's
compute_bounds(method='ibp', C) (fixtures from tests/golden/make_ibp_golden.py), to 1e-13."""
import os
import sys

import numpy as np
import pytest
import torch

from gear_b200 import graph, problems
from oracle.crown import ibp_output

HERE = os.path.dirname(__file__)
sys.path.insert(0, os.path.join(HERE, "golden"))
import models  # noqa: E402

GOLD = os.path.join(HERE, "golden", "ibp_out.npz")
KEYS = sorted({k.rsplit("_", 1)[0] for k in np.load(GOLD).files})


def model_graph(key):
    name, inst, _ = key.rsplit("_", 2)
    if name in problems.WORKLOADS:
        m, n = problems.make_instance(name, int(inst)), problems.WORKLOADS[name]["n"]
    else:
        cls, n = models.MODELS[name]
        m = cls(seed=int(inst) + 7)
    return m, graph.trace(m, torch.zeros(2, n, dtype=torch.float64))


@pytest.mark.parametrize("key", KEYS)
def test_oracle_ibp_pass_matches_reference(key):
    d = np.load(GOLD)
    _, g = model_graph(key)
    lo, _ = ibp_output(g, d[key + "_xL"], d[key + "_xU"], d[key + "_C"])
    ref = d[key + "_lb"]
    assert np.max(np.abs(lo - ref) / np.maximum(1.0, np.abs(ref))) < 1e-13
