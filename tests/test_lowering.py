"""Node-program lowering: programs emitted by the reference's gear front end
(tests/golden/make_program_golden.py) become IR graphs that compute the same function as the
source model and give the same CROWN bounds (oracle) as the directly traced model; the vnnlib
subset reader agrees with the reference's parse_vnnlib_subset on the recorded texts."""
import os
import sys

import numpy as np
import pytest
import torch

from gear_b200 import graph, problems
from gear_b200.lowering import LoweringError, graph_from_program, parse_vnnlib_subset
from oracle.crown import CrownOracle

HERE = os.path.dirname(__file__)
sys.path.insert(0, os.path.join(HERE, "golden"))
import models  # noqa: E402

DATA = torch.load(os.path.join(HERE, "golden", "programs.pt"), weights_only=False)


def source_model(name):
    if name in problems.WORKLOADS:
        return problems.make_instance(name, 0), problems.WORKLOADS[name]["n"]
    cls, n = models.MODELS[name]
    return cls().to(torch.float64), n


@pytest.mark.parametrize("name", sorted(DATA["programs"]))
def test_lowered_program_matches_traced_model(name):
    p = DATA["programs"][name]
    m, n = source_model(name)
    g_prog = graph_from_program(p["nodes_op"], p["nodes_in"], p["nodes_out"], n)
    g_model = graph.trace(m, torch.zeros(2, n, dtype=torch.float64))
    # the same function
    x = torch.rand(16, n, dtype=torch.float64, generator=torch.Generator().manual_seed(1)) * 2 - 1
    assert np.allclose(g_prog.forward_numpy(x.numpy()), m(x).detach().numpy(), rtol=1e-13, atol=1e-13)
    # the same IR structure
    assert [nd.kind for nd in g_prog.nodes] == [nd.kind for nd in g_model.nodes]
    # the same CROWN bounds
    lo = x[:4] - 0.1
    hi = x[:4] + 0.1
    a = CrownOracle(g_prog).compute_bounds(lo.numpy(), hi.numpy())
    b = CrownOracle(g_model).compute_bounds(lo.numpy(), hi.numpy())
    assert np.allclose(a[0], b[0], rtol=1e-12, atol=1e-12)
    assert np.allclose(a[2], b[2], rtol=1e-12, atol=1e-12)


def test_unsupported_node_is_refused():
    p = DATA["programs"]["sin_wide"]
    bad = [dict(nd) for nd in p["nodes_op"]]
    bad[0] = dict(bad[0], op="onnx::Tanh")
    with pytest.raises(LoweringError):
        graph_from_program(bad, p["nodes_in"], p["nodes_out"], 5)


@pytest.mark.parametrize("name", sorted(DATA["vnnlib"]))
def test_vnnlib_subset_matches_reference(name):
    r = DATA["vnnlib"][name]
    lo, hi, spec = parse_vnnlib_subset(r["text"], name)
    assert np.array_equal(lo, r["lo"].numpy()) and np.array_equal(hi, r["hi"].numpy())
    assert spec.num_outputs == r["num_outputs"]
    for k in ("indptr", "indices", "data", "rhs"):
        assert np.array_equal(getattr(spec, k), r[k].numpy())


@pytest.mark.parametrize("text", ["(declare-const X_0 Real)\n(assert (< X_0 1))",
                                  "(declare-const X_0 Real)\n(declare-const Y_0 Real)\n(assert (<= Y_0 1))",
                                  "(declare-const X_1 Real)\n(assert (<= X_1 1))\n(assert (>= X_1 0))"])
def test_vnnlib_outside_subset_raises(text):
    with pytest.raises(LoweringError):
        parse_vnnlib_subset(text)
