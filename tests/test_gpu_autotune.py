"""The autotuner (gear_b200.autotune): its candidates compute the same bounds (thread counts and
working-set placements agree with the default program to 1e-9 relative, exact-arithmetic
McCormick ties on both sides), the search covers the execution shapes and the tensor-core fold,
and the tuned engine's results agree with a plain CrownEngine's (1e-6: a tensor-core fold pick
differs from the float64 fold within its error term)."""
import numpy as np
import pytest
import torch

from gear_b200 import autotune, graph, problems
from gear_b200.autotune import Config, TunedEngine
from gear_b200.engine import CrownEngine, _Dag

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = a.cpu().numpy(), b.cpu().numpy()
    same = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
    return float(np.max(np.where(same, 0.0, np.abs(a - b) / np.maximum(1.0, np.abs(b)))))


@pytest.mark.parametrize("cfg", [Config("cta", 64, False), Config("cta", 256, True), Config("cta", 128, True),
                                 Config("simt", 0)])
def test_candidates_compute_the_same_bounds(cfg):
    m = problems.make_instance("dense_q_n200", 0)
    lo, hi = problems.make_boxes("dense_q_n200", 200, 2)
    g = graph.trace(m, lo[:2])
    xL, xU = lo.cuda(), hi.cuda()
    ref = CrownEngine(g, mode="cta", cta_threads=128, tie_rule="exact").lower(xL, xU)
    eng = TunedEngine(g, tie_rule="exact")
    e = eng._engine(cfg)
    got = e.lower(xL, xU)
    torch.cuda.synchronize()
    for a, b in zip(got, ref):
        assert _rel(a, b) < 1e-9


def test_tune_searches_and_engine_agrees():
    m = problems.make_instance("dense_a_n2048", 0)
    lo, hi = problems.make_boxes("dense_a_n2048", 256, 3)
    g = graph.trace(m, lo[:2])
    xL, xU = lo.cuda(), hi.cuda()
    cache = {}
    best, ms = autotune.tune(g, xL, xU, tie_rule="exact", cache=cache)
    assert best.name() in ms and ms[best.name()] == min(ms.values())
    assert any(k.startswith("cta256") for k in ms) and any(k.endswith("-tcfold") for k in ms)
    again, _ = autotune.tune(g, xL, xU, tie_rule="exact", cache=cache)
    assert again == best and len(cache) == 1
    eng = TunedEngine(g, tie_rule="exact")
    a = eng.lower(xL, xU)
    b = CrownEngine(g, mode="cta", cta_threads=256, tie_rule="exact").lower(xL, xU)
    torch.cuda.synchronize()
    assert eng.variant(256) is not None and eng.kernel_name(256).startswith("crown_")
    assert _rel(a[0], b[0]) < 1e-6
