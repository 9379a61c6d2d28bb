"""The autotuner's host side without a GPU: candidate names and the structure key (equal for equal
graphs, different for different ones)."""
from gear_b200 import autotune, graph, problems


def _g(wl, inst=0):
    m = problems.make_instance(wl, inst)
    lo, _ = problems.make_boxes(wl, 2, 0)
    return graph.trace(m, lo)


def test_config_names():
    C = autotune.Config
    assert C("simt", 0).name() == "simt"
    assert C("cta", 128).name() == "cta128"
    assert C("cta", 256, True, True).name() == "cta256-global-tcfold"


def test_structure_key():
    a, b = _g("quad_exp_n10", 0), _g("quad_exp_n10", 0)
    assert autotune.structure_key(a) == autotune.structure_key(b)
    assert autotune.structure_key(a) != autotune.structure_key(_g("quad_exp_n10", 1))
