"""The serving loop's compile-pool job without a GPU: a request's model and root box go in as a
plain pickle and its traced graph and stripped program come back as one, equal to a compile in
this process; and a spawned pool runs the job."""
import multiprocessing as mp
import pickle
from concurrent.futures import ProcessPoolExecutor

import numpy as np
import torch

from gear_b200 import graph, problems
from gear_b200.serve import _compile_program, _compile_request


def _same(a, b):
    for k in ("header", "node_arr", "step_arr", "pass_arr", "op_arr", "int_pool", "dbl_pool"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def _request(n=12, seed=5003):
    m = problems.QuadExpN10(n=n, seed=seed)
    return m, torch.full((1, n), -2.0, dtype=torch.float64)


def test_compile_job_round_trip():
    m, lo = _request()
    blob = _compile_request(pickle.dumps((m, lo, 128, 65536)))
    assert isinstance(blob, bytes)
    g, prog = pickle.loads(blob)
    direct = _compile_program(graph.trace(m, lo.repeat(2, 1)), 128, 65536)
    _same(prog, direct)
    assert prog.mode == direct.mode and len(g.nodes) == len(direct.g.nodes)


def test_compile_job_in_spawned_pool():
    m, lo = _request(20, 5004)
    with ProcessPoolExecutor(max_workers=1, mp_context=mp.get_context("spawn")) as pool:
        blob = pool.submit(_compile_request, pickle.dumps((m, lo, 128, 0))).result(timeout=600)
    _, prog = pickle.loads(blob)
    _same(prog, _compile_program(graph.trace(m, lo.repeat(2, 1)), 128, 0))
    assert prog.mode == "cta"
