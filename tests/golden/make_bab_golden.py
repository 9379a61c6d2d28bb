"""Record reference outputs of the BaB step functions (run where the reference source is
available; the committed .npz is what tests read).

    python tests/golden/make_bab_golden.py /path/to/reference

Calls, with the solver configured as the reference's GEAR preset does for them (solving
mode, sb branching with sb_sum, sb_min_width_ratio 0.001):
  get_remaining_index (prune mask), input_split_branching (split index), input_split_parallel
  (children), _raise_child_keys (child keys), and a stable descending argsort (queue order).
"""
import importlib.abc
import importlib.machinery
import os
import sys
import tempfile
import types
from types import SimpleNamespace

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))

STUB_ROOTS = ('onnx2pytorch', 'onnx', 'onnxruntime', 'onnxoptimizer', 'skl2onnx', 'vnnlib', 'highspy',
              'pyscipopt', 'gurobipy', 'cyipopt', 'graphviz')


class _Any:
    def __init__(self, *a, **k):
        pass

    def __call__(self, *a, **k):
        return _Any()

    def __getattr__(self, n):
        return _Any()

    def __iter__(self):
        return iter(())

    def __bool__(self):
        return False

    def __mro_entries__(self, bases):
        return (object,)


class _Mod(types.ModuleType):
    def __getattr__(self, n):
        if n.startswith('__'):
            raise AttributeError(n)
        return _Any()


class _Finder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    """Optional solver dependencies (ONNX, MIP/NLP solvers) the bounding code never calls."""

    def find_spec(self, name, path, target=None):
        if name.split('.')[0] in STUB_ROOTS:
            return importlib.machinery.ModuleSpec(name, self, is_package=True)
        return None

    def create_module(self, spec):
        m = _Mod(spec.name)
        m.__path__ = []
        return m

    def exec_module(self, module):
        pass


def main(ref_root):
    sys.meta_path.insert(0, _Finder())
    appdirs = types.ModuleType("appdirs")
    appdirs.user_cache_dir = lambda *a, **k: tempfile.gettempdir()
    appdirs.user_data_dir = lambda *a, **k: tempfile.gettempdir()
    sys.modules["appdirs"] = appdirs
    sys.path.insert(0, os.path.join(ref_root, "solver", "complete_verifier"))
    sys.path.insert(0, os.path.join(ref_root, "solver"))
    torch.set_default_dtype(torch.float64)
    import arguments
    try:
        arguments.Config.parse_config(args=[])
    except BaseException:
        pass
    isa = arguments.Config['bab']['branching']['input_split']
    isa['sb_sum'] = True
    isa['sb_min_width_ratio'] = 0.001
    isa['sb_coeff_thresh'] = 1e-3
    isa['touch_zero_score'] = 0
    arguments.Config['solving']['solving_mode'] = True
    from input_split.branching_heuristics import input_split_branching
    from input_split.branching_domains import UnsortedInputDomainList
    from input_split.split import input_split_parallel
    from input_split.batch_branch_and_bound import _raise_child_keys

    out = {}
    for case, (B, S, n, seed) in enumerate([(64, 3, 10, 1), (24, 51, 200, 2), (32, 1, 7, 3)]):
        g = torch.Generator().manual_seed(seed)
        lo = torch.rand(B, n, generator=g) * 2 - 1
        hi = lo + torch.rand(B, n, generator=g) * 0.5
        hi[:, 0] = lo[:, 0]                                   # a degenerate coordinate
        root_w = torch.full((n,), 2.5)
        lb = torch.randn(B, S, generator=g)
        thr = torch.randn(B, S, generator=g) * 0.5
        thr[::7, 0] = lb[::7, 0]                               # objective ties (>= prunes)
        thr[3::11] = torch.inf                                 # inactive rows
        lb[5::13, 0] = torch.inf                               # resolved domains
        lA = torch.randn(B, S, n, generator=g) * (torch.rand(B, S, n, generator=g) > 0.3)
        lA[::9] = lA[::9].round()                              # integer coefficients: score ties
        lbias = torch.randn(B, S, generator=g)
        # prune
        # thresholds arrive already relaxed by the instance's row tolerance (RowPool): identity pool
        pool = SimpleNamespace(thresholds=lambda t: t, tolerance=0.0)
        rem = UnsortedInputDomainList.get_remaining_index(B, lb, thr, lo, hi, check_dm_lbs=True,
                                                          check_input_boxes=False, rowpool=pool)
        keep = torch.zeros(B, dtype=torch.bool)
        keep[rem] = True
        # branch (finite lb for the SB score)
        lb_f = torch.where(torch.isfinite(lb), lb, torch.zeros_like(lb))
        hist = SimpleNamespace(root_width=root_w, angle_pairs=None, lifted_branch_score=None, node_pool=False)
        idx = input_split_branching(None, lb_f, lo, hi, lA, thr, 'sb', 1, history=hist)[:, 0]
        kept = torch.nonzero(keep).flatten()
        cl, cu, _ = input_split_parallel(lo[kept], hi[kept], shape=lo.shape, split_depth=1,
                                         i_idx=idx[kept].unsqueeze(1))
        keys = _raise_child_keys(torch.cat([lb_f[kept], lb_f[kept]]), cl, cu,
                                 torch.cat([lA[kept], lA[kept]]), torch.cat([lbias[kept], lbias[kept]]))
        qkey = lb_f[:, 0].clone()
        qkey[::6] = qkey[0]                                   # queue-key ties
        order = torch.argsort(qkey, descending=True, stable=True)
        pre = f"c{case}_"
        for k, v in dict(lo=lo, hi=hi, root_w=root_w, lb=lb, thr=thr, lA=lA, lbias=lbias, keep=keep, lb_f=lb_f,
                         idx=idx, kept=kept, child_lo=cl, child_hi=cu, child_key=keys, qkey=qkey,
                         order=order).items():
            out[pre + k] = v.numpy()
    np.savez_compressed(os.path.join(HERE, "bab_steps.npz"), **out)
    print("saved", len(out), "arrays")


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_ROOT")
    main(sys.argv[1])
