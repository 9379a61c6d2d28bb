"""Record golden CROWN outputs from the reference implementation (run in a container
that has the reference source; the committed .npz fixtures are what the tests read).

    python tests/golden/make_golden.py /path/to/reference

Calls the reference's BoundedModule.compute_bounds(method='CROWN', bound_upper=False,
return_A=True) in float64 on CPU with the hot-path bound options of the reference's
GEAR configuration (fp_enclosure.affine_backward, compare_crown_with_ibp_intermediate,
undefined_relaxation_rows/interval, domain_aware_ops), and stores x_L, x_U, C, lb, lA,
lbias plus the order of CROWN intermediate passes (node kind and width).
"""
import os
import sys
import tempfile
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

BOUND_OPTS = {'fp_enclosure': {'affine_backward': True}, 'domain_aware_ops': True,
              'compare_crown_with_ibp_intermediate': True, 'undefined_relaxation_rows': True,
              'undefined_relaxation_interval': True}


def _stub_modules():
    # the reference imports these two for logging/visualisation only
    appdirs = types.ModuleType("appdirs")
    appdirs.user_cache_dir = lambda *a, **k: tempfile.gettempdir()
    appdirs.user_data_dir = lambda *a, **k: tempfile.gettempdir()
    graphviz = types.ModuleType("graphviz")

    class Digraph:
        def __init__(self, *a, **k):
            pass

        def __getattr__(self, name):
            return lambda *a, **k: None
    graphviz.Digraph = Digraph
    sys.modules.setdefault("appdirs", appdirs)
    sys.modules.setdefault("graphviz", graphviz)


def map_nodes(bm, g):
    """Pair reference Bound nodes with IR node ids by walking both DAGs from the output
    (perturbed inputs in order); the IR keeps one node per perturbed reference node."""
    pairs = {}
    stack = [(bm.final_node(), g.output)]
    while stack:
        r, m = stack.pop()
        if m in pairs:
            continue
        pairs[m] = r
        rin = [i for i in r.inputs if i.perturbed]
        assert len(rin) == len(g[m].inputs), (r, g[m])
        for a, b in zip(rin, g[m].inputs):
            stack.append((a, b))
    return pairs


def main(ref_root):
    _stub_modules()
    sys.path.insert(0, os.path.join(ref_root, "solver"))
    torch.set_default_dtype(torch.float64)
    torch.set_num_threads(1)
    from auto_LiRPA import BoundedModule, BoundedTensor, PerturbationLpNorm
    import auto_LiRPA.bound_general as bg
    from gear_b200 import problems, graph
    import models

    passes = []
    orig = bg.BoundedModule.backward_general

    def logged(self, bound_node, C, *a, **k):
        passes.append((type(bound_node).__name__, int(np.prod(bound_node.output_shape[1:]))))
        return orig(self, bound_node, C, *a, **k)
    bg.BoundedModule.backward_general = logged

    cases = []
    for inst in range(4):
        cases.append(("quad_exp_n10", inst, 12))
    cases.append(("dense_q_n200", 0, 4))
    cases.append(("dense_a_n2048", 0, 2))
    cases.append(("mixed_ops", 0, 12))
    cases.append(("sin_wide", 0, 12))
    cases.append(("pow_ops", 0, 12))
    cases.append(("pow_ops", 1, 12))
    only = set(sys.argv[2:])
    if only:
        cases = [c for c in cases if c[0] in only]

    for name, inst, batch in cases:
        if name in problems.WORKLOADS:
            model = problems.make_instance(name, inst)
            n = problems.WORKLOADS[name]["n"]
            lo, hi = problems.make_boxes(name, batch - 1, inst)
            rl, rh = problems.root_box(name)
            lo, hi = torch.cat([rl, lo]), torch.cat([rh, hi])
        else:
            cls, n = models.MODELS[name]
            model = cls(seed=inst + 7)
            L, U = model.box
            g = torch.Generator().manual_seed(100 + inst)
            c = L + (U - L) * torch.rand(batch, n, generator=g)
            w = torch.rand(batch, n, generator=g) * (U - L) * 0.6
            w[1] = 0.0                      # a degenerate box
            lo, hi = torch.clamp(c - w / 2, min=L), torch.clamp(c + w / 2, max=U)
            lo[0], hi[0] = L, U
        bm = BoundedModule(model, torch.zeros(2, n), bound_opts=BOUND_OPTS, device='cpu')
        S = bm.final_node().output_shape[1]
        C = torch.eye(S).unsqueeze(0).expand(lo.shape[0], S, S).contiguous()
        x = BoundedTensor((lo + hi) / 2, PerturbationLpNorm(x_L=lo, x_U=hi))
        passes.clear()
        need = {bm.output_name[0]: {bm.input_name[0]}}
        lb, _, A = bm.compute_bounds(x=(x,), C=C, method='CROWN', bound_upper=False,
                                     return_A=True, needed_A_dict=need)
        rec = A[bm.output_name[0]][bm.input_name[0]]
        # intermediate bounds the reference kept, keyed by IR node id
        g = graph.trace(model, torch.zeros(2, n))
        inter = {}
        for m_id, r in map_nodes(bm, g).items():
            if m_id in (0, g.output):
                continue
            if (isinstance(r.lower, torch.Tensor) and isinstance(r.upper, torch.Tensor)
                    and r.lower.ndim >= 2 and r.lower.shape[0] == lo.shape[0]):
                inter[f"ib_lo_{m_id}"] = r.lower.detach().reshape(lo.shape[0], -1).numpy()
                inter[f"ib_hi_{m_id}"] = r.upper.detach().reshape(lo.shape[0], -1).numpy()
        out = os.path.join(HERE, f"crown_{name}_{inst}.npz")
        np.savez_compressed(out, x_L=lo.numpy(), x_U=hi.numpy(), C=C.numpy(), lb=lb.detach().numpy(),
                            lA=rec['lA'].detach().numpy(), lbias=rec['lbias'].detach().numpy(),
                            passes=np.array([f"{k}:{w}" for k, w in passes]), **inter)
        print(name, inst, lb.shape, [f"{k}:{w}" for k, w in passes])


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
