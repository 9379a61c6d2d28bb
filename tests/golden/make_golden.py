"""Record golden CROWN outputs from the reference implementation (run in a container
that has the reference source; the committed .npz fixtures are what the tests read).

    python tests/golden/make_golden.py /path/to/reference

Calls the reference's BoundedModule.compute_bounds(method='CROWN', bound_upper=False,
return_A=True) in float64 on CPU with the hot-path bound options of the reference's
GEAR configuration (fp_enclosure.affine_backward, compare_crown_with_ibp_intermediate,
undefined_relaxation_rows/interval, domain_aware_ops), and stores x_L, x_U, C, lb, lA,
lbias plus the order of CROWN intermediate passes (node kind and width).

Two more records per case:

* ``lb_exact``, ``lA_exact``, ``lbias_exact``: the same call with the reference's McCormick
  plane pick (BoundMul._compute_coeff_aware_r, operators/bivariate.py:219-257) decided in exact
  arithmetic -- a relative difference of the two candidates' box minima (maxima) below 1e-12
  counts as a tie and picks plane 1. This is the outcome of the reference's comparison
  whenever its operands are exact; it differs from the float comparison only where the two
  planes tie and rounding noise in the intermediate bounds decides.
* ``lb_ulp_dev``: per row, the largest relative change of the reference's lb over three runs on
  the boxes widened by one ulp (x_L down, x_U up, both). Rows where it exceeds 1e-5 are decided
  by such ties: the reference itself does not determine them to that tolerance.
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


def exact_tie_rule(BoundMul):
    """A replacement for BoundMul._compute_coeff_aware_r that decides ties in exact arithmetic."""
    tol = 1e-12

    def rule(self, x_l, x_u, y_l, y_u):
        xl, xu = x_l + torch.zeros_like(y_l), x_u + torch.zeros_like(y_u)
        yl, yu = y_l + torch.zeros_like(x_l), y_u + torch.zeros_like(x_u)
        m1 = BoundMul._affine_min_box(yl, xl, -xl * yl, xl, xu, yl, yu)
        m2 = BoundMul._affine_min_box(yu, xu, -xu * yu, xl, xu, yl, yu)
        M1 = BoundMul._affine_max_box(yu, xl, -yu * xl, xl, xu, yl, yu)
        M2 = BoundMul._affine_max_box(yl, xu, -yl * xu, xl, xu, yl, yu)
        r_l = (m1 >= m2 - tol * (m1.abs() + m2.abs())).to(xl.dtype)
        r_u = (M1 <= M2 + tol * (M1.abs() + M2.abs())).to(xl.dtype)
        return r_l, r_u
    return rule


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
    from auto_LiRPA.operators.bivariate import BoundMul
    float_rule = BoundMul._compute_coeff_aware_r
    exact_rule = exact_tie_rule(BoundMul)
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
    cases.append(("undef_ops", 0, 16))
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
        need = {bm.output_name[0]: {bm.input_name[0]}}

        def bound(lo_, hi_):
            x = BoundedTensor((lo_ + hi_) / 2, PerturbationLpNorm(x_L=lo_, x_U=hi_))
            lb_, _, A_ = bm.compute_bounds(x=(x,), C=C, method='CROWN', bound_upper=False,
                                           return_A=True, needed_A_dict=need)
            return lb_.detach(), A_[bm.output_name[0]][bm.input_name[0]]

        BoundMul._compute_coeff_aware_r = exact_rule
        lb_x, rec_x = bound(lo, hi)
        BoundMul._compute_coeff_aware_r = float_rule
        dev = torch.zeros_like(lb_x)
        down, up = torch.nextafter(lo, torch.tensor(-torch.inf)), torch.nextafter(hi, torch.tensor(torch.inf))
        ulp = []
        for plo, phi in ((down, hi), (lo, up), (down, up)):
            ulp.append(bound(plo, phi)[0])
        passes.clear()
        lb, rec = bound(lo, hi)
        for lp in ulp:
            dev = torch.maximum(dev, (lp - lb).abs() / torch.clamp(lb.abs(), min=1.0))
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
                            lb_exact=lb_x.numpy(), lA_exact=rec_x['lA'].detach().numpy(),
                            lbias_exact=rec_x['lbias'].detach().numpy(), lb_ulp_dev=dev.numpy(),
                            passes=np.array([f"{k}:{w}" for k, w in passes]), **inter)
        print(name, inst, lb.shape, [f"{k}:{w}" for k, w in passes],
              f"rows the reference moves by > 1e-5 under one ulp: {int((dev > 1e-5).sum())}/{dev.numel()}")


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_ROOT")
    main(sys.argv[1])
