"""Record golden CROWN bounds under cut rows from the reference implementation (run in a
container that has the reference source; the committed .npz fixtures are what the tests read).

    python tests/golden/make_cuts_golden.py /path/to/reference

Calls the reference's BoundedModule.compute_bounds(method='CROWN', bound_upper=False,
return_A=True) in float64 on CPU with the hot-path bound options, the perturbation carrying
linear rows A x + b <= 0 per box (PerturbationLpNorm(x_L, x_U, constraints=(A, b))): every
concretisation, the intermediate passes' included, is then the reference's constrained one
(sort_out_constr_batches + constraints_solving). The rows cut every box (their planes sit
inside the box's range) and one box of each case is covered by all of its rows; no row
excludes a box (the reference's batch result is not sound when one does). Stores x_L, x_U, C,
A, b, lb, lA, lbias and the intermediate bounds in tests/golden/cuts_<case>.npz, and lb_exact /
lA_exact / lbias_exact from a second run with the McCormick pick decided in exact arithmetic
(make_golden.exact_tie_rule).
"""
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)


def cut_rows(lo, hi, K, seed, t_lo=-1.0, t_hi=0.4, covered=1):
    """K rows per box whose plane sits at t half-ranges of the row over its box (t < 1: no row
    excludes the box); box `covered` gets t < -1 on every row (all rows redundant)."""
    g = torch.Generator().manual_seed(seed)
    B, n = lo.shape
    A = torch.randn(B, K, n, generator=g, dtype=torch.float64)
    t = torch.rand(B, K, generator=g, dtype=torch.float64) * (t_hi - t_lo) + t_lo
    t[covered] = -1.5
    x0, eps = (lo + hi) / 2, (hi - lo) / 2
    b = -(A * x0[:, None]).sum(-1) + t * (A.abs() * eps[:, None]).sum(-1)
    return A, b


def main(ref):
    import make_golden
    make_golden._stub_modules()
    sys.path.insert(0, os.path.join(ref, "solver"))
    torch.set_default_dtype(torch.float64)
    torch.set_num_threads(1)
    from auto_LiRPA import BoundedModule, BoundedTensor, PerturbationLpNorm
    from gear_b200 import graph, problems
    import models
    cases = [("quad_exp_n10", 0, 12, 4), ("quad_exp_n10", 1, 12, 6), ("mixed_ops", 0, 12, 4)]
    for name, inst, batch, K in cases:
        if name in problems.WORKLOADS:
            model = problems.make_instance(name, inst)
            n = problems.WORKLOADS[name]["n"]
            lo, hi = problems.make_boxes(name, batch, inst)
        else:
            cls, n = models.MODELS[name]
            model = cls(seed=inst + 7)
            L, U = model.box
            g = torch.Generator().manual_seed(200 + inst)
            c = L + (U - L) * torch.rand(batch, n, generator=g)
            w = torch.rand(batch, n, generator=g) * (U - L) * 0.6
            lo, hi = torch.clamp(c - w / 2, min=L), torch.clamp(c + w / 2, max=U)
        A, b = cut_rows(lo, hi, K, 300 + inst)
        bm = BoundedModule(model, torch.zeros(2, n), bound_opts=make_golden.BOUND_OPTS, device='cpu')
        S = bm.final_node().output_shape[1]
        C = torch.eye(S).unsqueeze(0).expand(lo.shape[0], S, S).contiguous()
        need = {bm.output_name[0]: {bm.input_name[0]}}

        def bound():
            x = BoundedTensor((lo + hi) / 2, PerturbationLpNorm(x_L=lo, x_U=hi, constraints=(A, b)))
            lb_, _, Ad = bm.compute_bounds(x=(x,), C=C, method='CROWN', bound_upper=False, return_A=True,
                                           needed_A_dict=need)
            return lb_.detach(), Ad[bm.output_name[0]][bm.input_name[0]]
        from auto_LiRPA.operators.bivariate import BoundMul
        float_rule = BoundMul._compute_coeff_aware_r
        BoundMul._compute_coeff_aware_r = make_golden.exact_tie_rule(BoundMul)
        lb_x, rec_x = bound()
        BoundMul._compute_coeff_aware_r = float_rule
        lb, rec = bound()
        gr = graph.trace(model, torch.zeros(2, n))
        inter = {}
        for m_id, r in make_golden.map_nodes(bm, gr).items():
            if m_id in (0, gr.output):
                continue
            if (isinstance(r.lower, torch.Tensor) and isinstance(r.upper, torch.Tensor)
                    and r.lower.ndim >= 2 and r.lower.shape[0] == lo.shape[0]):
                inter[f"ib_lo_{m_id}"] = r.lower.detach().reshape(lo.shape[0], -1).numpy()
                inter[f"ib_hi_{m_id}"] = r.upper.detach().reshape(lo.shape[0], -1).numpy()
        out = os.path.join(HERE, f"cuts_{name}_{inst}.npz")
        np.savez_compressed(out, x_L=lo.numpy(), x_U=hi.numpy(), C=C.numpy(), A=A.numpy(), b=b.numpy(),
                            lb=lb.detach().numpy(), lA=rec['lA'].detach().numpy(),
                            lbias=rec['lbias'].detach().numpy(), lb_exact=lb_x.numpy(),
                            lA_exact=rec_x['lA'].detach().numpy(), lbias_exact=rec_x['lbias'].detach().numpy(),
                            **inter)
        print(name, inst, "lb", lb.shape, "finite rows", int(torch.isfinite(lb).sum()))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_ROOT")
    main(sys.argv[1])
