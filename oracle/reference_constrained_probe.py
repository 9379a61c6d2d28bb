"""Recipe (test infrastructure, not product code): the reference's constrained CROWN bounds on a
batch in which one box is excluded by its cut rows.

    python oracle/reference_constrained_probe.py REFERENCE_ROOT

Bounds 12 quad_exp_n10 sub-boxes with BoundedModule.compute_bounds(method='CROWN') of the
reference, the perturbation carrying 4 cut rows per box (PerturbationLpNorm(constraints=(A, b)),
applied at every concretisation, intermediate passes included), three times: without cuts, with
cuts that every box satisfies in part, and with the same cuts except that one row of box 0
excludes that box. For boxes 2 and 3 it then samples 200 000 points of the box, keeps those
that satisfy the box's rows and prints the smallest objective values next to the reference's
lower bounds. Prints only; nothing is written.
"""
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "tests", "golden"))


def main(ref_root):
    import make_golden
    make_golden._stub_modules()
    sys.path.insert(0, os.path.join(ref_root, "solver"))
    torch.set_default_dtype(torch.float64)
    from auto_LiRPA import BoundedModule, BoundedTensor, PerturbationLpNorm
    from gear_b200 import problems
    model = problems.make_instance("quad_exp_n10", 0)
    n, batch, K = 10, 12, 4
    lo, hi = problems.make_boxes("quad_exp_n10", batch, 0)
    bm = BoundedModule(model, torch.zeros(2, n), bound_opts=make_golden.BOUND_OPTS, device='cpu')
    S = bm.final_node().output_shape[1]
    C = torch.eye(S).unsqueeze(0).expand(batch, S, S).contiguous()
    g = torch.Generator().manual_seed(3)
    A = torch.randn(batch, K, n, generator=g)
    x0, eps = (lo + hi) / 2, (hi - lo) / 2
    t = torch.rand(batch, K, generator=g) * 1.4 - 1.0          # planes that cut the boxes

    def rows(tt):
        return -(A * x0[:, None]).sum(-1) + tt * (A.abs() * eps[:, None]).sum(-1)

    def bound(cons):
        x = BoundedTensor(x0, PerturbationLpNorm(x_L=lo, x_U=hi, constraints=cons))
        lb, _ = bm.compute_bounds(x=(x,), C=C, method='CROWN', bound_upper=False)
        return lb.detach().numpy()

    b_cut = rows(t)
    t_ex = t.clone()
    t_ex[0, 0] = 1.5                                           # this row excludes box 0
    b_ex = rows(t_ex)
    lb_none, lb_cut, lb_ex = bound(None), bound((A, b_cut)), bound((A, b_ex))
    np.set_printoptions(precision=4, suppress=True)
    print("box 0 (excluded in the third batch):", lb_ex[0])
    gen = torch.Generator().manual_seed(9)
    for bi in (2, 3):
        P = lo[bi] + (hi[bi] - lo[bi]) * torch.rand(200000, n, generator=gen)
        feas = ((P @ A[bi].T + b_cut[bi]) <= 0).all(1)       # box bi's rows are the same in both batches
        with torch.no_grad():
            y = model(P[feas]).min(0).values.numpy()
        print(f"box {bi}: sampled min {y} ({int(feas.sum())} feasible points); lb without cuts {lb_none[bi]}, "
              f"with cuts {lb_cut[bi]}, with cuts and box 0 excluded {lb_ex[bi]}")


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_ROOT")
    main(sys.argv[1])
