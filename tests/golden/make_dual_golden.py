"""Record golden rigorous dual bounds from the reference implementation (run where the reference
source is available; the committed .npz is what the tests read).

    python tests/golden/make_dual_golden.py /path/to/reference

Calls the reference's Rows / dual_lower_bound / certify_infeasible
(complete_verifier/nlp_solver/rigorous_dual.py) in float64 on CPU on seeded random batched LPs:
finite boxes, boxes with infinite sides, multipliers with heavy cancellation (which trigger the
double-double step), a pattern with values shared by the batch, and Farkas rays of infeasible
systems. Stores inputs and (lb, E, dd) / the infeasibility verdicts in tests/golden/dual.npz.
"""
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))


def lp(seed, B, m, n, density=0.4, inf_sides=False, cancel=False, shared=False):
    g = torch.Generator().manual_seed(seed)
    F = torch.float64
    mask = torch.rand(m, n, generator=g) < density
    mask[0, :] = True                                           # every column has an entry
    row, col = mask.nonzero(as_tuple=True)
    nnz = row.numel()
    val = torch.randn(1 if shared else B, nnz, generator=g, dtype=F)
    c = torch.randn(B, n, generator=g, dtype=F)
    c0 = torch.randn(B, generator=g, dtype=F)
    h = torch.randn(B, m, generator=g, dtype=F).abs() + 0.1
    l = -torch.rand(B, n, generator=g, dtype=F) * 2
    u = torch.rand(B, n, generator=g, dtype=F) * 2
    y = torch.rand(B, m, generator=g, dtype=F) * (torch.rand(B, m, generator=g) > 0.3)
    if inf_sides:
        l[::3, ::4] = -torch.inf
        u[1::3, 1::5] = torch.inf
    if cancel:
        # huge multipliers whose products nearly cancel the costs: the float error term is large
        # and the double-double step runs
        y = y * 1e11
        gty = torch.zeros(B, n, dtype=F).index_add_(1, col, val.expand(B, -1) * y[:, row])
        c = -gty + torch.randn(B, n, generator=g, dtype=F)
        h = h * 1e-10                                           # keep the dual value itself O(1)
    return row, col, val, m, n, c, c0, h, l, u, y


def main(ref_root):
    sys.path.insert(0, HERE)
    import make_bab_golden                      # stubs for optional solver dependencies the package imports
    sys.meta_path.insert(0, make_bab_golden._Finder())
    import make_golden
    make_golden._stub_modules()
    sys.path.insert(0, os.path.join(ref_root, "solver", "complete_verifier"))
    sys.path.insert(0, os.path.join(ref_root, "solver"))
    from nlp_solver.rigorous_dual import Rows, dual_lower_bound, certify_infeasible
    out = {}
    cases = {"plain": lp(31, 48, 12, 20), "infsides": lp(32, 48, 10, 16, inf_sides=True),
             "cancel": lp(33, 32, 14, 24, cancel=True), "shared": lp(34, 40, 8, 30, shared=True),
             "dense": lp(35, 16, 40, 60, density=0.9)}
    for name, (row, col, val, m, n, c, c0, h, l, u, y) in cases.items():
        rows = Rows(row, col, val, m, n)
        lb, E, dd = dual_lower_bound(rows, c, c0, h, l, u, y)
        for k, v in dict(row=row, col=col, val=val, c=c, c0=c0, h=h, l=l, u=u, y=y, lb=lb, E=E, dd=dd).items():
            out[f"{name}_{k}"] = v.numpy()
        out[f"{name}_mn"] = np.array([m, n])
    # Farkas rays: G z <= h with z in a box; rows 0 and 1 are z_0 <= -3 and -z_0 <= -3 (infeasible)
    g = torch.Generator().manual_seed(36)
    B, m, n = 24, 6, 5
    G = torch.randn(B, m, n, generator=g, dtype=torch.float64)
    G[:, 0] = 0
    G[:, 1] = 0
    G[:, 0, 0] = 1.0
    G[:, 1, 0] = -1.0
    h = torch.rand(B, m, generator=g, dtype=torch.float64) + 1
    h[:, 0] = -3.0
    h[:, 1] = -3.0
    h[1::2, 1] = 3.0                                            # odd batches: feasible
    l, u = -torch.ones(B, n, dtype=torch.float64) * 10, torch.ones(B, n, dtype=torch.float64) * 10
    y = torch.zeros(B, m, dtype=torch.float64)
    y[:, 0] = 1.0
    y[:, 1] = 1.0
    y[::4] = 0.0                                                # no ray: proves nothing
    rows = Rows.from_dense(G)
    verdict = certify_infeasible(rows, h, l, u, y)
    for k, v in dict(row=rows.row, col=rows.col, val=rows.val, h=h, l=l, u=u, y=y, inf=verdict).items():
        out[f"farkas_{k}"] = v.numpy()
    out["farkas_mn"] = np.array([m, n])
    np.savez_compressed(os.path.join(HERE, "dual.npz"), **out)
    print("saved", len(out), "arrays")


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_ROOT")
    main(sys.argv[1])
