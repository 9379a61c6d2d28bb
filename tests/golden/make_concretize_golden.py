"""Record golden constrained-concretisation outputs from the reference implementation (run in
a container that has the reference source; the committed .npz is what the tests read).

    python tests/golden/make_concretize_golden.py /path/to/reference

Calls the reference's sort_out_constr_batches + constraints_solving (auto_LiRPA/
concretize_func.py, PyTorch sweep, sign -1, no_return_inf False) in float64 on CPU on
seeded random boxes, objectives and constraint rows, with and without the row cap
(MAX_CONSTRAINT_ROWS), and stores inputs and lower bounds in tests/golden/concretize.npz.
"""
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def make_case(seed, B, H, X, K, t_lo=-1.3, t_hi=1.15, nonfinite=False):
    """Rows a_k^T x + b_k <= 0 whose offset puts the plane at t in units of the row's
    half-range over the box: t < -1 never binds, t > 1 excludes the box, between cuts it."""
    g = torch.Generator().manual_seed(seed)
    c = torch.rand(B, X, generator=g, dtype=torch.float64) * 4 - 2
    w = torch.rand(B, X, generator=g, dtype=torch.float64) * 0.9 + 0.05
    xl, xu = c - w, c + w
    obj = torch.randn(B, H, X, generator=g, dtype=torch.float64)
    A = torch.randn(B, K, X, generator=g, dtype=torch.float64)
    t = torch.rand(B, K, generator=g, dtype=torch.float64) * (t_hi - t_lo) + t_lo
    x0 = (xl + xu) / 2
    eps = (xu - xl) / 2
    b = -(A * x0[:, None]).sum(-1) + t * (A.abs() * eps[:, None]).sum(-1)
    if nonfinite:
        A[0, 0, 0] = float("inf")
        b[1, 1] = float("nan")
    return xl, xu, obj, A, b


def main(ref):
    import make_golden
    make_golden._stub_modules()
    sys.path.insert(0, os.path.join(ref, "solver"))
    from auto_LiRPA import concretize_func as cf
    cases = {
        "kat": (torch.tensor([[-1., -2.]], dtype=torch.float64), torch.tensor([[2., 1.]], dtype=torch.float64),
                torch.eye(2, dtype=torch.float64)[None], torch.tensor([[[1.0, 1.0]]], dtype=torch.float64),
                torch.tensor([[2.0]], dtype=torch.float64)),
        "small": make_case(11, 64, 3, 12, 6),
        "wide": make_case(12, 24, 2, 50, 16),
        "tall": make_case(13, 16, 1, 200, 20, t_lo=-1.1, t_hi=0.6),
        "covered": make_case(14, 8, 2, 10, 4, t_lo=-3.0, t_hi=-1.5),
        "nonfinite": make_case(15, 12, 2, 9, 5, nonfinite=True),
    }
    out = {}
    for name, (xl, xu, obj, A, b) in cases.items():
        for cap in (0, 4):
            if cap and name in ("kat", "covered"):
                continue
            cf.MAX_CONSTRAINT_ROWS = cap or None
            cons, masks = cf.sort_out_constr_batches(xl, xu, (A, b))
            lb = cf.constraints_solving(xl, xu, obj, cons, -1.0, sorted_out_batches=masks or {})
            key = f"{name}_cap{cap}"
            out[f"{key}_xl"], out[f"{key}_xu"] = xl.numpy(), xu.numpy()
            out[f"{key}_obj"], out[f"{key}_A"], out[f"{key}_b"] = obj.numpy(), A.numpy(), b.numpy()
            out[f"{key}_lb"] = lb.reshape(lb.shape[0], -1).numpy()
    cf.MAX_CONSTRAINT_ROWS = None
    np.savez_compressed(os.path.join(HERE, "concretize.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_ROOT")
    main(sys.argv[1])
