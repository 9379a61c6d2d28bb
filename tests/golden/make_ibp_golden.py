"""Record the reference's IBP pass (compute_bounds(method='ibp') with a specification C, the
first step of get_lower_bound_with_ibp_enhancement) on the benchmark workloads and fixture
models (run where the reference source is available; tests read tests/golden/ibp_out.npz).

    python tests/golden/make_ibp_golden.py /path/to/reference
"""
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def main(ref_root):
    sys.path.insert(0, HERE)
    sys.path.insert(0, REPO)
    import make_golden
    make_golden._stub_modules()
    sys.path.insert(0, os.path.join(ref_root, "solver"))
    torch.set_default_dtype(torch.float64)
    from auto_LiRPA import BoundedModule, BoundedTensor, PerturbationLpNorm
    from gear_b200 import problems
    import models
    out = {}
    cases = [("quad_exp_n10", 0, 24, False), ("dense_q_n200", 0, 6, False), ("quad_exp_n10", 1, 16, True)]
    cases += [(name, 0, 12, False) for name in ("mixed_ops", "sin_wide", "pow_ops")]
    for name, inst, batch, dense in cases:
        if name in problems.WORKLOADS:
            model = problems.make_instance(name, inst)
            n = problems.WORKLOADS[name]["n"]
            lo, hi = problems.make_boxes(name, batch, inst, seed_offset=321)
        else:
            cls, n = models.MODELS[name]
            model = cls(seed=inst + 7)
            L, U = model.box
            g = torch.Generator().manual_seed(400 + inst)
            c = L + (U - L) * torch.rand(batch, n, generator=g)
            w = torch.rand(batch, n, generator=g) * (U - L) * 0.6
            lo, hi = torch.clamp(c - w / 2, min=L), torch.clamp(c + w / 2, max=U)
        bm = BoundedModule(model, torch.zeros(2, n), bound_opts=make_golden.BOUND_OPTS, device='cpu')
        S = bm.final_node().output_shape[1]
        if dense:
            g = torch.Generator().manual_seed(7)
            C = torch.randn(lo.shape[0], 2, S, generator=g)
        else:
            C = torch.eye(S).unsqueeze(0).expand(lo.shape[0], S, S).contiguous()
        x = BoundedTensor((lo + hi) / 2, PerturbationLpNorm(x_L=lo, x_U=hi))
        lb = bm.compute_bounds(x=(x,), C=C, method='ibp', bound_upper=False)[0]
        key = f"{name}_{inst}_{'dense' if dense else 'eye'}"
        out[key + "_xL"], out[key + "_xU"], out[key + "_C"] = lo.numpy(), hi.numpy(), C.numpy()
        out[key + "_lb"] = lb.detach().numpy()
    np.savez_compressed(os.path.join(HERE, "ibp_out.npz"), **out)
    print("saved", sorted({k.rsplit('_', 1)[0] for k in out}))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_ROOT")
    main(sys.argv[1])
