"""Record golden domain-clipping outputs from the reference implementation (run where the
reference source is available; the committed .npz is what the tests read).

    python tests/golden/make_clip_golden.py /path/to/reference

Calls the reference's clip_domains (complete_verifier/input_split/clip.py) in float64 on
CPU, solving mode, with the thresholds already relaxed (identity RowPool), lower planes,
no base input rows, for 1 and 2 clip iterations, on seeded random boxes and planes that
cut, certify or miss the boxes, and stores inputs and clipped boxes in
tests/golden/clip.npz.
"""
import os
import sys
from types import SimpleNamespace

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def make_case(seed, B, S, n, t_lo=-1.1, t_hi=0.2):
    g = torch.Generator().manual_seed(seed)
    c = torch.rand(B, n, generator=g, dtype=torch.float64) * 2 - 1
    w = torch.rand(B, n, generator=g, dtype=torch.float64) * 0.5 + 0.01
    xl, xu = c - w, c + w
    lA = torch.randn(B, S, n, generator=g, dtype=torch.float64)
    lA = lA * (torch.rand(B, S, n, generator=g) > 0.2)          # zero coefficients too
    xhat, eps = (xl + xu) / 2, (xu - xl) / 2
    lo_plane = (lA * xhat[:, None]).sum(-1) - (lA.abs() * eps[:, None]).sum(-1)
    span = 2 * (lA.abs() * eps[:, None]).sum(-1)
    thr = torch.randn(B, S, generator=g, dtype=torch.float64)
    # the plane's minimum over the box sits at t in units of its range above the threshold
    t = torch.rand(B, S, generator=g, dtype=torch.float64) * (t_hi - t_lo) + t_lo
    lbias = thr - lo_plane + t * span
    thr[2::9, 1 % S] = torch.inf                                   # inactive rows
    if B > 5:
        lA[5, 0, 0] = float("nan")                                  # a box with non-finite data
    return xl, xu, thr, lA, lbias


def main(ref_root):
    import make_bab_golden
    sys.meta_path.insert(0, make_bab_golden._Finder())
    import make_golden
    make_golden._stub_modules()
    sys.path.insert(0, os.path.join(ref_root, "solver", "complete_verifier"))
    sys.path.insert(0, os.path.join(ref_root, "solver"))
    torch.set_default_dtype(torch.float64)
    import arguments
    try:
        arguments.Config.parse_config(args=[])
    except BaseException:
        pass
    arguments.Config['solving']['solving_mode'] = True
    from input_split.clip import clip_domains
    pool = SimpleNamespace(thresholds=lambda t: t, tolerance=0.0, derived_cut_registry=None)
    out = {}
    cases = {"small": (64, 3, 10, 21, -1.1, 0.2), "wide": (24, 6, 200, 22, -0.03, -0.004),
             "one": (40, 1, 5, 23, -1.1, 0.2)}
    for name, (B, S, n, seed, t_lo, t_hi) in cases.items():
        xl, xu, thr, lA, lbias = make_case(seed, B, S, n, t_lo, t_hi)
        for iters in (1, 2):
            cl, cu = clip_domains(xl, xu, thr, lA, lbias, num_iters=iters, rowpool=pool)
            key = f"{name}_it{iters}"
            for k, v in dict(xl=xl, xu=xu, thr=thr, lA=lA, lbias=lbias, cl=cl, cu=cu).items():
                out[f"{key}_{k}"] = v.numpy()
    np.savez_compressed(os.path.join(HERE, "clip.npz"), **out)
    print("saved", len(out), "arrays")


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_ROOT")
    main(sys.argv[1])
