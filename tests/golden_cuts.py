"""Loading of the recorded reference fixtures under cut rows (tests/golden/cuts_*.npz)."""
import glob
import os

import numpy as np
import torch

from gear_b200 import graph, problems

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def cut_cases():
    return sorted(os.path.basename(f)[5:-4] for f in glob.glob(os.path.join(HERE, "cuts_*.npz")))


def load_cuts(case):
    import models
    d = dict(np.load(os.path.join(HERE, f"cuts_{case}.npz")))
    name, inst = case.rsplit("_", 1)
    inst = int(inst)
    if name in problems.WORKLOADS:
        m = problems.make_instance(name, inst)
        n = problems.WORKLOADS[name]["n"]
    else:
        cls, n = models.MODELS[name]
        m = cls(seed=inst + 7)
    g = graph.trace(m, torch.zeros(2, n, dtype=torch.float64))
    inject = {int(k[6:]): (d[k], d["ib_hi_" + k[6:]]) for k in d if k.startswith("ib_lo_")}
    return m, g, d, inject
