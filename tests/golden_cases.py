"""Loading of the recorded reference fixtures (tests/golden/crown_*.npz)."""
import glob
import os

import numpy as np
import torch

from gear_b200 import graph, problems

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def cases():
    return sorted(os.path.basename(f)[6:-4] for f in glob.glob(os.path.join(HERE, "crown_*.npz")))


def load(case):
    import models
    d = dict(np.load(os.path.join(HERE, f"crown_{case}.npz")))
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
