"""Timing recipe for the reference's own CPU path (test infrastructure, not product code).

Run in a container that has the reference source (it cannot travel to the GPU machine):

    python oracle/reference_cpu.py REFERENCE_ROOT [--out profiles/reference_cpu_baseline.md]

It measures, on this machine's cores, with torch using every core:

* ``BoundedModule.compute_bounds(method='CROWN')`` of the reference (float64, CPU, the bound
  options of GEAR's hot path: fp_enclosure.affine_backward, compare_crown_with_ibp_intermediate,
  undefined_relaxation_rows / interval, domain_aware_ops) on the quad_exp_n10 and dense_q_n200
  workloads, and the numpy restatement ``oracle/crown.py`` on the same boxes (the port that
  ``bench.py --impl reference`` times on the GPU machine's host), so the two can be related;
* branch and bound to relative gap 1e-4 on quad_exp_n10 instances, a plain loop built from the
  reference's own step functions (bound with compute_bounds, prune with
  UnsortedInputDomainList.get_remaining_index, branch with input_split_branching 'sb',
  bisect with input_split_parallel, child keys with _raise_child_keys, queue order by a stable
  descending sort of the objective key; incumbent = best feasible box midpoint).

The summary is written as markdown (the figures quoted beside the GPU numbers).
"""
import argparse
import importlib.abc
import importlib.machinery
import math
import os
import sys
import tempfile
import time
import types
from types import SimpleNamespace

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

BOUND_OPTS = {'fp_enclosure': {'affine_backward': True}, 'domain_aware_ops': True,
              'compare_crown_with_ibp_intermediate': True, 'undefined_relaxation_rows': True,
              'undefined_relaxation_interval': True}
STUB_ROOTS = ('onnx2pytorch', 'onnx', 'onnxruntime', 'onnxoptimizer', 'skl2onnx', 'vnnlib', 'highspy',
              'pyscipopt', 'gurobipy', 'cyipopt', 'graphviz')


class _Any:
    def __init__(self, *a, **k):
        pass

    def __call__(self, *a, **k):
        return _Any()

    def __getattr__(self, n):
        return _Any()

    def __iter__(self):
        return iter(())

    def __bool__(self):
        return False

    def __mro_entries__(self, bases):
        return (object,)


class _Mod(types.ModuleType):
    def __getattr__(self, n):
        if n.startswith('__'):
            raise AttributeError(n)
        return _Any()


class _Finder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    """Optional solver dependencies (ONNX, MIP/NLP solvers, graph drawing) the bounding code
    never calls."""

    def find_spec(self, name, path, target=None):
        if name.split('.')[0] in STUB_ROOTS:
            return importlib.machinery.ModuleSpec(name, self, is_package=True)
        return None

    def create_module(self, spec):
        m = _Mod(spec.name)
        m.__path__ = []
        return m

    def exec_module(self, module):
        pass


def import_reference(ref_root):
    sys.meta_path.insert(0, _Finder())
    appdirs = types.ModuleType("appdirs")
    appdirs.user_cache_dir = lambda *a, **k: tempfile.gettempdir()
    appdirs.user_data_dir = lambda *a, **k: tempfile.gettempdir()
    sys.modules["appdirs"] = appdirs
    sys.path.insert(0, os.path.join(ref_root, "solver", "complete_verifier"))
    sys.path.insert(0, os.path.join(ref_root, "solver"))
    torch.set_default_dtype(torch.float64)
    import arguments
    try:
        arguments.Config.parse_config(args=[])
    except BaseException:
        pass
    isa = arguments.Config['bab']['branching']['input_split']
    isa['sb_sum'] = True
    isa['sb_min_width_ratio'] = 0.001
    isa['sb_coeff_thresh'] = 1e-3
    isa['touch_zero_score'] = 0
    arguments.Config['solving']['solving_mode'] = True


def reference_bounder(model, n):
    """(BoundedModule, bound(lo, hi) -> (lb, lA, lbias)) of the reference for one model."""
    from auto_LiRPA import BoundedModule, BoundedTensor, PerturbationLpNorm
    bm = BoundedModule(model, torch.zeros(2, n), bound_opts=BOUND_OPTS, device='cpu')
    S = bm.final_node().output_shape[1]
    need = {bm.output_name[0]: {bm.input_name[0]}}

    def bound(lo, hi):
        C = torch.eye(S).unsqueeze(0).expand(lo.shape[0], S, S)
        x = BoundedTensor((lo + hi) / 2, PerturbationLpNorm(x_L=lo, x_U=hi))
        lb, _, A = bm.compute_bounds(x=(x,), C=C, method='CROWN', bound_upper=False, return_A=True,
                                     needed_A_dict=need)
        rec = A[bm.output_name[0]][bm.input_name[0]]
        return lb.detach(), rec['lA'].detach(), rec['lbias'].detach()
    return bm, S, bound


def time_compute_bounds(workload, batch, reps=3):
    """Seconds per reference compute_bounds call (best of reps after one warm-up) and per oracle
    port call on the same boxes."""
    from gear_b200 import graph, problems
    from oracle.crown import CrownOracle
    m = problems.make_instance(workload, 0)
    n = problems.WORKLOADS[workload]["n"]
    lo, hi = problems.make_boxes(workload, batch, 0, seed_offset=900)
    _, S, bound = reference_bounder(m, n)
    bound(lo, hi)
    ref = []
    for _ in range(reps):
        t = time.perf_counter()
        bound(lo, hi)
        ref.append(time.perf_counter() - t)
    g = graph.trace(m, lo[:2])
    o = CrownOracle(g)
    o.compute_bounds(lo.numpy()[:2], hi.numpy()[:2])
    port = []
    for _ in range(reps):
        t = time.perf_counter()
        o.compute_bounds(lo.numpy(), hi.numpy())
        port.append(time.perf_counter() - t)
    return {"workload": workload, "batch": batch, "reference_s": min(ref), "port_s": min(port),
            "reference_boxes_per_s": batch / min(ref), "port_boxes_per_s": batch / min(port)}


def time_constrained(batch, n, rows, reps=3):
    """Seconds per reference constrained concretisation (sort_out_constr_batches +
    constraints_solving, concretize_func.py:312-850, the PyTorch sweep, sign -1) of
    problems.cut_rows(batch, n, rows): best of reps after one warm-up; and of the numpy
    restatement oracle/concretize.py on the same inputs (one call: a per-box loop)."""
    from auto_LiRPA import concretize_func as cf
    from gear_b200 import problems
    from oracle import concretize as oc
    xl, xu, obj, A, b = problems.cut_rows(batch, n, rows)
    cf.MAX_CONSTRAINT_ROWS = None

    def ref():
        cons, masks = cf.sort_out_constr_batches(xl, xu, (A, b))
        return cf.constraints_solving(xl, xu, obj, cons, -1.0, sorted_out_batches=masks or {})
    ref()
    tr = []
    for _ in range(reps):
        t = time.perf_counter()
        ref()
        tr.append(time.perf_counter() - t)
    args = (xl.numpy(), xu.numpy(), obj.numpy(), A.numpy(), b.numpy())
    t = time.perf_counter()
    oc.constrained_lower(*args)
    tp = [time.perf_counter() - t]
    return {"batch": batch, "n": n, "rows": rows, "reference_s": min(tr), "port_s": min(tp)}


def reference_bab(inst, rel_gap=1e-4, batch=2048, time_limit=600.0):
    """Branch and bound to the relative gap on quad_exp_n10 instance `inst` with the reference's
    step functions; returns wall seconds, iterations, domains bounded and the final gap."""
    from gear_b200 import problems
    from input_split.branching_heuristics import input_split_branching
    from input_split.branching_domains import UnsortedInputDomainList
    from input_split.split import input_split_parallel
    from input_split.batch_branch_and_bound import _raise_child_keys
    m = problems.make_instance("quad_exp_n10", inst)
    n = 10
    _, S, bound = reference_bounder(m, n)
    rl, rh = problems.root_box("quad_exp_n10")
    root_w = (rh - rl).reshape(-1)
    rhs = torch.zeros(S - 1)
    lo, hi = rl.clone(), rh.clone()
    key = torch.full((1,), -math.inf)
    inc = math.inf
    disc = math.inf
    pool = SimpleNamespace(thresholds=lambda t: t, tolerance=0.0)
    hist = SimpleNamespace(root_width=root_w, angle_pairs=None, lifted_branch_score=None, node_pool=False)
    t0 = time.perf_counter()
    its, bounded, gap = 0, 0, math.inf
    while lo.shape[0] and time.perf_counter() - t0 < time_limit:
        order = torch.argsort(key, descending=True, stable=True)
        lo, hi, key = lo[order], hi[order], key[order]
        b = min(batch, lo.shape[0])
        plo, phi = lo[-b:], hi[-b:]
        lo, hi, key = lo[:-b], hi[:-b], key[:-b]
        with torch.no_grad():
            y = m((plo + phi) / 2)
        feas = (y[:, 1:] <= rhs).all(1)
        if feas.any():
            inc = min(inc, float(y[feas, 0].min()))
        lb, lA, lbias = bound(plo, phi)
        thr = torch.cat([torch.full((b, 1), inc), rhs.expand(b, S - 1)], 1)
        rem = UnsortedInputDomainList.get_remaining_index(b, lb, thr, plo, phi, check_dm_lbs=True,
                                                          check_input_boxes=False, rowpool=pool)
        keep = torch.zeros(b, dtype=torch.bool)
        keep[rem] = True
        dropped = (~keep) & (lb[:, 0] >= thr[:, 0])
        if dropped.any():
            disc = min(disc, float(thr[dropped, 0].min()))
        lb_f = torch.where(torch.isfinite(lb), lb, torch.zeros_like(lb))
        idx = input_split_branching(None, lb_f, plo, phi, lA, thr, 'sb', 1, history=hist)[:, 0]
        kept = torch.nonzero(keep).flatten()
        if kept.numel():
            cl, cu, _ = input_split_parallel(plo[kept], phi[kept], shape=plo.shape, split_depth=1,
                                             i_idx=idx[kept].unsqueeze(1))
            ck = _raise_child_keys(torch.cat([lb_f[kept], lb_f[kept]]), cl, cu,
                                   torch.cat([lA[kept], lA[kept]]), torch.cat([lbias[kept], lbias[kept]]))
            lo, hi, key = torch.cat([lo, cl]), torch.cat([hi, cu]), torch.cat([key, ck[:, 0]])
        its += 1
        bounded += b
        D = min(float(key.min()) if key.numel() else math.inf, disc)
        if math.isfinite(inc):
            gap = 0.0 if (not math.isfinite(D) and D > 0) else (inc - D) / max(1.0, abs(inc), abs(D))
        if gap <= rel_gap:
            break
    return {"instance": inst, "wall_s": time.perf_counter() - t0, "iterations": its, "bounded": bounded,
            "gap": gap, "closed": gap <= rel_gap}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("reference_root")
    ap.add_argument("--out", default=os.path.join(ROOT, "profiles", "reference_cpu_baseline.md"))
    ap.add_argument("--bab-instances", type=int, default=4)
    args = ap.parse_args()
    import_reference(args.reference_root)
    cores = os.cpu_count() or 1
    torch.set_num_threads(cores)
    rows = [time_compute_bounds("quad_exp_n10", 256), time_compute_bounds("dense_q_n200", 256)]
    cons = [time_constrained(1024, 200, 20), time_constrained(4096, 50, 16)]
    babs = [reference_bab(i) for i in range(args.bab_instances)]
    lines = ["# The reference's own CPU path, timed on this build container's cores", "",
             f"Command: `python oracle/reference_cpu.py REFERENCE_ROOT` ({cores} cores, torch threads = {cores}, "
             f"float64). The reference cannot travel to the GPU machine; `bench.py --impl reference` times the "
             f"numpy port there, and the ratio below relates the two.", "",
             "| workload | boxes | reference compute_bounds | boxes/s | numpy port | boxes/s | port / reference time |",
             "|---|---|---|---|---|---|---|"]
    for r in rows:
        lines.append(f"| {r['workload']} | {r['batch']} | {r['reference_s']:.3f} s | {r['reference_boxes_per_s']:.0f} | "
                     f"{r['port_s']:.3f} s | {r['port_boxes_per_s']:.0f} | {r['port_s'] / r['reference_s']:.2f} |")
    lines += ["", "Constrained concretisation (sort_out_constr_batches + constraints_solving, sign -1, no row cap) "
              "of `gear_b200.problems.cut_rows(batch, n, rows)`, one objective row per box:", "",
              "| batch | n | rows | reference | boxes/s | numpy port | boxes/s |", "|---|---|---|---|---|---|---|"]
    for r in cons:
        lines.append(f"| {r['batch']} | {r['n']} | {r['rows']} | {r['reference_s']:.3f} s | "
                     f"{r['batch'] / r['reference_s']:.0f} | {r['port_s']:.3f} s | {r['batch'] / r['port_s']:.0f} |")
    lines += ["", "Branch and bound to relative gap 1e-4 with the reference's step functions (batch 2048, "
              "quad_exp_n10 instances, CROWN bounds, incumbent from box midpoints):", "",
              "| instance | wall s | iterations | domains bounded | domains/s | final gap |", "|---|---|---|---|---|---|"]
    for b in babs:
        lines.append(f"| {b['instance']} | {b['wall_s']:.2f} | {b['iterations']} | {b['bounded']} | "
                     f"{b['bounded'] / b['wall_s']:.0f} | {b['gap']:.2e} |")
    ts = sorted(b["wall_s"] for b in babs)
    lines += ["", f"Time to gap p50 {ts[len(ts) // 2]:.2f} s, max {ts[-1]:.2f} s over {len(ts)} instances."]
    with open(args.out, "w") as f:
        f.write("\n".join(lines) + "\n")
    print("\n".join(lines))


if __name__ == "__main__":
    main()
