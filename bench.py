"""Benchmark: certified subdomain bounds per second of GEAR's CROWN hot path on B200.

A step is one CROWN ``compute_bounds`` over a batch of BaB subdomains of the
``dense_q_n200`` workload (n = 200, dense indefinite Q, 50 bilinear + linear constraint
rows, S = 51 specification rows; returns lb, lA (B, 51, 200) and lbias, float64).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl gear|reference]

N > 1 runs N independent replicas (one per rank, launched by torch.distributed.run): the
path does not exchange data between boxes, so there is no collective besides the timing
barrier; ``value`` is all ranks' subdomains over the slowest rank's device time.
``--impl reference`` times the CPU restatement of the reference algorithm (the oracle) on
the host cores on a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "certified subdomain bounds/sec"
UNIT = "subdomains/s"
WORKLOAD = "dense_q_n200"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- CPU leg (oracle)
def _cpu_worker(args):
    import numpy as np
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    sys.path.insert(0, ROOT)
    from oracle.crown import CrownOracle
    g, lo, hi = args
    o = CrownOracle(g)
    t = time.perf_counter()
    o.compute_bounds(lo, hi)
    return time.perf_counter() - t, lo.shape[0]


def cpu_baseline(per_core=16, cores=None, workload=WORKLOAD):
    """The float64 CPU oracle (restatement of the reference's compute_bounds) on a bounded
    sample: per_core boxes on each of `cores` spawned processes; value = boxes / slowest."""
    import multiprocessing as mp
    import torch
    from gear_b200 import graph, problems
    cores = cores or os.cpu_count() or 1
    m = problems.make_instance(workload, 0)
    lo, hi = problems.make_boxes(workload, per_core * cores, 0, seed_offset=900)
    g = graph.trace(m, lo[:2])
    jobs = [(g, lo[i * per_core:(i + 1) * per_core].numpy(), hi[i * per_core:(i + 1) * per_core].numpy())
            for i in range(cores)]
    env_before = os.environ.get("OMP_NUM_THREADS")
    os.environ["OMP_NUM_THREADS"] = "1"
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(_cpu_worker, jobs)
    if env_before is None:
        os.environ.pop("OMP_NUM_THREADS", None)
    slowest = max(r[0] for r in res)
    boxes = sum(r[1] for r in res)
    return {"value": boxes / slowest, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{boxes} {workload} sub-boxes ({per_core} per process on {cores} spawned processes, "
                      f"float64 numpy oracle, 1 thread each; slowest process {slowest:.2f} s)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    per_core = max(4, args.cpu_per_core)
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(per_core=per_core, workload=args.workload)
        if i >= args.warmup:
            vals.append(r["value"])
    v = statistics.median(vals)
    r["value"] = v
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * 1 / v,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "config": {"workload": args.workload, "batch": r["sample"]},
           "cpu_baseline": r, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


# ---------------------------------------------------------------- replicas (N > 1)
def rank_boxes(workload, batch, rank):
    """This rank's boxes: every rank bounds its own seeded sub-boxes of instance 0 (replicas,
    no exchange of boxes between ranks)."""
    from gear_b200 import problems
    return problems.make_boxes(workload, batch, 0, seed_offset=500 + 7919 * rank)


def max_over_ranks(value, world, device):
    """The slowest rank's value (timing is the max over ranks); identity for one rank."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------- branch and bound to the gap
def bab_to_gap(instances, dev, rel_gap=1e-4, batch=2048):
    """Branch and bound (select, CROWN, prune, SB branch, split on the device) to a relative gap
    on quad_exp_n10 instances 0..instances-1: wall time to the gap per instance (host loop
    included), p50 / p99, and subdomains bounded per second over all runs."""
    import torch
    from gear_b200 import graph, problems
    from gear_b200.bab import BaB
    times, bounded, iters, gaps = [], 0, [], []
    for inst in range(-1, instances):
        m = problems.make_instance("quad_exp_n10", max(inst, 0))
        lo, hi = problems.root_box("quad_exp_n10")
        g = graph.trace(m, lo.repeat(2, 1))
        m = m.to(dev)
        torch.cuda.synchronize(dev)
        t = time.perf_counter()
        bb = BaB(g, lo, hi, batch=batch, model=m, device=str(dev))
        P, D, gap = bb.run(rel_gap=rel_gap, max_iterations=5000, time_limit=60)
        torch.cuda.synchronize(dev)
        dt = time.perf_counter() - t
        if inst < 0:
            continue                                        # warm-up run (module load)
        times.append(dt)
        bounded += bb.stats.bounded
        iters.append(bb.stats.iterations)
        gaps.append(gap)
    q = sorted(times)
    p99 = q[min(len(q) - 1, int(round(0.99 * (len(q) - 1))))]
    return {"workload": "quad_exp_n10 (config-1 family)", "instances": instances, "rel_gap": rel_gap,
            "batch": batch, "time_to_gap_s": {"p50": statistics.median(times), "p99": p99, "max": max(times)},
            "closed": sum(1 for gp in gaps if gp <= rel_gap), "iterations_median": statistics.median(iters),
            "subdomains_per_s": bounded / sum(times), "timing": "wall clock, host loop included"}


# ---------------------------------------------------------------- GPU leg
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--impl", default="gear", choices=["gear", "reference"])
    ap.add_argument("--cpu-per-core", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--bab-instances", type=int, default=8,
                    help="also run branch and bound to relative gap 1e-4 on this many quad_exp_n10 instances "
                         "(time to gap, p50 / p99); 0 skips it")
    ap.add_argument("--workload", default=WORKLOAD, help="benchmark workload (profiling of other shapes)")
    ap.add_argument("--cta-threads", type=int, default=128, help="threads per CTA of --mode cta")
    ap.add_argument("--mode", default="auto", choices=["auto", "cta", "simt"],
                    help="CROWN kernel: one box per CTA, one box per thread, or the faster one timed on the "
                         "first (warm-up) call")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    from gear_b200 import problems, BoundedModule
    from gear_b200 import _lib
    B = args.batch
    model = problems.make_instance(args.workload, 0)
    lo, hi = rank_boxes(args.workload, B, rank)
    bm = BoundedModule(model, lo[:2], device=str(dev), bound_opts={"gear_mode": args.mode,
                                                                  "gear_cta_threads": args.cta_threads})
    S = bm.final_node_width()
    n = lo.shape[1]
    eng = bm._engine(S, False)
    xL, xU = lo.to(dev), hi.to(dev)
    lb = torch.empty(B, S, dtype=torch.float64, device=dev)
    lA = torch.empty(B, S, n, dtype=torch.float64, device=dev)
    lbias = torch.empty(B, S, dtype=torch.float64, device=dev)
    out = (lb, lA, lbias)

    def step():
        eng.lower(xL, xU, None, out=out)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    variant = eng.variant(B)

    def barrier():
        if world > 1:
            dist.barrier()

    # device-resident timed region
    launches = 0
    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            step()
            launches += _lib.lib().gear_last_launch_count()
        e1.record()
        torch.cuda.synchronize()
        barrier()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world, dev)
    value = B * args.steps * world / (ms_max / 1000.0)

    # end to end through the public API: pinned host boxes in, lb back to the host
    from gear_b200 import BoundedTensor, PerturbationLpNorm
    hL, hU = lo.pin_memory(), hi.pin_memory()
    hlb = torch.empty(B, S, dtype=torch.float64).pin_memory()
    e_steps = max(1, min(args.steps, 5))

    def e2e_step():
        dL = hL.to(dev, non_blocking=True)
        dU = hU.to(dev, non_blocking=True)
        x = BoundedTensor(dL, PerturbationLpNorm(x_L=dL, x_U=dU))
        r_lb, _, A = bm.compute_bounds(x=(x,), method="CROWN", bound_upper=False, return_A=True)
        hlb.copy_(r_lb, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(e_steps):
        e2e_step()
    f1.record()
    torch.cuda.synchronize()
    e2e_value = B * e_steps * world / (max_over_ranks(f0.elapsed_time(f1), world, dev) / 1000.0)

    if rank == 0:
        peak, peak_kind = _peaks()
        ms_launch = ms / args.steps
        # algorithmic bytes of the executed schedule (A entries read + written by the passes,
        # float64) plus boxes in and lb, lbias, lA out
        prog = eng.prog
        alg_bytes = B * prog.alg_bytes_per_box()
        achieved = alg_bytes / (ms_launch / 1000.0) / 1e9
        traffic = None
        tfile = os.path.join(ROOT, "profiles", "dram_traffic.json")
        if os.path.exists(tfile):
            try:
                with open(tfile) as f:
                    tj = json.load(f)
                kname = "crown_simt_kernel" if variant == "simt" else f"crown_megakernel<{variant[3:]}>"
                traffic = tj.get(args.workload, {}).get(kname, {}).get("bytes_per_box")
                traffic = traffic * B if traffic is not None else None
            except Exception:
                traffic = None
        res = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": args.workload, "batch": B, "n": n, "spec_rows": S, "kernel_mode": args.mode, "kernel_variant": variant,
                          "variant_ms": eng.timings.get(eng._bucket(B)),
                          "parallelism": f"replicas{world}",
                          "l2": "inputs (x_L, x_U) and outputs (lA) larger than the 126 MB L2"},
               "gpu_launches": launches,
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": traffic,
                            "kernel": "crown_simt_kernel" if variant == "simt" else f"crown_megakernel<{variant[3:]}>",
                            "peak_source": peak_kind,
                            "alg_bytes_per_box": prog.alg_bytes_per_box(), "work_per_box": prog.work,
                            "fp64_gemm_gflops": prog.work["gemm_flops"] * B / (ms_launch / 1000.0) / 1e9},
               "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * B * n * 8,
                       "d2h_bytes_per_step": B * S * 8},
               "clocks": clk.summary()}
        if args.bab_instances > 0:
            res["bab"] = bab_to_gap(args.bab_instances, dev)
        if world == 1 and not args.no_cpu_baseline:
            try:
                res["cpu_baseline"] = cpu_baseline(per_core=args.cpu_per_core, workload=args.workload)
            except Exception as ex:  # the baseline is reported, not required
                res["cpu_baseline"] = {"value": None, "error": str(ex)[:200]}
        print(json.dumps(res))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
