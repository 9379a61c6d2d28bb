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
                      f"float64 numpy oracle, 1 thread each; slowest process {slowest:.2f} s)",
            "sample_boxes": boxes, "sample_s": slowest}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    per_core = max(4, args.cpu_per_core)
    vals, secs = [], []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(per_core=per_core, workload=args.workload)
        if i >= args.warmup:
            vals.append(r["value"])
            secs.append(r["sample_s"])
    v = statistics.median(vals)
    r["value"] = v
    from gear_b200 import graph, problems
    m = problems.make_instance(args.workload, 0)
    lo, _ = problems.make_boxes(args.workload, 2, 0)
    g = graph.trace(m, lo)
    # the GPU arm's workload and shapes; each step bounds a sample of its boxes on the host cores
    config = {"workload": args.workload, "batch": args.batch, "n": int(lo.shape[1]), "spec_rows": int(g[g.output].width),
              "parallelism": f"replicas{args.gpus}", "sample_per_step": r["sample"]}
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.median(secs),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "config": config,
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
def bab_to_gap(instances, dev, rel_gap=1e-4, batch=2048, graph_capture=True):
    """Branch and bound (select, CROWN, prune, SB branch, split on the device) to a relative gap
    on quad_exp_n10 instances 0..instances-1: wall time to the gap per instance (host included),
    p50 / p99, and subdomains bounded per second over all runs. graph_capture=True: the queue on the
    device and 8 iterations per CUDA-graph replay (GraphBaB); False: the host-driven loop (BaB)."""
    import torch
    from gear_b200 import graph, problems
    from gear_b200.bab import BaB, GraphBaB
    times, bounded, iters, gaps = [], 0, [], []
    for inst in range(-1, instances):
        m = problems.make_instance("quad_exp_n10", max(inst, 0))
        lo, hi = problems.root_box("quad_exp_n10")
        g = graph.trace(m, lo.repeat(2, 1))
        m = m.to(dev)
        torch.cuda.synchronize(dev)
        t = time.perf_counter()
        if graph_capture:
            bb = GraphBaB(g, lo, hi, batch=batch, model=m, device=str(dev))
        else:
            bb = BaB(g, lo, hi, batch=batch, model=m, device=str(dev))
        P, D, gap = bb.run(rel_gap=rel_gap, max_iterations=5000, time_limit=60)
        torch.cuda.synchronize(dev)
        dt = time.perf_counter() - t
        if inst < 0:
            continue                                        # warm-up run (module load)
        times.append(dt)
        bounded += bb.status["bounded"] if graph_capture else bb.stats.bounded
        iters.append(bb.status["iterations"] if graph_capture else bb.stats.iterations)
        gaps.append(gap)
    q = sorted(times)
    p99 = q[min(len(q) - 1, int(round(0.99 * (len(q) - 1))))]
    return {"workload": "quad_exp_n10 (config-1 family)", "instances": instances, "rel_gap": rel_gap,
            "batch": batch, "time_to_gap_s": {"p50": statistics.median(times), "p99": p99, "max": max(times)},
            "closed": sum(1 for gp in gaps if gp <= rel_gap), "iterations_median": statistics.median(iters),
            "subdomains_per_s": bounded / sum(times),
            "form": "device queue, 8 iterations per CUDA-graph replay (GraphBaB)" if graph_capture else
                    "host-driven loop (BaB)",
            "timing": "wall clock per instance from construction (engine pick, capture) to the gap"}


def mixed_setup(instances=512, workers=None):
    """Instances 0..instances-1 of the mixed family, traced, compiled in a process pool and
    uploaded into one MultiEngine: (instances, graphs, engine, compile seconds)."""
    import torch
    from gear_b200 import graph, problems
    from gear_b200.engine import MultiEngine
    from gear_b200.program import compile_many
    t0 = time.perf_counter()
    insts = [problems.mixed_instance(k) for k in range(instances)]
    graphs = [graph.trace(m, torch.zeros(2, m.n, dtype=torch.float64)) for m in insts]
    from gear_b200.engine import PACK_SMEM_LIMIT, SIMT_PACK_ITEMS
    me = MultiEngine(graphs, programs=compile_many(graphs, kw=dict(mode="cta", cta_threads=256,
                                                                   smem_limit=PACK_SMEM_LIMIT),
                                                   simt_items_max=SIMT_PACK_ITEMS, workers=workers))
    return insts, graphs, me, time.perf_counter() - t0, {}


def mixed_batch(dev, setup, boxes=256, steps=2, warmup=1, baselines=True):
    """The uneven batch: instances 0..instances-1 of the mixed family (n log-uniform in [5, 500],
    depth 3-12, m = n // 4), `boxes` sub-boxes each. Certified subdomain bounds per second
    (device time, CUDA events) of (a) every instance in one persistent launch per kernel variant
    (MultiEngine), (b) the same programs launched alone, one launch per instance back to back on
    one stream, and (c) the plain form, one instance at a time with one launch per schedule step
    and per op. Results of (a) are compared bit for bit with (b) and (c)."""
    import torch
    from gear_b200 import _lib, problems
    from gear_b200.engine import _Dag
    from gear_b200.program import compile_many
    insts, graphs, me, compile_s = setup[:4]
    instances = len(insts)
    bx = [tuple(t.to(dev) for t in problems.mixed_boxes(m, boxes, k)) for k, m in enumerate(insts)]
    total = instances * boxes
    outs = me.outputs([boxes] * instances, dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    packed_ms = timed(lambda: me.lower(bx, out=outs), steps, warmup)
    me.record_groups(True)
    me.lower(bx, out=outs)
    group_ms = me.group_ms()
    me.record_groups(False)
    res = {"workload": "mixed family (n log-uniform [5, 500], depth 3-12, m = n // 4)", "instances": instances,
           "boxes_per_instance": boxes, "groups": me.group_names(), "group_ms": group_ms,
           "launches_per_call": me.launches(), "packed_ms": packed_ms,
           "packed_subdomains_per_s": total / (packed_ms / 1000.0), "compile_s": compile_s}
    if not baselines:
        return res
    # one launch per instance through gear_crown_lower, same programs
    L = _lib.lib()
    ws_bytes = max(int(L.gear_crown_workspace_bytes(d.handle, boxes)) for d in me.dags)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    alone = me.outputs([boxes] * instances, dev)
    stream = torch.cuda.current_stream(dev).cuda_stream

    def alone_step():
        for i, d in enumerate(me.dags):
            lb, lA, lbias = alone[i]
            _lib.check(L.gear_crown_lower(d.handle, bx[i][0].data_ptr(), bx[i][1].data_ptr(), boxes, None,
                                          lb.data_ptr(), lA.data_ptr(), lbias.data_ptr(), ws.data_ptr(), ws_bytes,
                                          stream), "gear_crown_lower")
    alone_ms = timed(alone_step, steps, warmup)
    same = all(torch.equal(a[0], b[0]) and torch.equal(a[1], b[1]) for a, b in zip(outs, alone))
    del ws
    res.update({"alone_ms": alone_ms, "alone_subdomains_per_s": total / (alone_ms / 1000.0),
                "packed_vs_alone": alone_ms / packed_ms, "bitwise_equal_alone": same})
    if baselines:
        t1 = time.perf_counter()
        pprogs = plain_programs(setup)
        pdags = [_Dag.from_program(p) for p in pprogs]
        compile_s += time.perf_counter() - t1
        pws_bytes = max(int(L.gear_crown_plain_workspace_bytes(d.handle, boxes)) for d in pdags)
        pws = torch.empty(pws_bytes, dtype=torch.uint8, device=dev)
        pl = me.outputs([boxes] * instances, dev)
        launches = [0]

        def plain_step():
            launches[0] = 0
            for i, d in enumerate(pdags):
                lb, lA, lbias = pl[i]
                _lib.check(L.gear_crown_lower_plain(d.handle, bx[i][0].data_ptr(), bx[i][1].data_ptr(), boxes, None,
                                                    lb.data_ptr(), lA.data_ptr(), lbias.data_ptr(), pws.data_ptr(),
                                                    pws_bytes, stream), "gear_crown_lower_plain")
                launches[0] += int(L.gear_last_launch_count())
        plain_ms = timed(plain_step, 1, 1)
        res.update({"plain_ms": plain_ms, "plain_subdomains_per_s": total / (plain_ms / 1000.0),
                    "plain_launches_per_call": launches[0], "packed_vs_plain": plain_ms / packed_ms,
                    "plain_difference": lb_difference(outs, pl)})
        del pws
    res.update({"compile_s": compile_s, "timing": f"CUDA events; packed and alone {steps} calls after {warmup} "
                "warm-up, plain 1 call after 1 warm-up call"})
    return res


def plain_programs(setup):
    """The plain form's programs of the uneven batch (pass working set in global memory,
    128 threads per CTA), compiled once per setup."""
    from gear_b200.program import compile_many
    cache = setup[4]
    if "plain" not in cache:
        cache["plain"] = compile_many(setup[1], kw=dict(mode="cta", cta_threads=128, smem_limit=0))
    return cache["plain"]


def lb_difference(a_outs, b_outs):
    """How the lower bounds of two runs of the same boxes differ: the largest relative difference
    (to max(1, |lb|)) and the share of rows that differ by more than 1e-9. Kernel variants sum in
    different orders, and where two McCormick planes tie (equal box minima) the reference's float
    comparison, used by default, follows those last bits: such rows can differ by much more than
    the rounding (both bounds are sound)."""
    import torch
    num, rows, worst = 0, 0, 0.0
    for (la, _, _), (lb_, _, _) in zip(a_outs, b_outs):
        if la.numel() == 0:
            continue
        same_inf = torch.isinf(la) & torch.isinf(lb_) & (torch.sign(la) == torch.sign(lb_))
        err = torch.where(same_inf, torch.zeros_like(la), (la - lb_).abs() / torch.clamp(lb_.abs(), min=1.0))
        err = torch.nan_to_num(err, nan=float("inf"))
        worst = max(worst, float(err.max()))
        num += int((err > 1e-9).sum())
        rows += err.numel()
    return {"max_rel": worst, "rows_over_1e-9": num, "rows": rows,
            "note": "default McCormick tie rule (the reference's float comparison): tie-decided rows follow the "
                    "summation order of the kernel variant; both arms' bounds are sound"}


def mixed_bab(dev, setup, batch=256, rel_gap=1e-4, time_limit=60.0, plain=False, graph_capture=True):
    """Branch and bound on the uneven batch to relative gap 1e-4, every instance at once
    (MultiBaB): certified subdomains per second (subdomains bounded, each with a sound lower bound,
    per second of wall time, host loop included), wall time to the gap per instance over the
    instances that reach it within the time limit. plain=False bounds every iteration's batches in
    one packed CROWN launch per kernel variant (MultiEngine); plain=True is the plain GPU form:
    each instance's batch bounded alone, one launch per schedule step and per op
    (PlainMultiEngine), the same loop otherwise. graph_capture (packed only): every instance's
    queue on the device and whole rounds replayed from a CUDA graph (MultiGraphBaB)."""
    import torch
    from gear_b200.bab import MultiBaB, MultiGraphBaB
    insts, graphs, me = setup[:3]
    if plain:
        from gear_b200.engine import PlainMultiEngine
        me = PlainMultiEngine(graphs, programs=plain_programs(setup))
    instances = len(insts)
    roots = [(torch.full((1, m.n), -2.0, dtype=torch.float64), torch.full((1, m.n), 2.0, dtype=torch.float64))
             for m in insts]
    models = [m.to(dev) for m in insts]
    graphed = graph_capture and not plain
    if graphed:
        mb = MultiGraphBaB(graphs, roots, models, batch=batch, engine=me, device=str(dev))
    else:
        mb = MultiBaB(graphs, roots, models, batch=batch, engine=me, device=str(dev))
    torch.cuda.synchronize(dev)
    t = time.perf_counter()
    res = mb.run(rel_gap=rel_gap, time_limit=time_limit)
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - t
    if graphed:
        # domains bounded per instance up to its retirement (the captured round may run on)
        mb.bounded = sum(r["bounded"] for r in res)
        mb.iterations = mb.rounds
        statuses = {}
        for r in res:
            statuses[r["status"]] = statuses.get(r["status"], 0) + 1
    ttg = sorted(r["time_to_gap"] for r in res if r["time_to_gap"] is not None)
    q = (lambda p: ttg[min(len(ttg) - 1, int(round(p * (len(ttg) - 1))))]) if ttg else (lambda p: None)
    closed_n = [insts[i].n for i, r in enumerate(res) if r["time_to_gap"] is not None]
    return {"workload": "mixed family (n log-uniform [5, 500], depth 3-12, m = n // 4)", "instances": instances,
            "form": "plain GPU form (one instance, one launch per step and per op, host-driven loop)" if plain else
                    ("packed launch per kernel variant, device queues, rounds replayed from a CUDA graph "
                     "(MultiGraphBaB)" if graphed else "packed launch per kernel variant, host-driven loop (MultiBaB)"),
            "statuses": statuses if graphed else None,
            "graph_captures": getattr(mb, "captures", None), "graph_replays": getattr(mb, "replays", None),
            "batch_per_instance": batch, "rel_gap": rel_gap, "time_limit_s": time_limit, "wall_s": wall,
            "iterations": mb.iterations, "closed": len(ttg), "closed_max_n": max(closed_n) if closed_n else None,
            "time_to_gap_s": {"p50": q(0.5), "p99": q(0.99), "max": ttg[-1] if ttg else None},
            "subdomains_per_s": mb.bounded / wall, "bounded": mb.bounded,
            "timing": "wall clock from the first iteration, host loop included"}


def serve(dev, seconds=10.0, rate=50.0, budget=30.0, batch=2048, rel_gap=1e-4, seed=0, round_bytes=16 << 20,
          max_live=128, admission="small_first", incumbent_every=4, round_cap=32, device_queues=True,
          compile_workers=8, preempt=False):
    """The serving loop under Poisson arrivals (rate per second for `seconds`): instances of the
    quad-exp family with n log-uniform in [5, 2000] (two bilinear constraints), each to the
    relative gap or its time budget (from arrival). Continuous batching: requests are admitted as
    memory allows and join the running rounds (Server: host-driven rounds; device_queues:
    DeviceServer, every request's queue on the device and its round in CUDA graphs). Time to gap
    = finish - arrival."""
    import math as _m
    import torch
    from gear_b200 import problems
    from gear_b200.serve import DeviceServer, Server
    g = torch.Generator().manual_seed(5000 + seed)
    t, arrivals = 0.0, []
    while True:
        t += float(-_m.log(1.0 - float(torch.rand(1, generator=g))) / rate)
        if t > seconds:
            break
        arrivals.append(t)
    ns = [int(round(_m.exp(_m.log(5) + (_m.log(2000) - _m.log(5)) * float(torch.rand(1, generator=g)))))
          for _ in arrivals]
    srv = (DeviceServer if device_queues else Server)(device=str(dev), compile_workers=compile_workers, batch=batch, rel_gap=rel_gap, time_budget=budget, round_bytes=round_bytes,
                 max_live=max_live, admission=admission, incumbent_every=incumbent_every, round_cap=round_cap,
                 preempt=preempt)
    t0 = time.perf_counter()
    clock = lambda: time.perf_counter() - t0
    srv.clock = clock
    k = 0
    while k < len(arrivals) or not srv.idle():
        now = clock()
        while k < len(arrivals) and arrivals[k] <= now:
            m = problems.QuadExpN10(n=ns[k], seed=5000 + k)
            srv.submit(k, m, torch.full((1, ns[k]), -2.0, dtype=torch.float64),
                       torch.full((1, ns[k]), 2.0, dtype=torch.float64), arrival=arrivals[k])
            k += 1
        if srv.idle():
            time.sleep(max(0.0, min(0.01, arrivals[k] - now)) if k < len(arrivals) else 0.0)
            continue
        srv.step()
    torch.cuda.synchronize(dev)
    srv.close()
    wall = clock()
    done = list(srv.done.values())
    ttg = sorted(r.finished - r.arrival for r in done if r.status == "closed")
    tis = sorted(r.finished - r.arrival for r in done)
    q = lambda v, p: v[min(len(v) - 1, int(round(p * (len(v) - 1))))] if v else None
    return {"workload": "quad-exp family, n log-uniform [5, 2000], m = 2", "arrival_rate_per_s": rate,
            "arrival_seconds": seconds, "requests": len(arrivals), "closed": len(ttg),
            "budget_reached": sum(1 for r in done if r.status == "budget"),
            "emptied": sum(1 for r in done if r.status == "emptied"),
            "preempted": sum(1 for r in done if r.status == "preempted"),
            "closed_by_n": {f"{a}-{b}": [sum(1 for r in done if a <= r.lo.shape[1] <= b and r.status == "closed"),
                                         sum(1 for r in done if a <= r.lo.shape[1] <= b)]
                            for a, b in ((5, 10), (11, 15), (16, 20), (21, 50), (51, 2000))},
            "time_to_gap_s": {"p50": q(ttg, 0.5), "p99": q(ttg, 0.99)},
            "time_in_system_s": {"p50": q(tis, 0.5), "p99": q(tis, 0.99)},
            "subdomains_per_s": srv.bounded / wall, "rounds": srv.rounds, "max_concurrent": srv.max_live,
            "rel_gap": rel_gap, "budget_s": budget, "batch_per_instance_max": batch, "round_bytes": round_bytes,
            "max_live": max_live, "waited_out": sum(1 for r in done if r.admitted is None),
            "admission": admission, "incumbent_every": incumbent_every, "round_cap": round_cap,
            "compile_workers": compile_workers, "preempt": preempt,
            "closed_n_max": max((r.lo.shape[1] for r in done if r.status == "closed"), default=None),
            "host_s": {"rounds": srv.t_round, "crown_launch_calls": srv.t_bound}, "wall_s": wall,
            "form": "device queues, per-request CUDA graphs (DeviceServer)" if device_queues else
                    "host-driven rounds (Server)",
            "timing": "wall clock; time to gap from each request's arrival to the round that closed it"}


def plain_gpu(dev, workload, lo, hi, fused_value, steps=3, warmup=1):
    """The plain GPU form on the headline workload (PlainEngine: one launch per schedule step
    and per op, box state through global memory), the same boxes: subdomains/s and the fused
    path's multiple of it."""
    import torch
    from gear_b200 import graph, problems
    from gear_b200.engine import PlainEngine
    m = problems.make_instance(workload, 0)
    pe = PlainEngine(graph.trace(m, lo[:2]))
    xl, xu = lo.to(dev), hi.to(dev)
    B = lo.shape[0]
    out = (torch.empty(B, pe.S, dtype=torch.float64, device=dev),
           torch.empty(B, pe.S, pe.n, dtype=torch.float64, device=dev),
           torch.empty(B, pe.S, dtype=torch.float64, device=dev))
    for _ in range(warmup):
        pe.lower(xl, xu, out=out)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        pe.lower(xl, xu, out=out)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    value = B / (ms / 1000.0)
    return {"value": value, "unit": UNIT, "ms_per_step": ms, "launches_per_step": pe.launches,
            "fused_vs_plain": fused_value / value,
            "form": "same device code, one launch per schedule step and per op of each CROWN pass, "
                    "box state in global memory between launches"}, out


def constrained(dev, cases=((1024, 200, 20), (4096, 50, 16), (65536, 200, 20)), steps=5, warmup=2):
    """Constrained concretisation (the reference's sort_out_constr_batches + constraints_solving,
    concretize_func.py:312-850, as one device call gear_constrained_lower) on
    problems.cut_rows(batch, n, rows): one objective row per box, rows that cut, skip or exclude
    the box. Inputs resident on the device; CUDA-event time per call. The first two cases are the
    ones the reference's PyTorch sweep was timed on, on CPU cores, by oracle/reference_cpu.py."""
    import torch
    from gear_b200 import problems
    from gear_b200.concretize import constraints_solving
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = []
    for batch, n, rows in cases:
        xl, xu, obj, A, b = (t.to(dev) for t in problems.cut_rows(batch, n, rows))
        for _ in range(warmup):
            lb, inf = constraints_solving(xl, xu, obj, (A, b), return_infeasible=True)
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(steps):
            constraints_solving(xl, xu, obj, (A, b))
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / steps
        out.append({"batch": batch, "n": n, "rows": rows, "ms_per_call": ms, "boxes_per_s": batch / (ms / 1000.0),
                    "infeasible": int(inf.sum()), "finite_bounds": int(torch.isfinite(lb).sum()),
                    "input_bytes": int(8 * batch * (2 * n + n + rows * n + rows))})
    return {"api": "gear_b200.concretize.constraints_solving (gear_constrained_lower)", "cases": out}


def dense_nodes(dev, batch=8192, steps=3, warmup=1):
    """The dense-node configuration (dense_a_n2048: y = A x with A 1024 x 2048, objective
    sum alpha_j y_j^2 + beta_j y_j y_{j+1}), `batch` boxes: CROWN with the fold products of the
    dense node on the tensor cores (int8 digit slicing on tcgen05, fold_tc.cuh) against the same
    kernel with the fold on FP64 CUDA cores; the tensor-core fold kernel alone; the error of the
    tensor-core path against the FP64 one (both with exact-arithmetic McCormick ties, so the
    difference is the fold's own; with the default tie rule tie-decided rows can differ more)."""
    import torch
    from gear_b200 import _lib, graph, problems
    from gear_b200.engine import CrownEngine
    wl = "dense_a_n2048"
    m = problems.make_instance(wl, 0)
    lo, hi = problems.make_boxes(wl, batch, 0)
    g = graph.trace(m, lo[:2])
    xL, xU = lo.to(dev), hi.to(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / steps

    res = {"workload": wl, "batch": batch, "n": 2048, "dense_node": "1024 x 2048"}
    lbs = {}
    for name, tc, tie in (("tensor_core_fold", True, "reference"), ("cuda_core_fold", False, "reference"),
                          ("tensor_core_fold_exact_ties", True, "exact"), ("cuda_core_fold_exact_ties", False, "exact")):
        eng = CrownEngine(g, mode="cta", cta_threads=256, fold_tc=tc, tie_rule=tie)
        out = eng.lower(xL, xU)
        if tie == "reference":
            ms = timed(lambda: eng.lower(xL, xU, out=out))
            res[name] = {"ms_per_call": ms, "subdomains_per_s": batch / (ms / 1000.0)}
        torch.cuda.synchronize(dev)
        lbs[name] = out[0].clone()
        if name == "tensor_core_fold":
            L = _lib.lib()
            ws = torch.empty(int(L.gear_crown_fold_workspace_bytes(eng.handle, batch)), dtype=torch.uint8, device=dev)
            fold = torch.empty(batch, eng.prog.fold_w, dtype=torch.float64, device=dev)
            st = torch.cuda.current_stream(dev).cuda_stream
            fms = timed(lambda: _lib.check(L.gear_crown_fold_vectors(eng.handle, xL.data_ptr(), xU.data_ptr(), batch,
                                                                     fold.data_ptr(), None, ws.data_ptr(), ws.numel(),
                                                                     st), "gear_crown_fold_vectors"))
            k_pad, w, K = (2048 + 63) // 64 * 64, 1024, 2048
            macs = 2 * 15 * batch * w * k_pad            # two products, 15 digit pairs (levels 2..6)
            res["fold_kernels_ms"] = fms
            res["fold_int8_tops"] = 2 * macs / (fms / 1000.0) / 1e12
            res["fold_fp64_equivalent_tflops"] = 2 * 2 * batch * w * K / (fms / 1000.0) / 1e12
            res["fold_kernels"] = "box_digits_kernel + fold_tc_kernel (tcgen05.mma.kind::i8, TMEM accumulators)"
            del ws, fold
        del eng, out
    a, b = lbs["tensor_core_fold_exact_ties"], lbs["cuda_core_fold_exact_ties"]
    res["error_vs_fp64"] = {"max_rel_lb": float(((a - b).abs() / torch.clamp(b.abs(), min=1.0)).max()),
                            "tie_rule": "exact (both)", "tolerance": 1e-5}
    a, b = lbs["tensor_core_fold"], lbs["cuda_core_fold"]
    res["default_rule_difference"] = {"max_rel_lb": float(((a - b).abs() / torch.clamp(b.abs(), min=1.0)).max())}
    res["speedup_tensor_core_fold"] = res["cuda_core_fold"]["ms_per_call"] / res["tensor_core_fold"]["ms_per_call"]
    return res


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
    ap.add_argument("--mixed-instances", type=int, default=512,
                    help="also bound the uneven batch of this many mixed-family instances in one launch per "
                         "kernel variant against one launch per instance; 0 skips it")
    ap.add_argument("--mixed-boxes", type=int, default=256, help="sub-boxes per mixed-family instance")
    ap.add_argument("--e2e-chunk", type=int, default=16384, help="boxes per chunk of the pipelined end-to-end call")
    ap.add_argument("--no-mixed-baselines", dest="mixed_baselines", action="store_false",
                    help="time only the packed launch of the uneven batch (no per-instance or plain-form runs)")
    ap.add_argument("--mixed-bab-seconds", type=float, default=45.0,
                    help="time limit of branch and bound on the uneven batch (all instances at once), for the "
                         "packed arm and again for the plain-form arm; 0 skips it")
    ap.add_argument("--serve-seconds", type=float, default=120.0,
                    help="run the serving loop under Poisson arrivals (50 per second) for this long; 0 skips it")
    ap.add_argument("--dense-batch", type=int, default=8192,
                    help="boxes of the dense-node configuration (dense_a_n2048, tensor-core fold); 0 skips it")
    ap.add_argument("--no-constrained", dest="constrained", action="store_false",
                    help="skip the constrained-concretisation block")
    ap.add_argument("--no-plain", dest="plain", action="store_false",
                    help="skip the plain GPU form (one launch per step and per op) on the workload")
    ap.add_argument("--workload", default=WORKLOAD, help="benchmark workload (profiling of other shapes)")
    ap.add_argument("--cta-threads", type=int, default=128, help="threads per CTA of --mode cta")
    ap.add_argument("--mode", default="tune", choices=["tune", "auto", "cta", "simt"],
                    help="CROWN kernel: the autotuner's pick (execution shape, working-set placement, GEMV "
                         "tile, tensor-core fold, searched on the first call), the faster of four variants, one "
                         "box per CTA, or one box per thread")
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
    if hasattr(eng, "kernel_name"):
        kname = eng.kernel_name(B)
    else:
        kname = "crown_simt_kernel" if variant == "simt" else f"crown_megakernel<{variant[3:]}, 0, 0>"

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

    def e2e_pipelined_step():
        # the public host-buffer call: chunked copies in / kernels / lb rows out on three streams
        bm.compute_bounds_host(hL, hU, chunk=args.e2e_chunk)   # lb lands in pinned host memory

    def timed_e2e(fn):
        fn()
        torch.cuda.synchronize()
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        for _ in range(e_steps):
            fn()
        f1.record()
        torch.cuda.synchronize()
        return B * e_steps * world / (max_over_ranks(f0.elapsed_time(f1), world, dev) / 1000.0)

    e2e_serial = timed_e2e(e2e_step)
    e2e_value = timed_e2e(e2e_pipelined_step)

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
                traffic = tj.get(args.workload, {}).get(kname.split(",")[0] + (">" if "," in kname else ""), {}).get("bytes_per_box")
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
                            "kernel": kname,
                            "peak_source": peak_kind,
                            "alg_bytes_per_box": prog.alg_bytes_per_box(), "work_per_box": prog.work,
                            "fp64_gemm_gflops": prog.work["gemm_flops"] * B / (ms_launch / 1000.0) / 1e9},
               "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * B * n * 8,
                       "d2h_bytes_per_step": B * S * 8,
                       "api": f"BoundedModule.compute_bounds_host (pinned host boxes in, lb out; chunks of "
                              f"{args.e2e_chunk} boxes, copies overlapped with the kernels)",
                       "serial_value": e2e_serial,
                       "serial_api": "compute_bounds on boxes copied in first, lb copied out after"},
               "clocks": clk.summary()}
        if args.plain:
            pg, pout = plain_gpu(dev, args.workload, lo, hi, value)
            pg["bitwise_equal"] = bool(torch.equal(pout[0], lb) and torch.equal(pout[1], lA))
            res["plain_gpu"] = pg
            del pout
        if args.bab_instances > 0:
            res["bab"] = bab_to_gap(args.bab_instances, dev)
        if args.mixed_instances > 0:
            setup = mixed_setup(args.mixed_instances)
            res["mixed"] = mixed_batch(dev, setup, args.mixed_boxes, baselines=args.mixed_baselines)
            if args.mixed_bab_seconds > 0:
                res["mixed_bab"] = mixed_bab(dev, setup, time_limit=args.mixed_bab_seconds)
                if args.mixed_baselines:
                    pb = mixed_bab(dev, setup, time_limit=args.mixed_bab_seconds, plain=True)
                    res["mixed_bab_plain"] = pb
                    res["mixed_bab_vs_plain"] = {
                        "certified_subdomains_per_s_ratio": res["mixed_bab"]["subdomains_per_s"] / pb["subdomains_per_s"],
                        "closed": [res["mixed_bab"]["closed"], pb["closed"]], "target": 10.0}
        if args.dense_batch > 0:
            res["dense_nodes"] = dense_nodes(dev, batch=args.dense_batch)
        if args.constrained:
            res["constrained"] = constrained(dev)
        if args.serve_seconds > 0:
            res["serve"] = serve(dev, seconds=args.serve_seconds)
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
