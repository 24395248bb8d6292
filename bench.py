"""Benchmark: converged physical steps per second of the artificial-compressibility loop.

A bench step is one converged physical step (a pseudo-time loop run to max residual < eps) of
every case of the workload.  ``value`` is the whole-job throughput in converged physical steps
per second with the state resident in HBM; ``e2e`` is the same metric through the C ABI with the
state copied from pinned host buffers before and back after every step.

The default workload, ws-153, is the batched solver with the learned warm start: 16 held-out
cases at 153 x 153 drawn from the batched configuration's parameter distribution, each step
started from the best of the plain, extrapolated and learned start (the U-Net inference and the
start selection are inside the timed region).  The plain GPU path is timed on the same steps
from the same state and reported beside it (``plain_gpu``).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--arith exact|fast]
    python bench.py --impl reference ...   # the CPU implementation of the loop on host cores

Warm-start policy options (off by default): --extrap-order 2 (quadratic extrapolated
candidate), --warm-eps E (residual tolerance of the warm-started cases of each step).

Multi-GPU (torchrun): each rank runs its own replica of the workload (cases are independent, so
there is no exchange on the data path); the elapsed time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: description
    "ws-153": "batched solver + learned warm start: 16 cases at 153 x 153, Re U[50,500], Da logU[1e-5,1e-2], "
              "porosity U[0.3,0.9], Ri U[0,2], random block position (30% area), full equation set, QUICK, "
              "residual 1e-6; cases seeded apart from the network's training cases",
    "full-102": "full equation set (u, v, p, T, C), QUICK, porous block 30% (porosity 0.4, Da 1e-3, Cf 0.55), "
                "Ri 1, Pr 0.7, Sc 1, Re 200, 102 x 102 stretched 2:1 channel, beta 1, dt 1e-3, residual 1e-6",
    "full-204": "as full-102 on a 204 x 204 mesh",
    "large-1024x512": "the combined configuration's single large case: 1024 x 512 stretched 2:1 channel, two porous "
                      "blocks (10% of the area each, porosity 0.4, Da 1e-3, Cf 0.55), Ri 1, Pr 0.7, Sc 1, scalars T "
                      "and C, Re 400, QUICK, residual 1e-6",
    "plain-51": "plain method (u, v, p), first-order upwind, isothermal, no porous block, Re 100, 51 x 51 "
                "stretched 2:1 channel, beta 1, dt 1e-3, residual 1e-6",
    "batch-256": "256 independent cases, nx, ny in {51,102,153,204}, Re U[50,500], Da logU[1e-5,1e-2], "
                 "porosity U[0.3,0.9], Ri U[0,2], random block position, full equation set, QUICK",
}
BYTES_PER_CELL_UPDATE = {"full": 204, "plain": 112}   # each FP64 field read and written once per routine
# per-node algorithmic bytes of the timed u-momentum kernel: reads u_in, um, um_tau, vm_tau, pn
# (5 x 8 B) and the porous mask (1 B), writes u_out (8 B)
U_KERNEL_BYTES = {"exact": 49, "fast": 41}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def max_over_ranks(x: float, world: int, device=None) -> float:
    """Max of a per-rank scalar over all ranks (the elapsed time of a step is the slowest rank's);
    the identity on one rank."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed_offset(rank: int) -> int:
    """Rank r runs its own replica of the workload with the seeds shifted by r (weak scaling:
    the same case sizes and parameter distribution, different cases, no data exchange)."""
    return rank


def build_workload(pkg, name, arith, seed_offset=0, max_iters=None):
    items, kind = _build_workload(pkg, name, arith, seed_offset)
    if max_iters:
        from dataclasses import replace
        items = [(replace(p, itc_max=max_iters),) + tuple(rest) for p, *rest in items]
    return items, kind


WS_CASES, WS_N, WS_SEED = 16, 153, 101   # held-out seed (the network trains on seed 100)


def _build_workload(pkg, name, arith, seed_offset=0):
    cfg = pkg.configs
    a = pkg.ARITH_FAST if arith == "fast" else pkg.ARITH_EXACT
    if name == "ws-153":
        items, _ = cfg.cfg_batch(WS_CASES, seed=WS_SEED + 1000 * seed_offset, sizes=(WS_N,), arith=a)
        return items, "full"
    if name == "batch-256":
        items, _ = cfg.cfg_batch(256, seed=seed_offset, arith=a)
        return items, "full"
    if name.startswith("large-"):
        nx, ny = (int(v) for v in name.split("-")[1].split("x"))
        prm, mesh, st, itc, _ = cfg.cfg_large(nx, ny, arith=a, seed=2 + seed_offset)
        return [(prm, mesh, st, itc)], "full"
    if name.startswith("full-"):
        n = int(name.split("-")[1])
        prm, mesh, st, itc, _ = cfg.cfg_full(n, arith=a, seed=1 + seed_offset)
        return [(prm, mesh, st, itc)], "full"
    if name.startswith("plain-"):
        n = int(name.split("-")[1])
        prm, mesh, st, itc, _ = cfg.cfg_plain(n, arith=a, seed=seed_offset)
        return [(prm, mesh, st, itc)], "plain"
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except OSError:
            rows = []
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) >= 9:
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def cpu_sample(orc, items, gpu_iters_per_step, budget_s=12.0, threads=None):
    """Time the oracle (the CPU implementation of the loop) on a bounded sample: for up to three
    cases, a capped number of pseudo-iterations from the case's current state; extrapolate the
    seconds per converged step with the pseudo-iteration counts of the GPU run (identical by
    the parity tests)."""
    import numpy as np
    from dataclasses import replace
    threads = threads or os.cpu_count() or 1
    orc.set_threads(threads)
    picks = sorted(range(len(items)), key=lambda c: items[c][0].imax * items[c][0].jmax)
    picks = [picks[0], picks[len(picks) // 2], picks[-1]] if len(picks) > 3 else picks
    per_cell_iter = []
    sampled = 0
    t_each = budget_s / len(picks)
    for c in picks:
        prm, mesh, st = items[c][0], items[c][1], items[c][2]
        cells = prm.imax * prm.jmax
        # size the sample to ~t_each seconds from a short probe
        probe = 20
        o = orc.OracleCase(replace(prm, itc_max=probe), mesh)
        s = {k: np.asfortranarray(v.copy()) for k, v in st.items()}
        t0 = time.perf_counter(); o.run(s, 1, 0); dt = time.perf_counter() - t0
        m = max(20, int(t_each / max(dt / probe, 1e-9)))
        o = orc.OracleCase(replace(prm, itc_max=m), mesh)
        t0 = time.perf_counter(); _, it, _ = o.run(s, 1, 0); dt = time.perf_counter() - t0
        per_cell_iter.append(dt / (int(it[0]) * cells))
        sampled += int(it[0])
    t_cell = statistics.mean(per_cell_iter)
    sec_per_step = sum(gpu_iters_per_step[c] * items[c][0].imax * items[c][0].jmax * t_cell
                       for c in range(len(items)))
    return {"steps_per_s": len(items) / sec_per_step, "cores": threads,
            "sample": f"{sampled} pseudo-iterations of {len(picks)} case(s) of the workload from its "
                      f"post-warm-up state; seconds per cell-iteration x the GPU run's pseudo-iterations "
                      f"per converged step"}


def run_product(args):
    import numpy as np
    import torch
    import __graft_entry__ as entry

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    pkg = entry.load_package()
    if pkg.device_count() < 1:
        raise SystemExit("no CUDA device")
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream()
    items, kind = build_workload(pkg, args.workload, args.arith, seed_offset=replica_seed_offset(rank),
                                 max_iters=args.max_iters)
    if args.workload.startswith("ws-"):
        return run_ws(args, pkg, items, kind, world, rank, dev, stream)
    tuned = None
    from importlib import import_module
    if args.launch_shape:
        t, c_, n_ = (int(v) for v in args.launch_shape.split(","))
        tuned = {"threads": t, "ctas_per_sm": c_, "nodes_per_cta": n_, "staged": args.stage}
    elif args.arith == "fast" and args.engine == "cluster":
        tuned = import_module(pkg.__name__ + ".autotune").tune(pkg, items, use_cache=not args.retune)
    eng_used = "graph" if (tuned or {}).get("engine") == 1 else args.engine
    batch = pkg.Batch([x[0] for x in items], [x[1] for x in items])
    batch.set_stream(stream.cuda_stream)
    batch.set_option(pkg.OPT_ENGINE, 0 if args.engine == "cluster" else 1)
    batch.set_option(pkg.OPT_STAGED, args.stage)
    if tuned:
        import_module(pkg.__name__ + ".autotune").apply(batch, pkg, tuned)
    for c, x in enumerate(items):
        batch.set_state(c, x[2])
    itc = np.array([x[3] for x in items], np.int32)
    n_cases = len(items)
    cells = sum(x[0].imax * x[0].jmax for x in items)
    l2 = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2

    for w in range(args.warmup):
        itc, _, _, st = batch.run(1, itc)
    torch.cuda.synchronize()
    # snapshot of the loop state at the start of the timed steps, so the end-to-end pass below
    # replays exactly the same steps (same pseudo-iteration counts)
    snap = [batch.get_state(c) for c in range(n_cases)]
    itc_snap = itc.copy()
    if world > 1:
        dist.barrier()
    iters = np.zeros((n_cases, args.steps), np.int64)
    launches = 0
    t_ev0, t_ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        torch.cuda.synchronize()
        t_ev0.record(stream)
        for k in range(args.steps):
            l2.fill_(float(k))
            itc, it, _, st = batch.run(1, itc)
            iters[:, k] = it[:, 0]
            launches += batch.launch_count()
        t_ev1.record(stream)
        torch.cuda.synchronize()
    elapsed = max_over_ranks(t_ev0.elapsed_time(t_ev1) / 1e3, world, dev)
    total_iters = int(iters.sum())
    steps_done = n_cases * args.steps
    capped = int(sum((iters[c] >= items[c][0].itc_max - 1).sum() for c in range(n_cases)))
    if args.record_iterations and rank == 0:
        with open(args.record_iterations, "w") as f:
            json.dump({"workload": args.workload, "warmup": args.warmup, "steps": args.steps,
                       "iterations": iters.tolist()}, f)
    value = steps_done * world / elapsed

    peak, peak_kind = measured_peaks()
    b_cu = BYTES_PER_CELL_UPDATE[kind]
    cell_updates = sum(iters[c].sum() * items[c][0].imax * items[c][0].jmax for c in range(n_cases))
    loop_gbs = b_cu * cell_updates / elapsed / 1e9
    if eng_used == "cluster":
        # the persistent engine kernel is the whole loop: one launch per size class and step
        kern = "k_engine (persistent cluster engine, %s arithmetic)" % args.arith
        achieved = loop_gbs
        per_launch = {"bytes_per_cell_update": b_cu, "launches": launches,
                      "cell_updates_per_launch": cell_updates / max(launches, 1),
                      "ms_per_launch": elapsed * 1e3 / max(launches, 1)}
    else:
        ms_u, nodes_u = batch.time_kernel(0, reps=50)
        b_node = U_KERNEL_BYTES[args.arith]
        kern = "k_u_stage_%s (u-momentum stage, graph engine)" % args.arith
        achieved = b_node * nodes_u / (ms_u * 1e-3) / 1e9
        per_launch = {"bytes_per_node": b_node, "nodes_per_launch": nodes_u, "ms_per_launch": ms_u}
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "engine_dram_bytes.json")
    if eng_used == "cluster" and os.path.exists(tfile):
        with open(tfile) as f:
            bpcu = json.load(f).get(kind, {}).get("dram_bytes_per_cell_update")
        if bpcu:
            traffic = bpcu * cell_updates / max(launches, 1)

    # end to end through the C ABI with host buffers (pinned): the same steps as the timed region
    e2e_steps = args.steps
    itc = itc_snap.copy()
    host = []
    h2d = d2h = 0
    for c in range(n_cases):
        got = snap[c]
        pinned = {}
        for n, a in got.items():
            t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
            v = t.numpy().reshape(a.shape, order="F")
            v[...] = a
            pinned[n] = (t, v)
            h2d += a.nbytes
            d2h += a.nbytes
        host.append(pinned)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        for c in range(n_cases):
            batch.set_state(c, {n: v for n, (t, v) in host[c].items()})
        itc, _, _, _ = batch.run(1, itc)
        for c in range(n_cases):
            batch.get_state(c, out={n: v for n, (t, v) in host[c].items()})
    torch.cuda.synchronize()
    e2e_elapsed = max_over_ranks(time.perf_counter() - t0, world, dev)
    e2e = n_cases * e2e_steps * world / e2e_elapsed

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as orc
        gips = [float(iters[c].mean()) for c in range(n_cases)]
        state_items = [(x[0], x[1], batch.get_state(c), 0) for c, x in enumerate(items)]
        cpu = cpu_sample(orc, state_items, gips, budget_s=args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": "converged physical steps/s at pseudo-time residual 1e-6",
            "value": value,
            "unit": "steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": elapsed / args.steps * 1e3,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded channel cases; no public dataset)",
            "config": {
                "workload": args.workload,
                "description": WORKLOADS[args.workload],
                "cases_per_gpu": n_cases,
                "cells_per_gpu": cells,
                "arith": args.arith,
                "engine": "graph" if (tuned or {}).get("engine") == 1 else args.engine,
                "staged": args.stage,
                "launch_shape": tuned,
                "pseudo_iterations_per_step_mean": total_iters / steps_done,
                "steps_capped_at_itc_max": capped,
                "l2": "flushed (256 MB write) before every timed step",
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            },
            "cell_updates_per_s": cell_updates * world / elapsed,
            "roofline": dict({
                "bound": "hbm",
                "kernel": kern,
                "achieved": achieved,
                "peak": peak,
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs, burst)" if peak_kind == "measured" else "fallback",
                "unit": "GB/s",
                "frac": achieved / peak,
                "traffic": traffic,
            }, **per_launch),
            "loop_roofline": {
                "bytes_per_cell_update": b_cu,
                "achieved": loop_gbs,
                "unit": "GB/s",
                "frac": loop_gbs / peak,
            },
            "e2e": {"value": e2e, "unit": "steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        if cpu is not None:
            line["cpu_baseline"] = {"value": cpu["steps_per_s"], "unit": "steps/s", "cores": cpu["cores"],
                                    "kind": "port", "sample": cpu["sample"]}
        print(json.dumps(line))
    batch.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _tuned_batch(pkg, items, args, stream):
    from importlib import import_module
    tuned = None
    if args.launch_shape:
        t, c_, n_ = (int(v) for v in args.launch_shape.split(","))
        tuned = {"threads": t, "ctas_per_sm": c_, "nodes_per_cta": n_, "staged": args.stage}
    elif args.arith == "fast" and args.engine == "cluster":
        tuned = import_module(pkg.__name__ + ".autotune").tune(pkg, items, use_cache=not args.retune)

    def make(states=None):
        b = pkg.Batch([x[0] for x in items], [x[1] for x in items])
        b.set_stream(stream.cuda_stream)
        b.set_option(pkg.OPT_ENGINE, 0 if args.engine == "cluster" else 1)
        b.set_option(pkg.OPT_STAGED, args.stage)
        if tuned:
            import_module(pkg.__name__ + ".autotune").apply(b, pkg, tuned)
        for c, x in enumerate(items):
            b.set_state(c, states[c] if states is not None else x[2])
        return b
    return make, tuned


def run_ws(args, pkg, items, kind, world, rank, dev, stream):
    """Batched solver with the learned warm start (ws-* workloads)."""
    import numpy as np
    import torch
    from importlib import import_module
    ws = import_module(pkg.__name__ + ".warmstart")
    unet = import_module(pkg.__name__ + ".unet")
    if world > 1:
        import torch.distributed as dist
    net, norm, H, W, meta = ws.load(args.weights)
    n_cases = len(items)
    make, tuned = _tuned_batch(pkg, items, args, stream)
    l2 = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2

    # cost-aware cluster sizes: a batched step lasts as long as its slowest case, so each case gets
    # CTAs in proportion to its pseudo-iterations of the previous step (cluster engine only)
    # the total stays that of the tuned launch shape; only its distribution over the cases changes
    # (--balance 2: the CTA slots of the whole GPU, SMs x CTAs per SM, instead)
    slots = 0
    if args.balance and tuned and tuned.get("engine", 0) == 0 and args.engine == "cluster":
        npc = tuned["nodes_per_cta"]
        for p, *_ in items:
            k = -(-((p.imax + 1) * (p.jmax + 1)) // npc)
            slots += max(1, min(k, 16, max(1, (p.jmax + 1) // 4)))
        if args.balance == 2:
            slots = max(slots, torch.cuda.get_device_properties(dev).multi_processor_count * tuned.get("ctas_per_sm", 1))

    def balance(batch, its):
        if slots and its is not None:
            batch.balance_clusters(its, slots)

    A = make()
    wA = ws.WarmStart(A, H, W, net, norm, extrap_order=args.extrap_order)
    itc = np.array([x[3] for x in items], np.int32)
    prev_snap = prev_snap2 = None
    it_last = None
    for w in range(args.warmup):
        if w == args.warmup - 2 and args.extrap_order == 2:
            prev_snap2 = [A.get_state(c) for c in range(n_cases)]
        if w == args.warmup - 1:
            prev_snap = [A.get_state(c) for c in range(n_cases)]
        itc, it_last, _, _ = wA.step(itc, "learned", warm_eps=args.warm_eps)
        balance(A, it_last)
    it_warm_last = None if it_last is None else np.array(it_last)
    torch.cuda.synchronize()
    snap = [A.get_state(c) for c in range(n_cases)]
    itc_snap = itc.copy()

    def timed(step_fn, batch, itc):
        """K steps; returns (elapsed s, iterations [n, K], chosen starts [n, K], engine ms, start ms,
        launches)."""
        iters = np.zeros((n_cases, args.steps), np.int64)
        chosen = np.zeros((n_cases, args.steps), np.int64)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        eng_ms = 0.0
        launches = 0
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ev[0].record(stream)
        for k in range(args.steps):
            l2.fill_(float(k))
            itc, it, ch, ms = step_fn(batch, itc)
            iters[:, k] = it
            chosen[:, k] = ch
            eng_ms += ms
            launches += batch.launch_count()
        ev[1].record(stream)
        torch.cuda.synchronize()
        el = max_over_ranks(ev[0].elapsed_time(ev[1]) / 1e3, world, dev)
        return el, iters, chosen, eng_ms, launches, itc

    def ws_step(batch, itc, w=wA):
        w.features()
        y = w.predict()
        chosen, _ = batch.set_start(y.data_ptr(), 8, w.norm.out_scale.data_ptr(), pkg.POLICY_BEST)
        if args.warm_eps is not None:
            for c in range(n_cases):
                batch.set_tolerance(c, args.warm_eps if chosen[c] != pkg.START_PLAIN else batch.params[c].eps)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        itc, it, _, _ = batch.run(1, itc)
        e1.record(stream)
        e1.synchronize()
        balance(batch, it[:, 0])
        return itc, it[:, 0], chosen, e0.elapsed_time(e1)

    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        el_ws, it_ws, ch_ws, eng_ms, launches, _ = timed(ws_step, A, itc_snap.copy())
    A.close()
    # network inference alone, timed on the same canvas (FLOPs of the 15 convolutions)
    x_in = net.input_buffer(n_cases, H, W)
    for _ in range(2):
        net.forward(n_cases, H, W)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    reps = 5
    for _ in range(reps):
        net.forward(n_cases, H, W)
    e1.record(stream)
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1) / reps
    fwd_flops = unet.conv_flops(H, W) * n_cases
    del x_in

    # plain GPU path, same steps from the same state: all K steps in one persistent launch, each
    # case advancing through its steps on its own
    B = make(snap)
    balance(B, it_warm_last)
    if world > 1:
        dist.barrier()
    l2.fill_(-1.0)
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    _, it_pl, _, _ = B.run(args.steps, itc_snap.copy())
    p1.record(stream)
    torch.cuda.synchronize()
    el_pl = max_over_ranks(p0.elapsed_time(p1) / 1e3, world, dev)
    it_pl = np.asarray(it_pl, np.int64)
    plain_state = [B.get_state(c, ("um", "vm", "pn", "T", "C")) for c in range(n_cases)]
    B.close()

    # end to end through the C ABI with pinned host buffers: the same steps again
    C_ = make(prev_snap2 if prev_snap2 is not None else prev_snap)
    balance(C_, it_warm_last)
    wC = ws.WarmStart(C_, H, W, net, norm, extrap_order=args.extrap_order)
    wC.features()                       # history: the fields at the start of the last warm-up step
    if prev_snap2 is not None:          # (and of the one before, for the quadratic candidate)
        for c in range(n_cases):
            C_.set_state(c, prev_snap[c])
        wC.features()
    host = []
    h2d = d2h = 0
    for c in range(n_cases):
        pinned = {}
        for nme, a in snap[c].items():
            t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
            v = t.numpy().reshape(a.shape, order="F")
            v[...] = a
            pinned[nme] = (t, v)
            h2d += a.nbytes
            d2h += a.nbytes
        host.append(pinned)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    itc = itc_snap.copy()
    it_e2e = np.zeros((n_cases, args.steps), np.int64)
    t0 = time.perf_counter()
    for k in range(args.steps):
        for c in range(n_cases):
            C_.set_state(c, {nme: v for nme, (t, v) in host[c].items()})
        itc, it, _, _ = ws_step(C_, itc, wC)
        it_e2e[:, k] = it
        for c in range(n_cases):
            C_.get_state(c, out={nme: v for nme, (t, v) in host[c].items()})
    torch.cuda.synchronize()
    e2e_el = time.perf_counter() - t0
    ws_state = [{k: host[c][k][1] for k in ("um", "vm", "pn", "T", "C")} for c in range(n_cases)]
    C_.close()
    e2e_el = max_over_ranks(e2e_el, world, dev)
    err = {}
    for c in range(n_cases):
        for k, v in ws.field_error(ws_state[c], plain_state[c]).items():
            err[k] = max(err.get(k, 0.0), v)

    # kernels of the warm start per step: history, scale, features; input normalisation; the
    # network (im2col + GEMM per convolution, pool/upsample/skip copy per level); candidates,
    # boundary passes, residual probes, commit
    n_unet = 2 * len(net.convs) + 3 * (net.levels - 1)
    ws_launches = args.steps * (3 + 1 + n_unet + 8)
    steps_done = n_cases * args.steps
    value = steps_done * world / el_ws
    plain_value = steps_done * world / el_pl
    peak, peak_kind = measured_peaks()
    b_cu = BYTES_PER_CELL_UPDATE[kind]
    cells = items[0][0].imax * items[0][0].jmax
    cu_ws = int(it_ws.sum()) * cells
    cu_pl = int(it_pl.sum()) * cells
    eng_gbs = b_cu * cu_ws / (eng_ms * 1e-3) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "engine_dram_bytes.json")
    if os.path.exists(tfile):
        with open(tfile) as f:
            bpcu = json.load(f).get(kind, {}).get("dram_bytes_per_cell_update")
        if bpcu:
            traffic = bpcu * cu_ws / max(launches, 1)
    bf16_peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            bf16_peak = float(json.load(f)["bf16_tflops"])
    except (OSError, KeyError, ValueError):
        bf16_peak = 1590.0
    if args.record_iterations and rank == 0:
        rec = {}
        if os.path.exists(args.record_iterations):
            with open(args.record_iterations) as f:
                rec = json.load(f)
        rec[args.workload] = {"warmup": args.warmup, "steps": args.steps,
                              "plain_iterations": it_pl.tolist(),
                              "mean_iterations_per_step": [float(v) for v in it_pl.mean(axis=1)],
                              "warm_start_iterations": it_ws.tolist()}
        with open(args.record_iterations, "w") as f:
            json.dump(rec, f, indent=1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as orc
        gips = [float(it_pl[c].mean()) for c in range(n_cases)]
        state_items = [(x[0], x[1], snap[c], 0) for c, x in enumerate(items)]
        cpu = cpu_sample(orc, state_items, gips, budget_s=args.cpu_seconds)
    if rank == 0:
        starts = np.bincount(ch_ws.ravel(), minlength=3) / ch_ws.size
        line = {
            "metric": "converged physical steps/s at pseudo-time residual 1e-6",
            "value": value,
            "unit": "steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": el_ws / args.steps * 1e3,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded channel cases; no public dataset)",
            "config": {
                "workload": args.workload,
                "description": WORKLOADS[args.workload],
                "cases_per_gpu": n_cases,
                "cells_per_gpu": cells * n_cases,
                "arith": args.arith,
                "engine": "graph" if (tuned or {}).get("engine") == 1 else args.engine,
                "staged": args.stage,
                "launch_shape": tuned,
                "network": {"weights": os.path.relpath(args.weights, ROOT), "canvas": [H, W],
                            "trained_snapshots": meta.get("snapshots")},
                "pseudo_iterations_per_step_mean": float(it_ws.mean()),
                "starts_plain_extrap_learned": starts.round(3).tolist(),
                "warm_start_tolerance": args.warm_eps if args.warm_eps is not None else "each case's own (1e-6)",
                "extrapolation_order": args.extrap_order,
                "cluster_sizes": ("the launch shape's CTAs redistributed in proportion to each case's pseudo-"
                                  f"iterations of the previous step, {slots} CTAs in total (plain run: by the "
                                  "last warm-up step)") if slots
                                 else "from the launch shape",
                "l2": "flushed (256 MB write) before every timed step",
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            },
            "plain_gpu": {"value": plain_value, "unit": "steps/s", "ms_per_step": el_pl / args.steps * 1e3,
                          "launch": "acs_batch_run over all timed steps in one launch (no per-step host sync)",
                          "pseudo_iterations_per_step_mean": float(it_pl.mean()),
                          "speedup_of_warm_start": value / plain_value,
                          "final_fields_max_rel_diff_warm_vs_plain": err},
            "cell_updates_per_s": cu_ws * world / el_ws,
            "roofline": {
                "bound": "hbm",
                "kernel": ("pseudo-time loop of the graph engine (per-stage kernels, %s arithmetic)" % args.arith
                           if (tuned or {}).get("engine") == 1 else
                           "k_engine (persistent cluster engine, %s arithmetic)" % args.arith),
                "achieved": eng_gbs,
                "peak": peak,
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs, burst)" if peak_kind == "measured" else "fallback",
                "unit": "GB/s",
                "frac": eng_gbs / peak,
                "traffic": traffic,
                "bytes_per_cell_update": b_cu,
                "launches": launches,
                "ms_per_launch": eng_ms / max(launches, 1),
                "engine_share_of_step": eng_ms * 1e-3 / el_ws,
            },
            "unet_inference": {"bound": "tensor", "flops_per_launch_set": fwd_flops, "ms": fwd_ms,
                               "achieved_tflops": fwd_flops / (fwd_ms * 1e-3) / 1e12,
                               "peak_tflops": bf16_peak, "frac": fwd_flops / (fwd_ms * 1e-3) / 1e12 / bf16_peak},
            "e2e": {"value": n_cases * args.steps * world / e2e_el, "unit": "steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": args.steps,
                    "same_iterations_as_timed": bool((it_e2e == it_ws).all())},
            "gpu_launches": launches + ws_launches,
            "gpu_launches_detail": {"engine": launches, "warm_start_and_network": ws_launches},
            "clocks": clk.summary(),
        }
        if cpu is not None:
            line["cpu_baseline"] = {"value": cpu["steps_per_s"], "unit": "steps/s", "cores": cpu["cores"],
                                    "kind": "port", "sample": cpu["sample"] + " (plain start's iteration counts)"}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def reference_iterations(workload):
    path = os.path.join(ROOT, "tests", "golden", "bench_iterations.json")
    try:
        with open(path) as f:
            return json.load(f).get(workload)
    except (OSError, ValueError):
        return None


def run_reference(args):
    """The reference's CPU implementation of the loop (the oracle restatement: the Fortran
    reference cannot be compiled without a Fortran compiler) on the host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import numpy as np
    import __graft_entry__ as entry
    from oracle import oracle as orc
    pkg = entry.load_package()
    items, kind = build_workload(pkg, args.workload, args.arith, max_iters=args.max_iters)
    rec = reference_iterations(args.workload)
    if rec is None:
        print(json.dumps({"impl": "reference", "unavailable": "tests/golden/bench_iterations.json lacks "
                          f"pseudo-iteration counts for workload {args.workload}"}))
        return
    per_case = rec["mean_iterations_per_step"]
    gips = per_case if isinstance(per_case, list) else [per_case] * len(items)
    vals = []
    t0 = time.perf_counter()
    cpu = None
    for k in range(args.warmup + args.steps):
        cpu = cpu_sample(orc, items, gips, budget_s=max(2.0, args.cpu_seconds / max(1, args.steps)))
        if k >= args.warmup:
            vals.append(cpu["steps_per_s"])
    value = statistics.mean(vals)
    elapsed = time.perf_counter() - t0
    line = {
        "impl": "reference",
        "metric": "converged physical steps/s at pseudo-time residual 1e-6",
        "value": value,
        "unit": "steps/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 / value,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded channel cases; no public dataset)",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload], "cases": len(items),
                   "pseudo_iterations_per_step_mean": float(np.mean(gips)),
                   "source_of_iteration_counts": "tests/golden/bench_iterations.json"},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": cpu["cores"], "kind": "port",
                         "sample": cpu["sample"] + " (initial state of the workload)"},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": elapsed,
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--workload", default="ws-153", choices=sorted(WORKLOADS))
    ap.add_argument("--weights", default=os.path.join(ROOT, "solver-cfd_b200", "unet", "weights", "ws_153.npz"),
                    help="trained warm-start network (ws-* workloads)")
    ap.add_argument("--arith", default="fast", choices=["exact", "fast"])
    ap.add_argument("--engine", default="cluster", choices=["cluster", "graph"])
    ap.add_argument("--retune", action="store_true", help="ignore the autotuner cache")
    ap.add_argument("--launch-shape", default=None,
                    help="threads,ctas_per_sm,nodes_per_cta: skip the autotuner (profiling runs)")
    ap.add_argument("--stage", type=int, default=1, choices=[0, 1],
                    help="FAST engine: stage stencil arrays in shared memory (1) or read them from L1/L2 (0)")
    ap.add_argument("--balance", type=int, default=1, choices=[0, 1, 2],
                    help="ws-* workloads: cluster sizes in proportion to each case's pseudo-iterations "
                         "(1: within the tuned shape's CTA total, 2: within all CTA slots of the GPU)")
    ap.add_argument("--extrap-order", type=int, default=1, choices=[1, 2],
                    help="warm-start workload: linear (1) or quadratic (2) extrapolated candidate")
    ap.add_argument("--warm-eps", type=float, default=None,
                    help="warm-start workload: residual tolerance of the warm-started cases of each step "
                         "(default: every case keeps its own, 1e-6)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--max-iters", type=int, default=None,
                    help="cap the pseudo-iterations of every physical step (profiling runs; the steps "
                         "are then not converged)")
    ap.add_argument("--record-iterations", default=None,
                    help="write the per-step pseudo-iteration counts of the run to this JSON file")
    args = ap.parse_args()
    if args.warmup < 0 or args.steps < 1:
        raise SystemExit("bad --steps/--warmup")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_product(args)


if __name__ == "__main__":
    main()
