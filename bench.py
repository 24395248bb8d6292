"""Benchmark: converged physical steps per second of the artificial-compressibility loop.

A bench step is one converged physical step (a pseudo-time loop run to max residual < eps) of
every case of the workload; the unit is converged case-steps per second.  ``value`` is the
whole-job throughput with the state resident in HBM; ``e2e`` is the first ``--sample-steps``
of the same steps again through the C ABI with the state copied from pinned host buffers before
and back after every step.

The default workload, ws-153, is the learned-warm-start configuration: 64 held-out cases at
153 x 153 drawn from the batched configuration's parameter distribution (seed 101; the network
trained on seed 100), the tile engine, FAST arithmetic.  The W warm-up steps run from rest with
the reference's (plain) start, recording the warm-start history; the K timed steps each start
from the best of the plain, extrapolated and learned start (the U-Net inference and the start
selection inside the timed region).  The plain GPU path is timed on the first ``--sample-steps``
steps of the same window from the same state (``plain_gpu``).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--engine tile|cluster|graph]
    python bench.py --impl reference ...   # the CPU implementation of the loop on host cores

The reference arm runs the oracle (the C++ restatement of the reference's OpenMP loop; no
Fortran compiler exists here) on all host cores: for a sample of the workload's cases
(``--ref-cases``) it converges the W warm-up steps from rest and then times the first
``--sample-steps`` steps of the same window (the steps the product's e2e pass replays), every step
converged to the same tolerance with the reference's start.  A converged CPU step of a 153 x 153
case takes one to four minutes, so the sample is bounded to those steps.  Its cases are built
with the oracle's own mesh and noise generators, so it never loads this package's library.

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
    "ws-153": "learned warm start: 64 held-out cases at 153 x 153, Re U[50,500], Da logU[1e-5,1e-2], "
              "porosity U[0.3,0.9], Ri U[0,2], random block position (30% area), full equation set, QUICK, "
              "beta 1, dt 1e-3, residual 1e-6; cases seeded apart from the network's training cases",
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
ENGINES = {"cluster": 0, "graph": 1, "tile": 2}
# per-node algorithmic bytes of one launch of the tile engine's U/V stage kernel (stage 2): reads
# u_in, v_in, um_tau, vm_tau, pn, um, vm, T (8 x 8 B) and the porous indicator (1 B, as in the
# fused model), writes u_out, v_out (2 x 8 B)
TILE_UV_BYTES = 8 * 8 + 1 + 2 * 8
# DRAM bytes per node of one k_te_uv<2> launch, measured by ncu on the 64-case ws-153 workload
# (dram__bytes_read.sum + dram__bytes_write.sum = 111,727,616 + 8,363,520 bytes for 1,498,176
# nodes, one pass; the command is in profiles/tile_engine_ws153_ncu.md).  Other case counts are
# scaled by their nodes.
TILE_UV2_DRAM_BYTES_PER_NODE = (111727616 + 8363520) / 1498176


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


def build_workload(pkg, name, arith, seed_offset=0, max_iters=None, cases=None):
    items, kind = _build_workload(pkg, name, arith, seed_offset, cases)
    if max_iters:
        from dataclasses import replace
        items = [(replace(p, itc_max=max_iters),) + tuple(rest) for p, *rest in items]
    return items, kind


WS_CASES, WS_N, WS_SEED = 64, 153, 101   # held-out seed (the network trains on seed 100)


def _build_workload(pkg, name, arith, seed_offset=0, cases=None):
    cfg = pkg.configs
    a = pkg.ARITH_FAST if arith == "fast" else pkg.ARITH_EXACT
    if name == "ws-153":
        n = cases if cases else WS_CASES
        items, _ = cfg.cfg_batch(n, seed=WS_SEED + 1000 * seed_offset, sizes=(WS_N,), arith=a)
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
                                 max_iters=args.max_iters, cases=args.cases)
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
    batch.set_option(pkg.OPT_ENGINE, ENGINES[args.engine])
    if args.engine == "cluster":
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
    elif eng_used == "tile":
        ms_u, nodes_u = batch.time_kernel(5, reps=20)
        b_node = TILE_UV_BYTES
        kern = "k_te_uv<2> (tile engine, U/V Runge-Kutta stage 2)"
        achieved = b_node * cells / (ms_u * 1e-3) / 1e9
        per_launch = {"bytes_per_node": b_node, "nodes_per_launch": cells, "ms_per_launch": ms_u}
    else:
        ms_u, nodes_u = batch.time_kernel(0, reps=50)
        b_node = U_KERNEL_BYTES[args.arith]
        kern = "k_u_stage_%s (u-momentum stage, graph engine)" % args.arith
        achieved = b_node * nodes_u / (ms_u * 1e-3) / 1e9
        per_launch = {"bytes_per_node": b_node, "nodes_per_launch": nodes_u, "ms_per_launch": ms_u}
    traffic = None  # DRAM bytes per launch come from ncu (profiles/), not from this run

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
                "engine": eng_used,
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
    if args.engine == "cluster":
        if args.launch_shape:
            t, c_, n_ = (int(v) for v in args.launch_shape.split(","))
            tuned = {"threads": t, "ctas_per_sm": c_, "nodes_per_cta": n_, "staged": args.stage}
        elif args.arith == "fast":
            tuned = import_module(pkg.__name__ + ".autotune").tune(pkg, items, use_cache=not args.retune)

    def make(states=None):
        b = pkg.Batch([x[0] for x in items], [x[1] for x in items])
        b.set_stream(stream.cuda_stream)
        b.set_option(pkg.OPT_ENGINE, ENGINES[args.engine])
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

    # ---- warm-up: W steps from rest with the reference's start; every step records the fields in
    # the warm-start history, so the first timed step can extrapolate
    A = make()
    wA = ws.WarmStart(A, H, W, net, norm, extrap_order=args.extrap_order)
    itc = np.array([x[3] for x in items], np.int32)
    hist = []   # states at the start of the last two warm-up steps (the end-to-end pass rebuilds
                # the same history from them)
    it_warmup = np.zeros((n_cases, args.warmup), np.int64)
    for w in range(args.warmup):
        hist = (hist + [[A.get_state(c) for c in range(n_cases)]])[-2:]
        wA.features()
        itc, it, _, _ = wA.step(itc, "plain")
        it_warmup[:, w] = it
    torch.cuda.synchronize()
    snap = [A.get_state(c) for c in range(n_cases)]
    itc_snap = itc.copy()

    def ws_step(w, batch, itc):
        w.features()
        y = w.predict()
        chosen, _ = batch.set_start(y.data_ptr(), 8, w.norm.out_scale.data_ptr(), pkg.POLICY_BEST)
        if args.warm_eps is not None:
            for c in range(n_cases):
                batch.set_tolerance(c, args.warm_eps if chosen[c] != pkg.START_PLAIN else batch.params[c].eps)
        itc, it, _, _ = batch.run(1, itc)
        return itc, it[:, 0], chosen

    # ---- timed: K warm-started steps, the state resident in HBM
    iters_ws = np.zeros((n_cases, args.steps), np.int64)
    chosen_ws = np.zeros((n_cases, args.steps), np.int64)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    launches = 0
    if world > 1:
        dist.barrier()
    itc = itc_snap.copy()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        torch.cuda.synchronize()
        ev[0].record(stream)
        for k in range(args.steps):
            l2.fill_(float(k))
            itc, it, ch = ws_step(wA, A, itc)
            iters_ws[:, k] = it
            chosen_ws[:, k] = ch
            launches += A.launch_count()
            ev[k + 1].record(stream)
        torch.cuda.synchronize()
    el_ws = max_over_ranks(ev[0].elapsed_time(ev[-1]) / 1e3, world, dev)
    step_s = [ev[k].elapsed_time(ev[k + 1]) / 1e3 for k in range(args.steps)]
    ws_state = [A.get_state(c, ("um", "vm", "pn", "T", "C")) for c in range(n_cases)]

    # the dominant kernel, timed alone on the live state (CUDA events on the batch's stream)
    roof_kernel = {"tile": 5, "graph": 0}.get(args.engine)
    k_ms = k_nodes = None
    if roof_kernel is not None:
        k_ms, k_nodes = A.time_kernel(roof_kernel, reps=20)
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

    # ---- end to end through the C ABI with pinned host buffers: the same K steps again, every
    # field uploaded before and downloaded after each step
    C_ = make(hist[0] if hist else None)
    wC = ws.WarmStart(C_, H, W, net, norm, extrap_order=args.extrap_order)
    for h in hist[1:]:
        wC.features()
        for c in range(n_cases):
            C_.set_state(c, h[c])
    if hist:
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
    n_e2e = max(1, min(args.steps, args.sample_steps))
    it_e2e = np.zeros((n_cases, n_e2e), np.int64)
    t0 = time.perf_counter()
    for k in range(n_e2e):
        for c in range(n_cases):
            C_.set_state(c, {nme: v for nme, (t, v) in host[c].items()})
        itc, it, _ = ws_step(wC, C_, itc)
        it_e2e[:, k] = it
        for c in range(n_cases):
            C_.get_state(c, out={nme: v for nme, (t, v) in host[c].items()})
    torch.cuda.synchronize()
    e2e_el = max_over_ranks(time.perf_counter() - t0, world, dev)
    C_.close()

    # ---- plain GPU path on the first m steps of the window from the same state, one launch
    m = max(1, min(args.steps, args.plain_steps if args.plain_steps is not None else args.sample_steps))
    B = make(snap)
    if world > 1:
        dist.barrier()
    l2.fill_(-1.0)
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    _, it_pl, _, _ = B.run(m, itc_snap.copy())
    p1.record(stream)
    torch.cuda.synchronize()
    el_pl = max_over_ranks(p0.elapsed_time(p1) / 1e3, world, dev)
    it_pl = np.asarray(it_pl, np.int64)
    plain_state = [B.get_state(c, ("um", "vm", "pn", "T", "C")) for c in range(n_cases)] if m == args.steps else None
    B.close()

    steps_done = n_cases * args.steps
    value = steps_done * world / el_ws
    plain_value = n_cases * m * world / el_pl
    warm_m_value = n_cases * m * world / max_over_ranks(sum(step_s[:m]), world, dev)
    peak, peak_kind = measured_peaks()
    b_cu = BYTES_PER_CELL_UPDATE[kind]
    cells = sum(x[0].imax * x[0].jmax for x in items)
    cu_ws = int(sum(iters_ws[c].sum() * items[c][0].imax * items[c][0].jmax for c in range(n_cases)))
    loop_gbs = b_cu * cu_ws / el_ws / 1e9
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            bf16_peak = float(json.load(f)["bf16_tflops"])
    except (OSError, KeyError, ValueError):
        bf16_peak = 1590.0
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as orc
        gips = [float(it_pl[c].mean()) for c in range(n_cases)]
        state_items = [(x[0], x[1], snap[c], 0) for c, x in enumerate(items)]
        cpu = cpu_sample(orc, state_items, gips, budget_s=args.cpu_seconds)
    if rank == 0:
        starts = np.bincount(chosen_ws.ravel(), minlength=3) / chosen_ws.size
        if k_ms is not None:
            kname = ("k_te_uv<2> (tile engine, U/V Runge-Kutta stage 2)" if args.engine == "tile"
                     else "k_u_stage (graph engine, u-momentum stage 1)")
            b_node = TILE_UV_BYTES if args.engine == "tile" else U_KERNEL_BYTES[args.arith]
            nodes = cells if args.engine == "tile" else k_nodes
            achieved = b_node * nodes / (k_ms * 1e-3) / 1e9
            roof = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                    "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs, burst)" if peak_kind == "measured" else "fallback",
                    "unit": "GB/s", "frac": achieved / peak,
                    "traffic": TILE_UV2_DRAM_BYTES_PER_NODE * nodes if args.engine == "tile" else None,
                    "bytes_per_node": b_node, "nodes_per_launch": nodes, "ms_per_launch": k_ms,
                    "traffic_note": ("bytes per launch: dram__bytes_read.sum + dram__bytes_write.sum of one "
                                     "ncu capture of k_te_uv<2> on the 64-case workload (80.2 B per node), "
                                     "scaled by this run's nodes" if args.engine == "tile" else
                                     "not captured for this engine")}
        else:
            roof = {"bound": "hbm", "kernel": "k_engine (persistent cluster engine)", "achieved": loop_gbs,
                    "peak": peak, "unit": "GB/s", "frac": loop_gbs / peak, "traffic": None,
                    "bytes_per_cell_update": b_cu}
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
                "cells_per_gpu": cells,
                "arith": args.arith,
                "engine": args.engine,
                "launch_shape": tuned,
                "network": {"weights": os.path.relpath(args.weights, ROOT), "canvas": [H, W],
                            "trained_snapshots": meta.get("snapshots")},
                "warmup_start": "plain (the reference's start), recording the warm-start history",
                "pseudo_iterations_per_step_mean": float(iters_ws.mean()),
                "pseudo_iterations_per_step_slowest_case_mean": float(iters_ws.max(axis=0).mean()),
                "warmup_pseudo_iterations_per_step_mean": it_warmup.mean(axis=0).round(1).tolist(),
                "starts_plain_extrap_learned": starts.round(3).tolist(),
                "warm_start_tolerance": args.warm_eps if args.warm_eps is not None else "each case's own (1e-6)",
                "extrapolation_order": args.extrap_order,
                "l2": "flushed (256 MB write) before every timed step",
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            },
            "plain_gpu": {"value": plain_value, "unit": "steps/s", "steps": m, "ms_per_step": el_pl / m * 1e3,
                          "launch": f"acs_batch_run over the first {m} timed steps in one launch",
                          "pseudo_iterations_per_step_mean": float(it_pl.mean()),
                          # the same steps of the cases the reference arm converges on the CPU (its
                          # config.pseudo_iterations_per_step holds the oracle's counts of them)
                          "pseudo_iterations_of_reference_cases": {
                              str(c): [int(v) for v in it_pl[c]] for c in reference_picks(n_cases, args.ref_cases)},
                          "warm_start_value_same_steps": warm_m_value,
                          "speedup_of_warm_start": warm_m_value / plain_value,
                          "warm_pseudo_iterations_per_step_mean_same_steps": float(iters_ws[:, :m].mean()),
                          "final_fields_max_rel_diff_warm_vs_plain": (
                              {k: max(ws.field_error(ws_state[c], plain_state[c])[k] for c in range(n_cases))
                               for k in ("um", "vm", "pn", "T", "C")} if plain_state is not None else None)},
            "cell_updates_per_s": cu_ws * world / el_ws,
            "roofline": roof,
            "loop_roofline": {"bytes_per_cell_update": b_cu, "achieved": loop_gbs, "unit": "GB/s",
                              "frac": loop_gbs / peak,
                              "note": "fused-kernel model bytes x cell-updates / whole timed region"},
            "unet_inference": {"bound": "tensor", "flops_per_launch_set": fwd_flops, "ms": fwd_ms,
                               "achieved_tflops": fwd_flops / (fwd_ms * 1e-3) / 1e12,
                               "peak_tflops": bf16_peak, "frac": fwd_flops / (fwd_ms * 1e-3) / 1e12 / bf16_peak},
            "e2e": {"value": n_cases * n_e2e * world / e2e_el, "unit": "steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": n_e2e,
                    "sample": f"the first {n_e2e} of the {args.steps} timed steps, replayed from the same state",
                    "same_iterations_as_timed": bool((it_e2e == iters_ws[:, :n_e2e]).all())},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        if cpu is not None:
            line["cpu_baseline"] = {"value": cpu["steps_per_s"], "unit": "steps/s", "cores": cpu["cores"],
                                    "kind": "port",
                                    "sample": cpu["sample"] + f" (plain start's counts of the first {m} steps)"}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _oracle_items(args):
    """The workload's cases built with the oracle's mesh and noise generators (this package's
    Python case builders, no call into its library)."""
    import __graft_entry__ as entry
    from oracle import oracle as orc
    pkg = entry.load_package()
    pkg.configs.use_backend(orc)
    try:
        items, kind = build_workload(pkg, args.workload, "exact", max_iters=args.max_iters, cases=args.cases)
    finally:
        pkg.configs.use_backend(None)
    return items, kind


def reference_picks(n: int, ref_cases: int) -> list:
    """The case ids the reference arm converges on the CPU: ref_cases of the n, spread evenly."""
    ns = max(1, min(ref_cases, n))
    return sorted({int(round(q * (n - 1) / max(1, ns - 1))) for q in range(ns)}) if ns > 1 else [0]


def run_reference(args):
    """The reference's CPU implementation of the loop on the host cores: the oracle, a C++
    restatement of OpenMp_Multicore/main.f90:116-186 and equations.f90 (the Fortran sources
    cannot be compiled here), in the reference's operation order with OpenMP over all host
    threads.  For `--ref-cases` cases of the workload (spread over its case ids) it runs the W
    warm-up steps from rest and then times the K steps of the window, every step converged with
    the reference's start; value = converged case-steps / seconds."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import numpy as np
    from oracle import oracle as orc
    items, kind = _oracle_items(args)
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    n = len(items)
    picks = reference_picks(n, args.ref_cases)
    n_steps = max(1, min(args.steps, args.sample_steps))
    t_all = time.perf_counter()
    secs = 0.0
    iters = {}
    for c in picks:
        prm, mesh, st, itc = items[c]
        o = orc.OracleCase(prm, mesh)
        s = {k: np.asfortranarray(v.copy()) for k, v in st.items()}
        if args.warmup:
            itc, _, _ = o.run(s, args.warmup, itc)
        t0 = time.perf_counter()
        itc, it, _ = o.run(s, n_steps, itc)
        secs += time.perf_counter() - t0
        iters[str(c)] = [int(v) for v in it]
    wall = time.perf_counter() - t_all
    value = len(picks) * n_steps / secs
    line = {
        "impl": "reference",
        "metric": "converged physical steps/s at pseudo-time residual 1e-6",
        "value": value,
        "unit": "steps/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": secs / n_steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded channel cases; no public dataset)",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload], "cases": n,
                   "sampled_cases": picks, "timed_steps": f"the first {n_steps} of the {args.steps} timed steps",
                   "pseudo_iterations_per_step": iters,
                   "start": "the reference's (plain) start in every step, warm-up included"},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads, "kind": "port",
                         "sample": f"cases {picks} of the {n}: {args.warmup} warm-up steps from rest, then the "
                                   f"first {n_steps} of the {args.steps} timed steps, converged, one case at a "
                                   f"time on all {threads} host threads"},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--workload", default="ws-153", choices=sorted(WORKLOADS))
    ap.add_argument("--weights", default=os.path.join(ROOT, "solver-cfd_b200", "unet", "weights", "ws_153.npz"),
                    help="trained warm-start network (ws-* workloads)")
    ap.add_argument("--arith", default="fast", choices=["exact", "fast"])
    ap.add_argument("--engine", default="tile", choices=sorted(ENGINES))
    ap.add_argument("--retune", action="store_true", help="ignore the autotuner cache (cluster engine)")
    ap.add_argument("--launch-shape", default=None,
                    help="cluster engine: threads,ctas_per_sm,nodes_per_cta (skip the autotuner)")
    ap.add_argument("--stage", type=int, default=1, choices=[0, 1],
                    help="cluster engine: stage stencil arrays in shared memory (1) or read them from L1/L2 (0)")
    ap.add_argument("--sample-steps", type=int, default=2,
                    help="ws-* workloads: the first steps of the timed window that the e2e pass replays, the "
                         "plain GPU path times and the reference arm converges on the CPU")
    ap.add_argument("--plain-steps", type=int, default=None,
                    help="ws-* workloads: steps of the window on which the plain GPU path is timed "
                         "(default: --sample-steps)")
    ap.add_argument("--extrap-order", type=int, default=1, choices=[1, 2],
                    help="warm-start workload: linear (1) or quadratic (2) extrapolated candidate")
    ap.add_argument("--warm-eps", type=float, default=None,
                    help="warm-start workload: residual tolerance of the warm-started cases of each step "
                         "(default: every case keeps its own, 1e-6)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ref-cases", type=int, default=1,
                    help="reference arm: cases of the workload run on the CPU (spread over the case ids)")
    ap.add_argument("--cases", type=int, default=None,
                    help="ws-* workloads: number of cases (default: the configuration's 64)")
    ap.add_argument("--max-iters", type=int, default=None,
                    help="cap the pseudo-iterations of every physical step (profiling runs; the steps "
                         "are then not converged)")
    args = ap.parse_args()
    if args.warmup < 0 or args.steps < 1:
        raise SystemExit("bad --steps/--warmup")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_product(args)


if __name__ == "__main__":
    main()
