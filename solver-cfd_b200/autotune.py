"""Autotuner of the persistent cluster engine.

The engine's launch shape is set per batch by four knobs (include/acs.h, ACS_OPT_*):
threads per CTA (256 or 512), resident CTAs per SM (1 or 2, 256 threads only), the target
number of nodes per CTA, which fixes how many CTAs (1..16, one cluster) each case is split into,
and whether each phase stages its stencil arrays in shared memory first.  The graph engine
(per-stage kernels spread over the whole GPU, the better choice for a single large case) is
timed as one more candidate.
Besides powers of two, the candidates include the splits that make one wave of clusters fill the
SMs (n_cases x K ~ SMs x CTAs per SM).  The best choice depends on the case sizes and on how many
cases share the GPU, so it is measured:
every candidate runs one physical step capped at a few hundred pseudo-iterations on a copy of the
workload, and the candidate with the most cell-updates per second wins.  Results are cached in
JSON (``tuning/`` beside this file) keyed by the device name and a signature of the workload.
"""
from __future__ import annotations

import hashlib
import json
import os
import time
from dataclasses import replace

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE_DIR = os.path.join(HERE, "tuning")

SHAPES = [(512, 1), (256, 2), (256, 1)]       # (threads, CTAs per SM)
NODES = [256, 512, 1024, 2048, 4096, 8192]


def signature(items) -> str:
    """Workload key: the multiset of (imax, jmax, scheme, scalars, arith) of its cases."""
    keys = sorted((p.imax, p.jmax, p.scheme, p.solve_scalars, p.arith) for p, *_ in items)
    h = hashlib.sha1(json.dumps(keys).encode()).hexdigest()[:12]
    return f"n{len(items)}-{h}"


def _device_name(pkg) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0).replace(" ", "_")
    except Exception:  # noqa: BLE001 - a name is only used as a cache key
        return "cuda"


def apply(batch, pkg, cfg: dict) -> None:
    batch.set_option(pkg.OPT_THREADS, cfg["threads"])
    batch.set_option(pkg.OPT_CTAS_PER_SM, cfg["ctas_per_sm"])
    batch.set_option(pkg.OPT_NODES_PER_CTA, cfg["nodes_per_cta"])
    batch.set_option(pkg.OPT_L1_LOADS, 1)
    batch.set_option(pkg.OPT_STAGED, cfg.get("staged", 1))
    batch.set_option(pkg.OPT_ENGINE, cfg.get("engine", 0))


def _sm_count() -> int:
    try:
        import torch
        return int(torch.cuda.get_device_properties(0).multi_processor_count)
    except Exception:  # noqa: BLE001 - without a device only the fixed candidates are used
        return 0


def fill_candidates(items, sms: int, per_sm: int):
    """Nodes per CTA that split every case into K CTAs with n_cases * K close to the resident
    CTA slots (sms * per_sm), so one wave of clusters covers the GPU (K <= 16)."""
    if sms <= 0:
        return []
    n = len(items)
    biggest = max((p.imax + 1) * (p.jmax + 1) for p, *_ in items)
    out = set()
    k_fill = max(1, min(16, (sms * per_sm) // max(n, 1)))
    for K in (k_fill, k_fill - 1, min(16, k_fill + 1)):
        if K >= 1:
            out.add((biggest + K - 1) // K)
    return sorted(out)


def tune(pkg, items, iters: int = 200, use_cache: bool = True, verbose: bool = False) -> dict:
    """Return the best launch configuration for this workload (FAST engine)."""
    os.makedirs(CACHE_DIR, exist_ok=True)
    key = f"{_device_name(pkg)}-{signature(items)}"
    path = os.path.join(CACHE_DIR, key + ".json")
    if use_cache and os.path.exists(path):
        try:
            with open(path) as f:
                return json.load(f)["best"]
        except (OSError, ValueError, KeyError):
            pass  # unreadable cache entry: tune again
    capped = [(replace(p, itc_max=iters, arith=pkg.ARITH_FAST), m, s, itc) for p, m, s, itc in items]
    batch = pkg.Batch([x[0] for x in capped], [x[1] for x in capped])
    cells = np.array([p.imax * p.jmax for p, *_ in capped], float)
    table = []
    try:
        sms = _sm_count()
        cands = []
        for threads, per_sm in SHAPES:
            for nodes in sorted(set(NODES) | set(fill_candidates(capped, sms, per_sm))):
                for staged in ((0, 1) if per_sm == 1 else (0,)):
                    cands.append({"threads": threads, "ctas_per_sm": per_sm, "nodes_per_cta": nodes,
                                  "staged": staged})
        # the graph engine (per-stage kernels over the whole GPU): wins for single large cases
        cands.append({"threads": 512, "ctas_per_sm": 1, "nodes_per_cta": 4096, "staged": 0, "engine": 1})
        for cfg in cands:
            apply(batch, pkg, cfg)
            for c, x in enumerate(capped):
                batch.set_state(c, x[2])
            itc = np.array([x[3] for x in capped], np.int32)
            t0 = time.perf_counter()
            _, it, _, _ = batch.run(1, itc)
            dt = time.perf_counter() - t0
            rate = float((it[:, 0] * cells).sum()) / dt
            table.append(dict(cfg, cell_updates_per_s=rate, seconds=dt))
            if verbose:
                print("autotune", cfg, f"{rate / 1e9:.3f} Gcell-updates/s", flush=True)
    finally:
        batch.close()
    best = max(table, key=lambda r: r["cell_updates_per_s"])
    best = {k: best[k] for k in ("threads", "ctas_per_sm", "nodes_per_cta", "staged")} | {"engine": best.get("engine", 0)}
    # ranks of a multi-GPU run may tune the same workload at once: write a private file, then
    # rename it into place (atomic), so a reader never sees a partial entry
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump({"key": key, "iterations_per_candidate": iters, "best": best, "table": table}, f, indent=1)
    os.replace(tmp, path)
    return best
