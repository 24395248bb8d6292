"""Train and evaluate the learned warm start on n x n cases (default 153 x 153).

Cases follow the batched configuration's parameter distribution (Re ~ U[50,500], Darcy number
log-uniform in [1e-5, 1e-2], porosity ~ U[0.3,0.9], Richardson number ~ U[0,2], a porous block
of 30 % area at a uniform interior position; QUICK, buoyancy, scalars T and C, FP64 solver)
with the grid fixed at n x n.  Steps:

1. snapshots: `--train-cases` seeded cases (seed `--seed`) run `--gen-steps` physical steps
   with the extrapolated start; every step from the third on gives one snapshot per case;
2. training: Adam on the library's tcgen05 kernels, `--epochs` passes in minibatches of
   `--batch`;
3. evaluation: `--eval-cases` held-out cases (seed `--seed` + 1) run `--eval-steps` physical
   steps three times -- plain start (the reference's), extrapolated, learned -- to the same
   residual tolerance; pseudo-iterations per step, device seconds per step and the final
   fields' relative max-norm difference to the plain run are reported.

Writes the weights (`--out`, .npz) and a JSON report (`--report`).  `--eval-only` skips steps
1 and 2 and compares the starts that need no network; `--step-log` records every case's step.

    python solver-cfd_b200/train_warmstart.py --n 153 --train-cases 16 --gen-steps 30 \\
        --epochs 100 --eval-cases 4 --eval-steps 10
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _pkg():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import __graft_entry__ as entry
    return entry.load_package()


def make_cases(pkg, n, count, seed, arith):
    cases, _ = pkg.configs.cfg_batch(count, seed=seed, sizes=(n,), arith=arith)
    return cases


def make_batch(pkg, cases, options=None, launch_shape=None):
    b = pkg.Batch([c[0] for c in cases], [c[1] for c in cases])
    for k, c in enumerate(cases):
        b.set_state(k, c[2])
    for opt, val in (options or {}).items():
        b.set_option(opt, val)
    if launch_shape is not None:
        from importlib import import_module
        import_module(pkg.__name__ + ".autotune").apply(b, pkg, launch_shape)
    return b


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--n", type=int, default=153)
    ap.add_argument("--train-cases", type=int, default=16)
    ap.add_argument("--gen-steps", type=int, default=30)
    ap.add_argument("--epochs", type=int, default=100)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--grad-weight", type=float, default=0.0,
                    help="weight of the squared x/y differences of the error in the loss")
    ap.add_argument("--smooth", type=int, default=0, help="3x3 box passes over the network output")
    ap.add_argument("--eval-cases", type=int, default=4)
    ap.add_argument("--eval-steps", type=int, default=10)
    ap.add_argument("--seed", type=int, default=100)
    ap.add_argument("--arith", choices=("fast", "exact"), default="fast")
    ap.add_argument("--modes", default="plain,extrap,learned")
    ap.add_argument("--out", default=os.path.join(HERE, "unet", "weights", "ws_153.npz"))
    ap.add_argument("--report", default=None)
    ap.add_argument("--step-log", default=None,
                    help="append one JSON line per case and evaluation step (iterations, error, start kept)")
    ap.add_argument("--load", default=None, help="skip generation and training; evaluate these weights")
    ap.add_argument("--eval-only", action="store_true",
                    help="no network: evaluate the plain and extrapolated starts only (--modes plain,extrap)")
    ap.add_argument("--extrap-order", type=int, default=1, choices=[1, 2],
                    help="evaluation: linear (1) or quadratic (2) extrapolated candidate")
    ap.add_argument("--autotune", action="store_true",
                    help="evaluate with the autotuner's launch shape for the held-out cases")
    a = ap.parse_args(argv)

    import torch
    pkg = _pkg()
    from importlib import import_module
    ws = import_module(pkg.__name__ + ".warmstart")
    unet = import_module(pkg.__name__ + ".unet")
    arith = pkg.ARITH_FAST if a.arith == "fast" else pkg.ARITH_EXACT
    H, W = ws.canvas_for(a.n, a.n)
    t0 = time.time()
    log = lambda m: print(f"[{time.time() - t0:8.1f}s] {m}", flush=True)
    report = {"n": a.n, "canvas": [H, W], "args": vars(a)}

    if a.eval_only:
        if "learned" in a.modes.split(","):
            raise SystemExit("--eval-only evaluates the starts that need no network: --modes plain,extrap")
        net = norm = None
    elif a.load:
        net, norm, H2, W2, meta = ws.load(a.load)
        assert (H2, W2) == (H, W)
        if a.smooth:
            norm.smooth = a.smooth
        report["trained"] = meta
    else:
        cases = make_cases(pkg, a.n, a.train_cases, a.seed, arith)
        b = make_batch(pkg, cases)
        X, T, Wt, it_gen = ws.generate(b, H, W, a.gen_steps, 1, skip=2, log=log)
        b.close()
        del cases
        log(f"snapshots: {X.shape[0]} ({X.numel() * 4 / 2**30:.2f} GiB of features)")
        take = min(X.shape[0], 64)
        norm = ws.Normalizer.from_samples(X[:take].cpu().numpy().reshape(-1, H, W, 11),
                                          T[:take].cpu().numpy().reshape(-1, H, W, 8),
                                          Wt[:take].cpu().numpy().reshape(-1, H, W, 8))
        norm.smooth = a.smooth
        net = unet.UNet(11, 5, 32, 4, seed=a.seed)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        losses = ws.train(net, X, T, Wt, H, W, norm, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed,
                          log=log, grad_weight=a.grad_weight)
        e1.record()
        torch.cuda.synchronize()
        train_s = e0.elapsed_time(e1) / 1e3
        n_steps_train = a.epochs * (X.shape[0] // a.batch)
        flops = 3 * unet.conv_flops(H, W) * a.batch * n_steps_train
        log(f"training: {a.epochs} epochs, {train_s:.1f} s, losses {[round(x, 4) for x in losses[::max(1, a.epochs // 10)]]}"
            f", {flops / train_s / 1e12:.1f} TFLOP/s (convolution FLOPs x3)")
        meta = {"snapshots": int(X.shape[0]), "gen_iterations_mean_per_step": it_gen.mean(axis=0).round(1).tolist(),
                "losses": [float(x) for x in losses], "train_seconds": train_s,
                "train_tflops": flops / train_s / 1e12}
        report["trained"] = meta
        del X, T, Wt
        torch.cuda.empty_cache()
        os.makedirs(os.path.dirname(a.out), exist_ok=True)
        ws.save(a.out, net, norm, H, W, meta)
        log(f"weights written to {a.out}")

    held = make_cases(pkg, a.n, a.eval_cases, a.seed + 1, arith)
    modes = tuple(a.modes.split(","))
    shape = None
    if a.autotune:
        shape = import_module(pkg.__name__ + ".autotune").tune(pkg, held)
        report["launch_shape"] = shape
        log(f"launch shape {shape}")
    step_log = ws.StepLog(a.step_log) if a.step_log else None
    out = ws.evaluate(lambda: make_batch(pkg, held, launch_shape=shape), H, W, a.eval_steps, 1, net, norm,
                      modes=modes, log=log, step_log=step_log, extrap_order=a.extrap_order)
    if step_log is not None:
        step_log.close()
    res = {}
    for m in modes:
        it = out[m]["iters"]
        res[m] = {"iterations_per_step": it.mean(axis=0).round(1).tolist(),
                  "sec_per_step": out[m]["sec_per_step"].round(4).tolist(),
                  "starts_plain_extrap_learned": np.asarray(out[m]["kept"]).round(3).tolist()}
    if "plain" in out:
        for m in modes:
            if m == "plain":
                continue
            errs = [ws.field_error(out[m]["fields"][c], out["plain"]["fields"][c]) for c in range(len(held))]
            res[m]["max_rel_error_vs_plain"] = {k: max(e[k] for e in errs) for k in errs[0]}
    report["eval"] = res
    s0 = 3
    summary = {}
    for m in modes:
        it = out[m]["iters"][:, s0:]
        sec = out[m]["sec_per_step"][s0:]
        summary[m] = {"iterations_per_step": float(it.mean()), "case_steps_per_s": float(len(held) * len(sec) / sec.sum())}
    report["summary_from_step_3"] = summary
    log(json.dumps(summary))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)
    return report


if __name__ == "__main__":
    main()
