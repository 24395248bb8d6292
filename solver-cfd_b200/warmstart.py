"""Learned warm start of the pseudo-time loop (no counterpart in the reference).

Between physical steps n-1 -> n -> n+1 the reference starts each pseudo-time loop from the
stale pseudo-iterate of the previous step (main.f90:145-149 are skipped on exit).  Here the
start is predicted instead: with ``inc`` the increment over the last step and ``s`` its RMS
over the case (per field),

    start = fields + inc + s * scale * UNet(fields, porous mask, inc / s)

so the network predicts how the increment changes from one step to the next, relative to the
increment's size (a correction of the linear extrapolation ``fields + inc``; its
zero-initialised head makes an untrained network exactly that extrapolation).
``acs_batch_set_start`` evaluates the initial residual of the plain, the extrapolated and the
learned start and commits the smallest, and the pseudo-time loop then iterates to the same
tolerance, so the solver judges every result.

Data flow per physical step, all on the device and on one stream:
``acs_batch_ws_features`` (fields -> FP32 canvas) -> ``unet_normalize`` (-> BF16 network input)
-> U-Net forward (tcgen05 GEMMs) -> ``acs_batch_set_start`` -> ``acs_batch_run`` (one step).
Training snapshots come from the same loop: ``acs_batch_ws_target`` writes the change of the
increment over the step just run.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from . import OPT_EXTRAP_ORDER, POLICY_BEST, START_PLAIN, WS_IN, WS_OUT, Batch
from .unet import UNet, kernels as unet_kernels

N_FIELDS = 5
FIELD_NAMES = ("u", "v", "p", "T", "C")


def canvas_for(nx: int, ny: int, multiple: int = 8):
    """Smallest canvas (H, W) holding (ny+1) x (nx+1) nodes with sides divisible by `multiple`."""
    up = lambda v: (v + multiple - 1) // multiple * multiple
    return up(ny + 1), up(nx + 1)


def valid_nodes(nx: int, ny: int) -> int:
    """Nodes of the five fields on one case: um (nx+1) ny, vm nx (ny+1), p, T, C nx ny."""
    return (nx + 1) * ny + nx * (ny + 1) + 3 * nx * ny


class Normalizer:
    """Per-channel input shift/scale and output scale (device float vectors)."""

    def __init__(self, in_shift, in_mul, out_scale, device="cuda", inc_weight=None, smooth=0):
        import torch
        self.smooth = int(smooth)   # 3 x 3 box passes over the network output before it is used
        self.in_shift = torch.tensor(np.asarray(in_shift, np.float32), device=device)
        self.in_mul = torch.tensor(np.asarray(in_mul, np.float32), device=device)
        osc = np.ones(WS_OUT, np.float32)
        osc[:N_FIELDS] = np.asarray(out_scale, np.float32)[:N_FIELDS]
        self.out_mul = torch.tensor((1.0 / osc).astype(np.float32), device=device)
        # acs_batch_set_start's scale vector: correction scales, then increment weights
        inc_w = np.ones(WS_OUT, np.float32) if inc_weight is None else np.asarray(inc_weight, np.float32)
        self.out_scale = torch.tensor(np.concatenate([osc, inc_w]), device=device)
        self.zero_out = torch.zeros(WS_OUT, dtype=torch.float32, device=device)

    @staticmethod
    def identity(device="cuda"):
        return Normalizer(np.zeros(WS_IN), np.ones(WS_IN), np.ones(N_FIELDS), device)

    @staticmethod
    def from_samples(X: np.ndarray, T: np.ndarray, Wt: np.ndarray, device="cuda"):
        """X [..., 11], T/Wt [..., 8] host samples; statistics over the nodes that exist."""
        m = Wt[..., 0] > 0
        shift = np.zeros(WS_IN)
        mul = np.ones(WS_IN)
        for c in range(WS_IN):
            if c == 5:  # porous indicator stays 0/1
                continue
            v = X[..., c][m].astype(np.float64)
            sd = v.std()
            shift[c] = v.mean()
            mul[c] = 1.0 / sd if sd > 0 else 1.0
        osc = np.ones(N_FIELDS)
        for c in range(N_FIELDS):
            mc = Wt[..., c] > 0
            r = math.sqrt(float(np.mean(T[..., c][mc].astype(np.float64) ** 2))) if mc.any() else 0.0
            osc[c] = r if r > 0 else 1.0
        return Normalizer(shift, mul, osc, device)

    def to_dict(self):
        return {"in_shift": self.in_shift.cpu().numpy(), "in_mul": self.in_mul.cpu().numpy(),
                "out_scale": self.out_scale.cpu().numpy()[:N_FIELDS],
                "inc_weight": self.out_scale.cpu().numpy()[WS_OUT:], "smooth": self.smooth}


START_NAMES = ("plain", "extrap", "learned")
STATUS_NAMES = ("running", "done", "failed")


class StepLog:
    """Per-step record of every case, one JSON object per line: the physical step, the case, its
    pseudo-iterations, the loop's last error (max of the dtau-scaled u, v and p residuals, the
    `error` of main.f90:139), the case status, and with a warm start the start that was kept and
    the initial residual of each candidate (null where a candidate was not built)."""

    def __init__(self, path_or_file, label: str | None = None):
        self._own = isinstance(path_or_file, (str, os.PathLike))
        self.f = open(path_or_file, "a") if self._own else path_or_file
        self.label = label

    @staticmethod
    def records(step, iters, err, status=None, chosen=None, res0=None, label=None) -> list:
        iters = np.asarray(iters).reshape(-1)
        err = np.asarray(err, np.float64).reshape(-1)
        out = []
        for c in range(iters.size):
            r = {"step": int(step), "case": c, "pseudo_iterations": int(iters[c]), "error": float(err[c])}
            if label is not None:
                r["run"] = label
            if status is not None:
                r["status"] = STATUS_NAMES[int(status[c])]
            if chosen is not None:
                r["start"] = START_NAMES[int(chosen[c])]
            if res0 is not None:
                r["initial_residual"] = {n: (None if not math.isfinite(v) else float(v))
                                         for n, v in zip(START_NAMES, np.asarray(res0, np.float64)[c])}
            out.append(r)
        return out

    def write(self, step, iters, err, status=None, chosen=None, res0=None):
        for r in self.records(step, iters, err, status, chosen, res0, self.label):
            self.f.write(json.dumps(r) + "\n")
        self.f.flush()

    def close(self):
        if self._own:
            self.f.close()


class WarmStart:
    """Warm start of a Batch of cases drawn on one H x W canvas."""

    def __init__(self, batch: Batch, H: int, W: int, net: UNet | None = None, norm: Normalizer | None = None,
                 extrap_order: int = 1):
        """extrap_order 2 makes the extrapolated candidate the quadratic through the last three
        step starts (ACS_OPT_EXTRAP_ORDER)."""
        import torch
        self.torch = torch
        self.b = batch
        self.n = batch.n
        self.H, self.W = H, W
        self.net = net
        self.norm = norm or Normalizer.identity()
        self.log: StepLog | None = None     # set to record every step as JSON lines
        self.steps_done = 0
        batch.set_stream(torch.cuda.current_stream().cuda_stream)
        batch.ws_enable(H, W)
        if extrap_order != 1:
            batch.set_option(OPT_EXTRAP_ORDER, extrap_order)
        f32 = dict(dtype=torch.float32, device="cuda")
        self.X = torch.zeros(self.n * H * W * WS_IN, **f32)
        self.T = torch.zeros(self.n * H * W * WS_OUT, **f32)
        self.Wt = torch.zeros(self.n * H * W * WS_OUT, **f32)
        self.inc_scale = torch.zeros(self.n * WS_OUT, **f32)

    def features(self):
        self.b.ws_features(self.X.data_ptr(), self.inc_scale.data_ptr())
        return self.X

    def target(self):
        self.b.ws_target(self.T.data_ptr(), self.Wt.data_ptr())
        return self.T, self.Wt

    def predict(self):
        """Network output (FP32 [n*H*W*8], normalised increment correction) for the last
        features() call."""
        net = self.net
        xin = net.input_buffer(self.n, self.H, self.W)
        code = unet_kernels().unet_normalize(self.X.data_ptr(), self.n * self.H * self.W, WS_IN,
                                             self.norm.in_shift.data_ptr(), self.norm.in_mul.data_ptr(),
                                             xin.data_ptr(), None, self.torch.cuda.current_stream().cuda_stream)
        if code:
            raise RuntimeError(f"unet_normalize failed with code {code}")
        y = net.forward(self.n, self.H, self.W)
        return self.smoothed(y)

    def smoothed(self, y):
        """`norm.smooth` passes of the 3 x 3 box mean over the network output."""
        if self.norm.smooth <= 0:
            return y
        if getattr(self, "_sm", None) is None or self._sm[0].numel() != y.numel():
            self._sm = (self.torch.empty_like(y), self.torch.empty_like(y))
        K = unet_kernels()
        st = self.torch.cuda.current_stream().cuda_stream
        src = y
        for k in range(self.norm.smooth):
            dst = self._sm[k % 2]
            code = K.unet_smooth3(src.data_ptr(), self.n, self.H, self.W, WS_OUT, dst.data_ptr(), st)
            if code:
                raise RuntimeError(f"unet_smooth3 failed with code {code}")
            src = dst
        return src

    def step(self, itc, mode: str = "learned", warm_eps: float | None = None):
        """One physical step of every case.  mode: "plain" (the reference's start), "extrap"
        (best of plain and extrapolated) or "learned" (best of plain, extrapolated and learned).
        warm_eps: residual tolerance for the cases whose chosen start is not the plain one (the
        others keep their params' eps); None keeps every case's own tolerance.
        Returns (itc, iters[n], chosen[n], res0[n,3])."""
        chosen = np.zeros(self.n, np.int32)
        res0 = np.full((self.n, 3), np.nan)
        if mode != "plain":
            self.features()
            if mode == "learned" and self.net is not None:
                y = self.predict()
                chosen, res0 = self.b.set_start(y.data_ptr(), WS_OUT, self.norm.out_scale.data_ptr(), POLICY_BEST)
            else:
                chosen, res0 = self.b.set_start(None, WS_OUT, None, POLICY_BEST)
        if warm_eps is not None:
            for c in range(self.n):
                self.b.set_tolerance(c, warm_eps if chosen[c] != START_PLAIN else self.b.params[c].eps)
        itc, iters, err, st = self.b.run(1, itc)
        if self.log is not None:
            self.log.write(self.steps_done, iters[:, 0], err[:, 0], st,
                           None if mode == "plain" else chosen, None if mode == "plain" else res0)
        self.steps_done += 1
        return itc, iters[:, 0], chosen, res0


# ---------------------------------------------------------------------------------------------
# snapshots, training, evaluation
# ---------------------------------------------------------------------------------------------
def generate(batch: Batch, H: int, W: int, n_steps: int, itc, skip: int = 2, mode: str = "extrap",
             net=None, norm=None, log=None):
    """Run n_steps physical steps with the warm start and collect one snapshot per case and
    step from step `skip` on: (X [H,W,11], T [H,W,8], Wt [H,W,8]) stacked into device tensors
    of shape [count, H*W*ch].  Returns (X, T, Wt, iterations [n, n_steps])."""
    torch = __import__("torch")
    ws = WarmStart(batch, H, W, net, norm)
    n = batch.n
    Xs, Ts, Ws = [], [], []
    iters_all = np.zeros((n, n_steps), np.int64)
    itc = np.broadcast_to(np.asarray(itc, np.int32), (n,)).copy()
    for s in range(n_steps):
        ws.features()
        Xcur = ws.X.clone() if s >= skip else None
        if mode == "learned" and net is not None:
            y = ws.predict()
            ws.b.set_start(y.data_ptr(), WS_OUT, ws.norm.out_scale.data_ptr(), POLICY_BEST)
        elif mode == "extrap":
            ws.b.set_start(None, WS_OUT, None, POLICY_BEST)
        itc, iters, err, st = batch.run(1, itc)
        iters_all[:, s] = iters[:, 0]
        if s >= skip:
            T, Wt = ws.target()
            Xs.append(Xcur.view(n, -1))
            Ts.append(T.clone().view(n, -1))
            Ws.append(Wt.clone().view(n, -1))
        if log:
            log(f"step {s}: iterations min {iters[:, 0].min()} mean {iters[:, 0].mean():.0f} max {iters[:, 0].max()}")
    X = torch.cat(Xs) if Xs else None
    T = torch.cat(Ts) if Ts else None
    Wt = torch.cat(Ws) if Ws else None
    return X, T, Wt, iters_all


def train(net: UNet, X, T, Wt, H, W, norm: Normalizer, epochs=10, batch=16, lr=1e-3, seed=0, log=None,
          lr_final=1e-4, grad_weight=0.0):
    """Minibatch Adam on the snapshots (device tensors from generate()).  The loss is the masked
    MSE, plus grad_weight x the squared x/y differences of the error when grad_weight > 0.
    Returns the per-epoch mean losses."""
    torch = net.torch
    rng = np.random.default_rng(seed)
    K = unet_kernels()
    s = torch.cuda.current_stream().cuda_stream
    N = X.shape[0]
    f32 = dict(dtype=torch.float32, device="cuda")
    tgt = torch.zeros(batch * H * W * WS_OUT, **f32)
    wgt = torch.zeros(batch * H * W * WS_OUT, **f32)
    xin = net.input_buffer(batch, H, W)
    counts = Wt.sum(dim=1).double().cpu().numpy()  # existing nodes per snapshot
    losses = []
    steps_total = epochs * (N // batch)
    k = 0
    for ep in range(epochs):
        perm = rng.permutation(N)
        acc = torch.zeros(1, **f32)
        nb = 0
        for q in range(0, N - batch + 1, batch):
            idx = torch.as_tensor(perm[q:q + batch], device="cuda")
            xb = X.index_select(0, idx).reshape(-1)
            K.unet_normalize(xb.data_ptr(), batch * H * W, WS_IN, norm.in_shift.data_ptr(), norm.in_mul.data_ptr(),
                             xin.data_ptr(), None, s)
            tb = T.index_select(0, idx).reshape(-1)
            K.unet_normalize(tb.data_ptr(), batch * H * W, WS_OUT, norm.zero_out.data_ptr(), norm.out_mul.data_ptr(),
                             None, tgt.data_ptr(), s)
            wgt.copy_(Wt.index_select(0, idx).reshape(-1))
            count = float(counts[perm[q:q + batch]].sum())
            # cosine learning-rate decay from lr to lr_final
            a = 0.5 * (1 + math.cos(math.pi * k / max(1, steps_total)))
            cur = lr_final + (lr - lr_final) * a
            loss = net.train_step(batch, H, W, tgt, wgt, 1.0 / count, cur, lam=grad_weight)
            acc += loss
            nb += 1
            k += 1
        m = float(acc.item()) / max(1, nb)
        losses.append(m)
        if log and (ep % max(1, epochs // 20) == 0 or ep == epochs - 1):
            log(f"epoch {ep}: loss {m:.4e}")
    if net.wait_error():
        raise RuntimeError("a GEMM wait timed out during training")
    return losses


def save(path, net: UNet, norm: Normalizer, H, W, meta=None):
    d = norm.to_dict()
    np.savez_compressed(path, params=net.params(), H=H, W=W, cin=net.cin, cout=net.cout, base=net.base,
                        levels=net.levels, meta=json.dumps(meta or {}), **d)


def load(path, device="cuda"):
    z = np.load(path)
    net = UNet(int(z["cin"]), int(z["cout"]), int(z["base"]), int(z["levels"]), device=device)
    net.set_params(z["params"])
    norm = Normalizer(z["in_shift"], z["in_mul"], z["out_scale"], device,
                      z["inc_weight"] if "inc_weight" in z.files else None,
                      int(z["smooth"]) if "smooth" in z.files else 0)
    return net, norm, int(z["H"]), int(z["W"]), json.loads(str(z["meta"]))


def evaluate(make_batch, H, W, n_steps, itc0, net=None, norm=None, modes=("plain", "extrap", "learned"),
             log=None, step_log: StepLog | None = None, extrap_order: int = 1):
    """Run fresh copies of the same cases for n_steps in each mode.  Returns per mode the
    iterations [n, n_steps], the seconds per step (device time, CUDA events around the whole
    step: features, network, start selection and the pseudo-time loop), the fraction of cases
    per step that started plain / extrapolated / learned ("kept", [n_steps, 3]) and the final
    fields.  With step_log, every case's step is also recorded as a JSON line labelled by mode."""
    torch = __import__("torch")
    out = {}
    for mode in modes:
        b = make_batch()
        ws = WarmStart(b, H, W, net if mode == "learned" else None, norm, extrap_order=extrap_order)
        if step_log is not None:
            step_log.label = mode
            ws.log = step_log
        itc = np.broadcast_to(np.asarray(itc0, np.int32), (b.n,)).copy()
        iters = np.zeros((b.n, n_steps), np.int64)
        kept = []
        times = []
        for s in range(n_steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            itc, it, chosen, res0 = ws.step(itc, mode)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
            iters[:, s] = it
            kept.append(np.bincount(chosen, minlength=3) / b.n)
            if log:
                log(f"{mode} step {s}: iterations mean {it.mean():.0f}, starts plain/extrap/learned {kept[-1]}, "
                    f"{times[-1]:.3f} s")
        fields = [b.get_state(c, ("um", "vm", "p", "pn", "T", "C")) for c in range(b.n)]
        out[mode] = {"iters": iters, "sec_per_step": np.array(times), "kept": np.array(kept), "fields": fields}
        b.close()
    return out


def field_error(a: dict, b: dict):
    """Relative max-norm difference per field: max|a-b| / max|b| (vm's dead corner excluded)."""
    res = {}
    for k in ("um", "vm", "pn", "T", "C"):
        x, y = a[k].copy(), b[k].copy()
        if k == "vm":
            x[-1, -1] = y[-1, -1] = 0.0
        den = float(np.abs(y).max())
        res[k] = float(np.abs(x - y).max()) / (den if den > 0 else 1.0)
    return res
