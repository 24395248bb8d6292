"""BF16 U-Net of the learned warm start, run on the library's own kernels (include/unet.h).

Every product is the tcgen05 GEMM of ``unet_gemm``: a 3x3 "same" convolution is
``col(X) @ W^T`` with ``col`` built by ``unet_im2col`` (NHWC activations, K index
``(ky*3+kx)*Cin + c`` padded to a multiple of 8); in the forward pass, layers whose Cin is a
multiple of 8 use ``unet_conv3x3``, the same GEMM gathering ``col`` on the fly.  Its gradients are ``dW^T = col(X)^T dZ``
(split-K GEMM with FP32 atomics) and ``dX = col2im(dZ W)``.  Pooling (2x2 average), nearest
upsampling, skip concatenation, ReLU backward, bias gradients, the masked MSE and Adam are the
kernels of ``unet_ops.cu``.  torch only allocates device memory and orders work on its current
stream; it performs none of the network's arithmetic.

Architecture (4 levels, ``base`` channels at the top level, two 3x3 conv + ReLU per block):
encoder ``cin -> b -> 2b -> 4b``, bottleneck ``8b``, decoder with skip concatenations, and a
3x3 head to ``cout`` channels (padded to 8) without activation.  The head starts at zero, so an
untrained network outputs 0.  Weights are FP32 master copies with BF16 copies for the GEMMs;
activations are BF16 with FP32 accumulation; gradients are FP32.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

V = C.c_void_p
F = C.c_float
LL = C.c_longlong
I = C.c_int

_SIG = {
    "unet_gemm": [V, I, V, I, I, I, I, I, V, V, I, V, I, I, V, V],
    "unet_conv3x3": [V, I, I, I, I, V, I, I, I, V, V, I, V, I, V, V],
    "unet_im2col": [V, I, I, I, I, I, V, V],
    "unet_col2im": [V, I, I, I, I, I, V, V],
    "unet_transpose_bf16": [V, I, I, I, V, I, V],
    "unet_pool_fwd": [V, I, I, I, I, V, V],
    "unet_pool_bwd": [V, I, I, I, I, V, I, V],
    "unet_up_fwd": [V, I, I, I, I, V, I, I, V],
    "unet_up_bwd": [V, I, I, I, I, I, I, V, V],
    "unet_copy_channels": [V, LL, I, V, I, I, V],
    "unet_take_channels": [V, I, I, LL, I, V, I, V],
    "unet_act_bwd": [V, V, LL, I, V, V],
    "unet_bias_grad": [V, LL, I, V, V],
    "unet_f32_to_bf16": [V, LL, V, V],
    "unet_mse": [V, V, V, LL, F, V, V, V],
    "unet_mse_grad": [V, V, V, I, I, I, I, F, F, V, V, V],
    "unet_smooth3": [V, I, I, I, I, V, V],
    "unet_normalize": [V, LL, I, V, V, V, V, V],
    "unet_adam": [V, V, V, V, LL, F, F, F, F, I, V, V],
}

OUT_PAD = 8


def kernels():
    """The unet_* entry points of libacs_b200.so with their argument types."""
    from .. import lib
    L = lib()
    if not getattr(L, "_unet_declared", False):
        for name, args in _SIG.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L._unet_declared = True
    return L


def _p(t):
    return None if t is None else t.data_ptr()


def _ok(code, what):
    if code != 0:
        raise RuntimeError(f"{what} failed with code {code}")


class Conv:
    """One 3x3 convolution: weights W^T [kp][cout] and bias [cout] inside the flat buffers."""

    def __init__(self, name, cin, cout, relu, off):
        self.name, self.cin, self.cout, self.relu = name, cin, cout, relu
        self.kp = (9 * cin + 7) // 8 * 8
        self.off_w = off
        self.off_b = off + self.kp * cout
        self.size = self.kp * cout + cout
        self.off_wb = 0  # offset of W [cout][kp] in the BF16 forward copy


def layer_table(cin=11, cout=5, base=32, levels=4):
    c = [base * 2 ** l for l in range(levels)]
    convs = []
    off = 0

    def add(name, a, b, relu=True):
        nonlocal off
        L = Conv(name, a, b, relu, off)
        off += (L.size + 63) // 64 * 64
        convs.append(L)

    prev = cin
    for l in range(levels):
        add(f"enc{l}a", prev, c[l])
        add(f"enc{l}b", c[l], c[l])
        prev = c[l]
    for l in range(levels - 2, -1, -1):
        add(f"dec{l}a", c[l + 1] + c[l], c[l])
        add(f"dec{l}b", c[l], c[l])
    add("head", c[0], OUT_PAD, relu=False)
    return convs, off


def conv_flops(H, W, cin=11, cout=5, base=32, levels=4):
    """Forward FLOPs of one H x W sample: 2 * 9 * Cin * Cout * pixels per convolution (the head
    counted at its 5 real output channels)."""
    convs, _ = layer_table(cin, cout, base, levels)
    total = 0
    for L in convs:
        lvl = int(L.name[3]) if L.name != "head" else 0
        pix = (H >> lvl) * (W >> lvl)
        co = cout if L.name == "head" else L.cout
        total += 2 * 9 * L.cin * co * pix
    return total


class UNet:
    def __init__(self, cin=11, cout=5, base=32, levels=4, seed=0, device="cuda"):
        import torch
        self.torch = torch
        self.cin, self.cout, self.base, self.levels = cin, cout, base, levels
        self.convs, self.n_params = layer_table(cin, cout, base, levels)
        self.by_name = {L.name: L for L in self.convs}
        self.dev = device
        f32 = dict(dtype=torch.float32, device=device)
        self.master = torch.zeros(self.n_params, **f32)
        self.grad = torch.zeros(self.n_params, **f32)
        self.m = torch.zeros(self.n_params, **f32)
        self.v = torch.zeros(self.n_params, **f32)
        self.wt_bf16 = torch.zeros(self.n_params, dtype=torch.bfloat16, device=device)
        off = 0
        for L in self.convs:
            L.off_wb = off
            off += (L.kp * L.cout + 63) // 64 * 64
        self.w_bf16 = torch.zeros(off, dtype=torch.bfloat16, device=device)
        self.t = 0
        self.implicit = True   # forward convolutions with C % 8 == 0 as implicit GEMMs
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        self._ws = {}
        self.init_weights(seed)

    # ---- parameters ------------------------------------------------------------------------
    def init_weights(self, seed):
        """He-normal weights for the ReLU layers, zero biases, zero head."""
        rng = np.random.default_rng(seed)
        host = np.zeros(self.n_params, np.float32)
        for L in self.convs:
            if L.name == "head":
                continue
            std = math.sqrt(2.0 / (9 * L.cin))
            w = np.zeros((L.kp, L.cout), np.float32)
            w[: 9 * L.cin] = rng.standard_normal((9 * L.cin, L.cout)).astype(np.float32) * std
            host[L.off_w: L.off_w + L.kp * L.cout] = w.ravel()
        self.set_params(host)

    def set_params(self, host: np.ndarray):
        self.master.copy_(self.torch.from_numpy(np.ascontiguousarray(host, np.float32)).to(self.dev))
        self.m.zero_()
        self.v.zero_()
        self.t = 0
        self.refresh_bf16()

    def params(self) -> np.ndarray:
        return self.master.cpu().numpy().copy()

    def weight(self, name):
        """(W^T [kp][cout], bias) of one layer as host FP32 arrays."""
        L = self.by_name[name]
        h = self.params()
        return h[L.off_w: L.off_w + L.kp * L.cout].reshape(L.kp, L.cout), h[L.off_b: L.off_b + L.cout]

    def grad_of(self, name):
        L = self.by_name[name]
        h = self.grad.cpu().numpy()
        return h[L.off_w: L.off_w + L.kp * L.cout].reshape(L.kp, L.cout), h[L.off_b: L.off_b + L.cout]

    def refresh_bf16(self):
        K = kernels()
        s = self._stream()
        _ok(K.unet_f32_to_bf16(_p(self.master), self.n_params, _p(self.wt_bf16), s), "f32_to_bf16")
        self._transpose_weights()

    def _transpose_weights(self):
        K = kernels()
        s = self._stream()
        for L in self.convs:
            src = self.wt_bf16.data_ptr() + 2 * L.off_w
            dst = self.w_bf16.data_ptr() + 2 * L.off_wb
            _ok(K.unet_transpose_bf16(src, L.kp, L.cout, L.cout, dst, L.kp, s), "transpose")

    def _stream(self):
        return self.torch.cuda.current_stream().cuda_stream

    # ---- workspace -------------------------------------------------------------------------
    def workspace(self, B, H, W):
        key = (B, H, W)
        if key in self._ws:
            return self._ws[key]
        torch = self.torch
        lv = self.levels
        if H % (1 << (lv - 1)) or W % (1 << (lv - 1)):
            raise ValueError(f"canvas {H}x{W} must be divisible by {1 << (lv - 1)}")
        Ms = [B * (H >> l) * (W >> l) for l in range(lv)]
        if any(m % 8 for m in Ms):
            raise ValueError("pixels per level must be a multiple of 8")
        c = [self.base * 2 ** l for l in range(lv)]
        bf = dict(dtype=torch.bfloat16, device=self.dev)
        f32 = dict(dtype=torch.float32, device=self.dev)
        ws = {"B": B, "H": H, "W": W, "M": Ms, "c": c}
        act = {}
        # activation tensors (BF16) and their gradients (FP32)
        for l in range(lv):
            act[f"a{l}"] = Ms[l] * c[l]
            act[f"E{l}"] = Ms[l] * c[l]
            if l + 1 < lv:
                act[f"P{l}"] = Ms[l + 1] * c[l]
        for l in range(lv - 1):
            act[f"cat{l}"] = Ms[l] * (c[l + 1] + c[l])
            act[f"d{l}"] = Ms[l] * c[l]
            act[f"D{l}"] = Ms[l] * c[l]
        ws["act"] = {k: torch.zeros(n, **bf) for k, n in act.items()}
        ws["grad"] = {k: torch.zeros(n, **f32) for k, n in act.items()}
        ws["x"] = torch.zeros(Ms[0] * self.cin, **bf)
        ws["y"] = torch.zeros(Ms[0] * OUT_PAD, **f32)
        ws["dy"] = torch.zeros(Ms[0] * OUT_PAD, **f32)
        max_col = max(Ms[self._level(L)] * L.kp for L in self.convs)
        max_z = max(Ms[self._level(L)] * L.cout for L in self.convs)
        ws["col"] = torch.zeros(max_col, **bf)
        ws["colT"] = torch.zeros(max_col, **bf)
        ws["dcol"] = torch.zeros(max_col, **f32)
        ws["dz"] = torch.zeros(max_z, **bf)
        ws["dzT"] = torch.zeros(max_z, **bf)
        ws["loss"] = torch.zeros(1, **f32)
        self._ws[key] = ws
        return ws

    @staticmethod
    def _level(L):
        return 0 if L.name == "head" else int(L.name[3])

    # ---- forward ---------------------------------------------------------------------------
    def _conv_fwd(self, ws, L, X, Y, lvl, out_f32=False):
        K = kernels()
        s = self._stream()
        B, H, W = ws["B"], ws["H"] >> lvl, ws["W"] >> lvl
        M = B * H * W
        wb = self.w_bf16.data_ptr() + 2 * L.off_wb
        bias = self.master.data_ptr() + 4 * L.off_b
        if self.implicit and L.cin % 8 == 0 and L.kp == 9 * L.cin:
            # implicit GEMM: the A operand is gathered from X, no col matrix in memory
            if out_f32:
                code = K.unet_conv3x3(_p(X), B, H, W, L.cin, wb, L.kp, L.cout, 3, _p(Y), None, L.cout, bias, 0,
                                      _p(self.err), s)
            else:
                code = K.unet_conv3x3(_p(X), B, H, W, L.cin, wb, L.kp, L.cout, 2, None, _p(Y), L.cout, bias,
                                      1 if L.relu else 0, _p(self.err), s)
            _ok(code, f"conv3x3 {L.name}")
            return
        col = ws["col"]
        _ok(K.unet_im2col(_p(X), B, H, W, L.cin, L.kp, _p(col), s), "im2col")
        if out_f32:
            code = K.unet_gemm(_p(col), L.kp, wb, L.kp, M, L.cout, L.kp, 3, _p(Y), None, L.cout, bias, 0, 1,
                               _p(self.err), s)
        else:
            code = K.unet_gemm(_p(col), L.kp, wb, L.kp, M, L.cout, L.kp, 2, None, _p(Y), L.cout, bias,
                               1 if L.relu else 0, 1, _p(self.err), s)
        _ok(code, f"gemm {L.name}")

    def input_buffer(self, B, H, W):
        """The workspace's BF16 input [B*H*W*cin] (NHWC), for kernels that write it in place."""
        return self.workspace(B, H, W)["x"]

    def forward(self, B, H, W, X_bf16=None):
        """Forward pass of the input buffer (X_bf16, NHWC BF16, is copied into it when given).
        Returns the workspace's FP32 output [B*H*W*8] (channels >= cout stay 0) and remembers
        the activations for backward()."""
        ws = self.workspace(B, H, W)
        if X_bf16 is not None and X_bf16.data_ptr() != ws["x"].data_ptr():
            ws["x"].copy_(X_bf16.reshape(-1))
        self._last = ws
        K = kernels()
        s = self._stream()
        A, c, lv = ws["act"], ws["c"], self.levels
        x = ws["x"]
        for l in range(lv):
            self._conv_fwd(ws, self.by_name[f"enc{l}a"], x, A[f"a{l}"], l)
            self._conv_fwd(ws, self.by_name[f"enc{l}b"], A[f"a{l}"], A[f"E{l}"], l)
            if l + 1 < lv:
                _ok(K.unet_pool_fwd(_p(A[f"E{l}"]), B, H >> l, W >> l, c[l], _p(A[f"P{l}"]), s), "pool")
                x = A[f"P{l}"]
        below = A[f"E{lv - 1}"]
        for l in range(lv - 2, -1, -1):
            cat = A[f"cat{l}"]
            ctot = c[l + 1] + c[l]
            _ok(K.unet_up_fwd(_p(below), B, H >> (l + 1), W >> (l + 1), c[l + 1], _p(cat), ctot, 0, s), "up")
            _ok(K.unet_copy_channels(_p(A[f"E{l}"]), ws["M"][l], c[l], _p(cat), ctot, c[l + 1], s), "copy")
            self._conv_fwd(ws, self.by_name[f"dec{l}a"], cat, A[f"d{l}"], l)
            self._conv_fwd(ws, self.by_name[f"dec{l}b"], A[f"d{l}"], A[f"D{l}"], l)
            below = A[f"D{l}"]
        self._conv_fwd(ws, self.by_name["head"], below, ws["y"], 0, out_f32=True)
        return ws["y"]

    # ---- backward --------------------------------------------------------------------------
    def _conv_bwd(self, ws, L, X, Yact, dY, dX, lvl):
        K = kernels()
        s = self._stream()
        B, H, W = ws["B"], ws["H"] >> lvl, ws["W"] >> lvl
        M = B * H * W
        dz, dzT, col, colT, dcol = ws["dz"], ws["dzT"], ws["col"], ws["colT"], ws["dcol"]
        _ok(K.unet_act_bwd(_p(dY), _p(Yact) if L.relu else None, M * L.cout, 1 if L.relu else 0, _p(dz), s),
            "act_bwd")
        gb = self.grad.data_ptr() + 4 * L.off_b
        _ok(K.unet_bias_grad(_p(dz), M, L.cout, gb, s), "bias_grad")
        _ok(K.unet_transpose_bf16(_p(dz), M, L.cout, L.cout, _p(dzT), M, s), "transpose dz")
        _ok(K.unet_im2col(_p(X), B, H, W, L.cin, L.kp, _p(col), s), "im2col")
        _ok(K.unet_transpose_bf16(_p(col), M, L.kp, L.kp, _p(colT), M, s), "transpose col")
        gw = self.grad.data_ptr() + 4 * L.off_w
        tiles = ((L.kp + 127) // 128) * max(1, (L.cout + 255) // 256)
        ktiles = (M + 63) // 64
        splits = max(1, min(ktiles, (4 * 148 + tiles - 1) // tiles))
        _ok(K.unet_gemm(_p(colT), M, _p(dzT), M, L.kp, L.cout, M, 1, gw, None, L.cout, None, 0, splits,
                        _p(self.err), s), f"gemm dW {L.name}")
        if dX is not None:
            wt = self.wt_bf16.data_ptr() + 2 * L.off_w
            _ok(K.unet_gemm(_p(dz), L.cout, wt, L.cout, M, L.kp, L.cout, 0, _p(dcol), None, L.kp, None, 0, 1,
                            _p(self.err), s), f"gemm dX {L.name}")
            _ok(K.unet_col2im(_p(dcol), B, H, W, L.cin, L.kp, _p(dX), s), "col2im")

    def backward(self, dy=None):
        """Gradients of every parameter (into self.grad, zeroed first) from dLoss/dY (FP32
        [B*H*W*8], default: the workspace buffer written by the loss)."""
        ws = self._last
        K = kernels()
        s = self._stream()
        B, H, W = ws["B"], ws["H"], ws["W"]
        A, G, c, lv, Ms = ws["act"], ws["grad"], ws["c"], self.levels, ws["M"]
        self.grad.zero_()
        dy = ws["dy"] if dy is None else dy
        top = A["D0"] if lv > 1 else A["E0"]
        gtop = G["D0"] if lv > 1 else G["E0"]
        self._conv_bwd(ws, self.by_name["head"], top, None, dy, gtop, 0)
        for l in range(lv - 1):
            cat = A[f"cat{l}"]
            self._conv_bwd(ws, self.by_name[f"dec{l}b"], A[f"d{l}"], A[f"D{l}"], G[f"D{l}"], G[f"d{l}"], l)
            self._conv_bwd(ws, self.by_name[f"dec{l}a"], cat, A[f"d{l}"], G[f"d{l}"], G[f"cat{l}"], l)
            ctot = c[l + 1] + c[l]
            below = f"D{l + 1}" if l + 1 < lv - 1 else f"E{lv - 1}"
            _ok(K.unet_up_bwd(_p(G[f"cat{l}"]), ctot, 0, B, H >> (l + 1), W >> (l + 1), c[l + 1], _p(G[below]), s),
                "up_bwd")
            _ok(K.unet_take_channels(_p(G[f"cat{l}"]), ctot, c[l + 1], Ms[l], c[l], _p(G[f"E{l}"]), 0, s), "take")
        for l in range(lv - 1, -1, -1):
            if l + 1 < lv:
                _ok(K.unet_pool_bwd(_p(G[f"P{l}"]), B, H >> l, W >> l, c[l], _p(G[f"E{l}"]), 1, s), "pool_bwd")
            self._conv_bwd(ws, self.by_name[f"enc{l}b"], A[f"a{l}"], A[f"E{l}"], G[f"E{l}"], G[f"a{l}"], l)
            xin = A[f"P{l - 1}"] if l > 0 else ws["x"]
            dxin = G[f"P{l - 1}"] if l > 0 else None
            self._conv_bwd(ws, self.by_name[f"enc{l}a"], xin, A[f"a{l}"], G[f"a{l}"], dxin, l)

    def loss(self, target, weight, inv_norm, lam=0.0):
        """Masked MSE of the last forward output against target (FP32 [B*H*W*8]), plus lam x the
        squared x/y differences of the error when lam > 0; writes dLoss/dY into the workspace and
        returns the loss as a device scalar."""
        ws = self._last
        K = kernels()
        ws["loss"].zero_()
        n = ws["y"].numel()
        if lam > 0.0:
            _ok(K.unet_mse_grad(_p(ws["y"]), _p(target), _p(weight), ws["B"], ws["H"], ws["W"], OUT_PAD, float(lam),
                                float(inv_norm), _p(ws["dy"]), _p(ws["loss"]), self._stream()), "mse_grad")
        else:
            _ok(K.unet_mse(_p(ws["y"]), _p(target), _p(weight), n, float(inv_norm), _p(ws["dy"]), _p(ws["loss"]),
                           self._stream()), "mse")
        return ws["loss"]

    def adam(self, lr, b1=0.9, b2=0.999, eps=1e-8):
        K = kernels()
        self.t += 1
        _ok(K.unet_adam(_p(self.master), _p(self.grad), _p(self.m), _p(self.v), self.n_params, lr, b1, b2, eps,
                        self.t, _p(self.wt_bf16), self._stream()), "adam")
        self._transpose_weights()

    def train_step(self, B, H, W, target, weight, inv_norm, lr, X_bf16=None, lam=0.0):
        """forward + masked MSE (+ difference term) + backward + Adam; returns the loss."""
        self.forward(B, H, W, X_bf16)
        loss = self.loss(target, weight, inv_norm, lam)
        self.backward()
        self.adam(lr)
        return loss

    def wait_error(self) -> int:
        """1 if any GEMM wait timed out since the last reset (checked on the host)."""
        v = int(self.err.item())
        self.err.zero_()
        return v
