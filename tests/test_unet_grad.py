"""The warm-start U-Net on the library's kernels against the torch CPU autograd oracle.

Tolerances (stated here, used below):
* forward output: relative L2 error < 2e-2.  Both sides round the input, the weights and every
  stored activation to BF16; they differ in FP32 summation order only, which flips an
  occasional BF16 rounding.
* parameter gradients: relative L2 error < 8e-2 per layer and cosine similarity > 0.998 over
  all parameters.  The product also rounds each layer's output gradient to BF16 before its two
  GEMMs (the oracle keeps it in FP32), which adds about 0.4 % noise per element.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def un(gpu):
    import importlib
    return importlib.import_module("solver_cfd_b200.unet")


def _rand_params(un, net, seed):
    rng = np.random.default_rng(seed)
    host = np.zeros(net.n_params, np.float32)
    for L in net.convs:
        std = np.sqrt(2.0 / (9 * L.cin))
        w = np.zeros((L.kp, L.cout), np.float32)
        co = net.cout if L.name == "head" else L.cout
        w[: 9 * L.cin, :co] = rng.standard_normal((9 * L.cin, co)) * std
        host[L.off_w: L.off_w + L.kp * L.cout] = w.ravel()
        b = np.zeros(L.cout, np.float32)
        b[:co] = 0.05 * rng.standard_normal(co)
        host[L.off_b: L.off_b + L.cout] = b
    return host


def _case(un, B, H, W, seed, base=32, levels=4):
    import torch
    net = un.UNet(11, 5, base, levels, seed=seed)
    params = _rand_params(un, net, seed)
    net.set_params(params)
    rng = np.random.default_rng(seed + 1)
    X = rng.standard_normal((B, H, W, 11)).astype(np.float32)
    T = np.zeros((B, H, W, 8), np.float32)
    T[..., :5] = rng.standard_normal((B, H, W, 5))
    Wt = np.zeros((B, H, W, 8), np.float32)
    Wt[..., :5] = (rng.random((B, H, W, 5)) < 0.8).astype(np.float32)
    inv_norm = 1.0 / float(Wt.sum())
    return net, params, X, T, Wt, inv_norm


def _gpu_forward_backward(un, net, X, T, Wt, inv_norm):
    import torch
    B, H, W, _ = X.shape
    xb = torch.from_numpy(X).cuda().to(torch.bfloat16).reshape(-1)
    y = net.forward(B, H, W, xb)
    tt = torch.from_numpy(T).cuda().reshape(-1)
    ww = torch.from_numpy(Wt).cuda().reshape(-1)
    loss = net.loss(tt, ww, inv_norm)
    net.backward()
    torch.cuda.synchronize()
    assert net.wait_error() == 0
    return float(loss.item()), y.cpu().numpy().reshape(B, H, W, 8), net.grad.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("B,H,W", [(2, 32, 32), (1, 16, 64)])
def test_forward_and_gradients_match_cpu_autograd(un, B, H, W):
    from oracle import unet_ref
    net, params, X, T, Wt, inv_norm = _case(un, B, H, W, seed=B * 100 + H)
    loss_g, y_g, g_g = _gpu_forward_backward(un, net, X, T, Wt, inv_norm)
    loss_r, y_r, g_r = unet_ref.forward_loss(net.convs, net.levels, params, X, T, Wt, inv_norm)
    rel_y = np.linalg.norm(y_g - y_r) / np.linalg.norm(y_r)
    assert rel_y < 2e-2, rel_y
    assert abs(loss_g - loss_r) / loss_r < 2e-2, (loss_g, loss_r)
    worst = []
    for L in net.convs:
        sl = slice(L.off_w, L.off_b + L.cout)
        a, b = g_g[sl], g_r[sl]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        worst.append((rel, L.name))
        assert rel < 8e-2, (L.name, rel)
    cos = float(g_g @ g_r / (np.linalg.norm(g_g) * np.linalg.norm(g_r)))
    assert cos > 0.998, cos
    print("max per-layer gradient error", max(worst), "cosine", cos, "forward", rel_y)


def test_training_reduces_loss(un):
    import torch
    B, H, W = 2, 32, 32
    net, params, X, T, Wt, inv_norm = _case(un, B, H, W, seed=7)
    # a learnable target: a fixed smooth function of the input
    T[..., :5] = 0.5 * np.tanh(X[..., :5] + X[..., 6:11])
    xb = torch.from_numpy(X).cuda().to(torch.bfloat16).reshape(-1)
    tt = torch.from_numpy(T).cuda().reshape(-1)
    ww = torch.from_numpy(Wt).cuda().reshape(-1)
    losses = [float(net.train_step(B, H, W, tt, ww, inv_norm, 2e-3, xb).item()) for _ in range(60)]
    assert net.wait_error() == 0
    assert losses[-1] < 0.3 * losses[0], losses[::10]


@pytest.mark.parametrize("Cc", [5, 16])   # scalar path; 16-byte vector path (C multiple of 8)
def test_im2col_col2im_adjoint_and_pool_up(un, Cc):
    """<im2col(x), c> = <x, col2im(c)>; pooling and upsampling against their definitions."""
    import torch
    K = un.kernels()
    s = torch.cuda.current_stream().cuda_stream
    B, H, W = 2, 8, 16
    kp = (9 * Cc + 7) // 8 * 8
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn(B * H * W * Cc, device="cuda", generator=g).to(torch.bfloat16)
    col = torch.zeros(B * H * W * kp, dtype=torch.bfloat16, device="cuda")
    assert K.unet_im2col(x.data_ptr(), B, H, W, Cc, kp, col.data_ptr(), s) == 0
    cvec = torch.randn(B * H * W * kp, device="cuda", generator=g)
    dx = torch.zeros(B * H * W * Cc, device="cuda")
    assert K.unet_col2im(cvec.data_ptr(), B, H, W, Cc, kp, dx.data_ptr(), s) == 0
    lhs = float((col.double() * cvec.double()).sum())
    rhs = float((x.double() * dx.double()).sum())
    assert abs(lhs - rhs) <= 1e-4 * max(1.0, abs(lhs)), (lhs, rhs)
    # im2col against torch's unfold (same K order after a permutation)
    xn = x.float().view(B, H, W, Cc).permute(0, 3, 1, 2)
    unf = torch.nn.functional.unfold(xn, 3, padding=1)  # [B, Cc*9, H*W], index c*9 + ky*3 + kx
    ref = unf.view(B, Cc, 9, H * W).permute(0, 3, 2, 1).reshape(B * H * W, 9 * Cc)
    got = col.float().view(B * H * W, kp)
    assert torch.equal(got[:, : 9 * Cc], ref) and not got[:, 9 * Cc:].any()
    # pooling and upsampling
    y = torch.zeros(B * (H // 2) * (W // 2) * Cc, dtype=torch.bfloat16, device="cuda")
    assert K.unet_pool_fwd(x.data_ptr(), B, H, W, Cc, y.data_ptr(), s) == 0
    refp = torch.nn.functional.avg_pool2d(xn, 2).permute(0, 2, 3, 1).reshape(-1)
    assert (y.float() - refp).abs().max().item() <= 1e-2 * refp.abs().max().item()
    up = torch.zeros(B * H * W * 2 * Cc, dtype=torch.bfloat16, device="cuda")
    assert K.unet_up_fwd(y.data_ptr(), B, H // 2, W // 2, Cc, up.data_ptr(), 2 * Cc, Cc, s) == 0
    refu = torch.nn.functional.interpolate(y.float().view(B, H // 2, W // 2, Cc).permute(0, 3, 1, 2), scale_factor=2,
                                           mode="nearest").permute(0, 2, 3, 1)
    assert torch.equal(up.float().view(B, H, W, 2 * Cc)[..., Cc:], refu)


def test_adam_matches_formula(un):
    import torch
    K = un.kernels()
    s = torch.cuda.current_stream().cuda_stream
    n = 1000
    g = torch.Generator(device="cuda").manual_seed(11)
    p = torch.randn(n, device="cuda", generator=g)
    p0 = p.clone()
    m = torch.zeros(n, device="cuda")
    v = torch.zeros(n, device="cuda")
    pb = torch.zeros(n, dtype=torch.bfloat16, device="cuda")
    rp, rm, rv = p0.double(), torch.zeros(n, dtype=torch.float64, device="cuda"), torch.zeros(n, dtype=torch.float64,
                                                                                              device="cuda")
    for t in range(1, 4):
        gr = torch.randn(n, device="cuda", generator=g)
        assert K.unet_adam(p.data_ptr(), gr.data_ptr(), m.data_ptr(), v.data_ptr(), n, 1e-2, 0.9, 0.999, 1e-8, t,
                           pb.data_ptr(), s) == 0
        rm = 0.9 * rm + 0.1 * gr.double()
        rv = 0.999 * rv + 0.001 * gr.double() ** 2
        rp = rp - 1e-2 * (rm / (1 - 0.9 ** t)) / ((rv / (1 - 0.999 ** t)).sqrt() + 1e-8)
    assert (p.double() - rp).abs().max().item() < 1e-5
    assert torch.equal(pb, p.to(torch.bfloat16))


def test_difference_loss_and_smoothing(un):
    """unet_mse_grad: loss and gradient against torch autograd of
    sum w e^2 + lam sum over valid x/y neighbour pairs of (e' - e)^2 (times inv_norm);
    unet_smooth3 against a 3x3 mean over the existing neighbours."""
    import torch
    K = un.kernels()
    s = torch.cuda.current_stream().cuda_stream
    B, H, W, Cc = 2, 9, 12, 8
    g = torch.Generator(device="cuda").manual_seed(21)
    out = torch.randn(B, H, W, Cc, device="cuda", generator=g)
    tgt = torch.randn(B, H, W, Cc, device="cuda", generator=g)
    w = (torch.rand(B, H, W, Cc, device="cuda", generator=g) < 0.8).float()
    lam, inv = 3.0, 1.0 / 77.0
    dout = torch.zeros_like(out)
    loss = torch.zeros(1, device="cuda")
    assert K.unet_mse_grad(out.data_ptr(), tgt.data_ptr(), w.data_ptr(), B, H, W, Cc, lam, inv, dout.data_ptr(),
                           loss.data_ptr(), s) == 0
    o = out.double().cpu().requires_grad_(True)
    t, m = tgt.double().cpu(), w.double().cpu()
    e = (o - t) * (m > 0)
    ref = (m * e * e).sum()
    vx = (m[:, :, 1:] > 0) & (m[:, :, :-1] > 0)
    vy = (m[:, 1:] > 0) & (m[:, :-1] > 0)
    ref = ref + lam * (((e[:, :, 1:] - e[:, :, :-1]) ** 2) * vx).sum() + lam * (((e[:, 1:] - e[:, :-1]) ** 2) * vy).sum()
    ref = ref * inv
    ref.backward()
    assert abs(float(loss.item()) - float(ref)) <= 1e-4 * abs(float(ref))
    assert torch.allclose(dout.double().cpu(), o.grad, rtol=1e-4, atol=1e-6)
    sm = torch.zeros_like(out)
    assert K.unet_smooth3(out.data_ptr(), B, H, W, Cc, sm.data_ptr(), s) == 0
    x = out.permute(0, 3, 1, 2)
    refs = torch.nn.functional.avg_pool2d(x, 3, stride=1, padding=1, count_include_pad=False).permute(0, 2, 3, 1)
    assert torch.allclose(sm, refs, rtol=1e-5, atol=1e-6)
