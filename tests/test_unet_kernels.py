"""Tensor-core kernels of the learned warm start against FP32 references (torch on the GPU for
plain products, torch CPU autograd for the network's gradients)."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def _gemm(L, A, B, M, N, K, epi, Cbuf=None, Y=None, ldc=None, bias=None, relu=0, splits=1, err=None):
    import torch
    code = L.unet_gemm(C.c_void_p(A.data_ptr()), A.shape[1], C.c_void_p(B.data_ptr()), B.shape[1], M, N, K, epi,
                       C.c_void_p(Cbuf.data_ptr() if Cbuf is not None else 0),
                       C.c_void_p(Y.data_ptr() if Y is not None else 0), ldc or N,
                       C.c_void_p(bias.data_ptr() if bias is not None else 0), relu, splits,
                       C.c_void_p(err.data_ptr() if err is not None else 0), None)
    torch.cuda.synchronize()
    return code


@pytest.fixture(scope="module")
def L(gpu):
    lib = gpu.lib()
    lib.unet_gemm.restype = C.c_int
    lib.unet_gemm.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                              C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    return lib


@pytest.mark.parametrize("M,N,K", [(128, 16, 64), (300, 32, 104), (1000, 64, 288), (777, 256, 1152),
                                   (5000, 128, 2304), (129, 48, 72), (64, 5, 32)])
def test_gemm_matches_fp32_reference(L, M, N, K):
    import torch
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    Cm = torch.full((M, N), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert _gemm(L, A, B, M, N, K, 0, Cbuf=Cm, err=err) == 0
    ref = A.float() @ B.float().t()
    assert int(err.item()) == 0
    rel = ((Cm - ref).abs().max() / ref.abs().max()).item()
    assert rel < 1e-5, rel


def test_gemm_split_k_and_epilogues(L):
    import torch
    M, N, K = 2000, 64, 1600
    g = torch.Generator(device="cuda").manual_seed(5)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    ref = A.float() @ B.float().t()
    Cm = torch.zeros(M, N, device="cuda")
    assert _gemm(L, A, B, M, N, K, 1, Cbuf=Cm, splits=5) == 0
    assert ((Cm - ref).abs().max() / ref.abs().max()).item() < 1e-5
    bias = torch.randn(N, device="cuda", generator=g)
    Y = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
    assert _gemm(L, A, B, M, N, K, 2, Y=Y, bias=bias, relu=1) == 0
    refy = torch.relu(ref + bias)
    assert ((Y.float() - refy).abs().max() / refy.abs().max()).item() < 1e-2   # one BF16 rounding
    Cb = torch.zeros(M, N, device="cuda")
    assert _gemm(L, A, B, M, N, K, 3, Cbuf=Cb, bias=bias) == 0
    assert ((Cb - (ref + bias)).abs().max() / ref.abs().max()).item() < 1e-5


@pytest.mark.parametrize("B,H,W,Cc,Cout", [(2, 8, 12, 8, 32), (1, 20, 20, 32, 64), (3, 7, 9, 96, 16),
                                            (1, 16, 16, 64, 256), (2, 10, 6, 16, 8)])
def test_implicit_conv_equals_im2col_gemm(L, B, H, W, Cc, Cout):
    """unet_conv3x3 gathers col(X) inside the GEMM; same K order and zero fill as im2col, so
    the results are bit-identical to unet_im2col + unet_gemm."""
    import torch
    L.unet_im2col.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    L.unet_conv3x3.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                               C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    g = torch.Generator(device="cuda").manual_seed(B * 1000 + Cc + Cout)
    M, K = B * H * W, 9 * Cc
    X = torch.randn(M, Cc, device="cuda", generator=g).to(torch.bfloat16)
    Wt = torch.randn(Cout, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(Cout, device="cuda", generator=g)
    col = torch.zeros(M, K, dtype=torch.bfloat16, device="cuda")
    assert L.unet_im2col(X.data_ptr(), B, H, W, Cc, K, col.data_ptr(), None) == 0
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    for epi in (2, 3):
        if epi == 2:
            y0 = torch.zeros(M, Cout, dtype=torch.bfloat16, device="cuda")
            y1 = torch.zeros_like(y0)
            assert _gemm(L, col, Wt, M, Cout, K, 2, Y=y0, bias=bias, relu=1) == 0
            assert L.unet_conv3x3(X.data_ptr(), B, H, W, Cc, Wt.data_ptr(), K, Cout, 2, None, y1.data_ptr(), Cout,
                                  bias.data_ptr(), 1, err.data_ptr(), None) == 0
        else:
            y0 = torch.zeros(M, Cout, device="cuda")
            y1 = torch.zeros_like(y0)
            assert _gemm(L, col, Wt, M, Cout, K, 3, Cbuf=y0, bias=bias) == 0
            assert L.unet_conv3x3(X.data_ptr(), B, H, W, Cc, Wt.data_ptr(), K, Cout, 3, y1.data_ptr(), None, Cout,
                                  bias.data_ptr(), 0, err.data_ptr(), None) == 0
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        assert torch.equal(y0, y1), (epi, (y0.float() - y1.float()).abs().max().item())
    # and against the FP32 definition of the convolution
    xn = X.float().view(B, H, W, Cc).permute(0, 3, 1, 2)
    wn = Wt.float().view(Cout, 3, 3, Cc).permute(0, 3, 1, 2)
    ref = torch.nn.functional.conv2d(xn, wn, bias, padding=1).permute(0, 2, 3, 1).reshape(M, Cout)
    assert ((y1 - ref).abs().max() / ref.abs().max()).item() < 1e-5
