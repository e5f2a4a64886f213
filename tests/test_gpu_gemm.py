"""The tcgen05 BF16 GEMM (C = A B^T, FP32 accumulation in tensor memory) against an FP64 product
of the same BF16 inputs, on shapes that are not tile multiples (TMA zero-fills the edges), for
every tile width and epilogue."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPI_ACCUM, EPI_BIAS, EPI_RELU, EPI_BF16 = 1, 2, 4, 8


def _gemm(V, a, b, out, flags=0, bias=None, bn=128):
    import torch
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    M, K = a.shape
    N = b.shape[0]
    rc = V.lib.vl_nn_gemm_bf16(C.c_void_p(a.data_ptr()), K, C.c_void_p(b.data_ptr()), K, M, N, K,
                               C.c_void_p(out.data_ptr()), out.shape[1],
                               C.cast(C.c_void_p(bias.data_ptr() if bias is not None else 0), C.POINTER(C.c_float)),
                               flags, bn, C.cast(C.c_void_p(err.data_ptr()), C.POINTER(C.c_int)), None)
    assert rc == 0, V._lib.last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0


@pytest.mark.parametrize("M,N,K,bn", [(128, 32, 64, 32), (256, 64, 128, 64), (300, 200, 1000, 128),
                                      (1000, 256, 576, 256), (130, 96, 72, 32), (4096, 128, 288, 128),
                                      (32, 320, 4096, 256), (4096, 320, 16, 256), (512, 8, 64, 32),
                                      (2048, 64, 8, 64)])
def test_gemm_matches_fp64(gpu, M, N, K, bn):
    V = gpu
    import torch
    g = torch.Generator().manual_seed(M * 7 + N * 3 + K)
    a = torch.randn(M, K, generator=g).bfloat16()
    b = torch.randn(N, K, generator=g).bfloat16()
    ref = a.double() @ b.double().T
    out = torch.zeros(M, N, dtype=torch.float32, device="cuda")
    _gemm(V, a.cuda(), b.cuda(), out, bn=bn)
    got = out.cpu().double()
    assert torch.max(torch.abs(got - ref)).item() <= 1e-4 * max(1.0, torch.max(torch.abs(ref)).item()) * (K ** 0.5)


def test_gemm_epilogues(gpu):
    V = gpu
    import torch
    g = torch.Generator().manual_seed(5)
    M, N, K = 384, 64, 192
    a = torch.randn(M, K, generator=g).bfloat16()
    b = torch.randn(N, K, generator=g).bfloat16()
    bias = torch.randn(N, generator=g).float()
    ref = a.double() @ b.double().T + bias.double()
    out = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
    _gemm(V, a.cuda(), b.cuda(), out, flags=EPI_BIAS | EPI_RELU | EPI_BF16, bias=bias.cuda(), bn=64)
    expect = torch.clamp(ref, min=0).float().bfloat16().double()
    assert torch.max(torch.abs(out.cpu().double() - expect)).item() <= 0.02 * torch.max(torch.abs(expect)).item()
    acc = torch.ones(M, N, dtype=torch.float32, device="cuda")
    _gemm(V, a.cuda(), b.cuda(), acc, flags=EPI_ACCUM, bn=64)
    ref2 = 1.0 + a.double() @ b.double().T
    assert torch.max(torch.abs(acc.cpu().double() - ref2)).item() <= 1e-3 * torch.max(torch.abs(ref2)).item()


def test_gemm_split_k_accumulates(gpu):
    """Few output tiles over a long K run as split-K partial tiles summed in a fixed order; the
    accumulate flag adds the sum to the output."""
    V = gpu
    import torch
    g = torch.Generator().manual_seed(8)
    M, N, K = 40, 96, 8192
    a = torch.randn(M, K, generator=g).bfloat16()
    b = torch.randn(N, K, generator=g).bfloat16()
    ref = a.double() @ b.double().T
    out = torch.full((M, N), 2.0, dtype=torch.float32, device="cuda")
    _gemm(V, a.cuda(), b.cuda(), out, flags=EPI_ACCUM, bn=128)
    got = out.cpu().double() - 2.0
    assert torch.max(torch.abs(got - ref)).item() <= 1e-4 * torch.max(torch.abs(ref)).item() * (K ** 0.5)
    again = torch.zeros(M, N, dtype=torch.float32, device="cuda")
    _gemm(V, a.cuda(), b.cuda(), again, bn=128)
    again2 = torch.zeros(M, N, dtype=torch.float32, device="cuda")
    _gemm(V, a.cuda(), b.cuda(), again2, bn=128)
    assert torch.equal(again, again2)


@pytest.mark.parametrize("layout", ["mn_k", "k_mn", "mn_mn"])
@pytest.mark.parametrize("M,N,K,bn", [(256, 64, 128, 64), (200, 96, 1000, 128), (640, 32, 4096, 64),
                                      (136, 256, 72, 256)])
def test_gemm_mn_major_operands(gpu, layout, M, N, K, bn):
    """Operands stored transposed (MN-major: A as [K][M], B as [K][N]) give the same product."""
    V = gpu
    import torch
    g = torch.Generator().manual_seed(M + 3 * N + 7 * K)
    a = torch.randn(M, K, generator=g).bfloat16()
    b = torch.randn(N, K, generator=g).bfloat16()
    ref = a.double() @ b.double().T
    a_mn, b_mn = layout.startswith("mn"), layout.endswith("_mn")
    ad = (a.T.contiguous() if a_mn else a).cuda()
    bd = (b.T.contiguous() if b_mn else b).cuda()
    out = torch.zeros(M, N, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    flags = (16 if a_mn else 0) | (32 if b_mn else 0)
    rc = V.lib.vl_nn_gemm_bf16(C.c_void_p(ad.data_ptr()), M if a_mn else K, C.c_void_p(bd.data_ptr()),
                               N if b_mn else K, M, N, K, C.c_void_p(out.data_ptr()), N, None, flags, bn,
                               C.cast(C.c_void_p(err.data_ptr()), C.POINTER(C.c_int)), None)
    assert rc == 0, V._lib.last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    got = out.cpu().double()
    assert torch.max(torch.abs(got - ref)).item() <= 1e-4 * max(1.0, torch.max(torch.abs(ref)).item()) * (K ** 0.5)


def test_gemm_wait_that_runs_out_reports_and_leaves_the_context_usable(gpu):
    """Failure detection without a fault: with the test hook the first operand load of every tile
    is never issued, so the tile's bounded waits run out; the kernel skips the tile, frees its
    tensor memory and sets the error word, and the next GEMM on the same context is correct."""
    V = gpu
    import torch
    g = torch.Generator().manual_seed(12)
    M, N, K = 256, 64, 256
    a = torch.randn(M, K, generator=g).bfloat16().cuda()
    b = torch.randn(N, K, generator=g).bfloat16().cuda()
    out = torch.full((M, N), 7.0, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = V.lib.vl_nn_gemm_bf16(C.c_void_p(a.data_ptr()), K, C.c_void_p(b.data_ptr()), K, M, N, K,
                               C.c_void_p(out.data_ptr()), N, None, 64, 64,
                               C.cast(C.c_void_p(err.data_ptr()), C.POINTER(C.c_int)), None)
    assert rc == 0, V._lib.last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 1
    assert bool(torch.all(out == 7.0))
    _gemm(V, a, b, out, bn=64)
    ref = a.cpu().double() @ b.cpu().double().T
    assert torch.max(torch.abs(out.cpu().double() - ref)).item() <= 1e-4 * torch.max(torch.abs(ref)).item() * K ** 0.5
