"""The tcgen05 BF16 GEMM (gsv_mlp_gemm) against a plain PyTorch FP32
reference of the same product on the same BF16 inputs.

Products of BF16 values are exact in FP32, so only the accumulation order
differs: relative error bar 1e-5 for FP32 outputs; BF16 outputs are compared
after rounding the reference the same way (bar: 1 BF16 ulp)."""
import ctypes

import pytest
import torch

from gs_tmi_b200._lib import check, lib

pytestmark = pytest.mark.gpu

EPI_F32, EPI_BIAS_GELU, EPI_GELU_GRAD, EPI_ATOMIC_F32 = 0, 1, 2, 3


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def gemm(a, a_strides, b, b_strides, M, N, K, epi, out_f32=None, out_bf16=None, z=None, bias=None, c_strides=None,
         splits=1, col_sum=None):
    err = torch.zeros(1, dtype=torch.int32, device=a.device)
    c_sm, c_sn = c_strides if c_strides else (N, 1)
    check(lib.gsv_mlp_gemm(_p(a), a_strides[0], a_strides[1], _p(b), b_strides[0], b_strides[1], M, N, K, splits,
                           _p(bias), _p(out_f32), _p(out_bf16), _p(z), c_sm, c_sn, epi, _p(col_sum), _p(err),
                           ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), "gsv_mlp_gemm")
    torch.cuda.synchronize()
    assert int(err.item()) == 0, "tensor-core wait timed out"


def rel(a, b):
    return float((a.double() - b.double()).norm() / b.double().norm().clamp_min(1e-30))


@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (256, 256, 256), (300, 256, 250), (1000, 16, 256),
                                   (128, 16, 16), (512, 512, 64)])
def test_gemm_f32_k_major(M, N, K, cuda_device):
    g = torch.Generator(device=cuda_device).manual_seed(M * 7 + N + K)
    a = torch.randn(M, K, device=cuda_device, generator=g).bfloat16()
    b = torch.randn(N, K, device=cuda_device, generator=g).bfloat16()
    bias = torch.randn(N, device=cuda_device, generator=g)
    out = torch.empty(M, N, device=cuda_device)
    gemm(a, (K, 1), b, (K, 1), M, N, K, EPI_F32, out_f32=out, bias=bias)
    ref = a.float() @ b.float().t() + bias
    assert rel(out, ref) < 1e-5


@pytest.mark.parametrize("B,F1,F2", [(4096, 256, 256), (1000, 240, 196), (777, 16, 256)])
def test_gemm_transposed_operands_split_k(B, F1, F2, cuda_device):
    """Weight-gradient shape: C = dZ^T X with K = batch, split over CTAs
    (row-contiguous operands: MN-major copies; F2 = 196 takes the
    element-wise path for A)."""
    g = torch.Generator(device=cuda_device).manual_seed(3)
    dz = torch.randn(B, F2, device=cuda_device, generator=g).bfloat16()
    x = torch.randn(B, F1, device=cuda_device, generator=g).bfloat16()
    out = torch.zeros(F2, F1, device=cuda_device)
    gemm(dz, (1, F2), x, (1, F1), F2, F1, B, EPI_ATOMIC_F32, out_f32=out, splits=16)
    ref = dz.float().t() @ x.float()
    assert rel(out, ref) < 1e-5
    # transposed output store: C^T via output strides
    out_t = torch.zeros(F1, F2, device=cuda_device)
    gemm(dz, (1, F2), x, (1, F1), F2, F1, B, EPI_ATOMIC_F32, out_f32=out_t, splits=8, c_strides=(1, F2))
    assert rel(out_t, ref.t()) < 1e-5


def test_gemm_gelu_epilogues(cuda_device):
    M, N, K = 384, 256, 256
    g = torch.Generator(device=cuda_device).manual_seed(5)
    x = torch.randn(M, K, device=cuda_device, generator=g).bfloat16()
    w = (torch.randn(N, K, device=cuda_device, generator=g) * 0.1).bfloat16()
    bias = torch.randn(N, device=cuda_device, generator=g) * 0.1
    z = torch.empty(M, N, device=cuda_device)
    y = torch.empty(M, N, device=cuda_device, dtype=torch.bfloat16)
    gemm(x, (K, 1), w, (K, 1), M, N, K, EPI_BIAS_GELU, out_bf16=y, z=z, bias=bias)
    zr = x.float() @ w.float().t() + bias
    assert rel(z, zr) < 1e-5
    yr = torch.nn.functional.gelu(zr, approximate="tanh")
    assert (y.float() - yr).abs().max() <= 2 ** -7 * yr.abs().max()
    # backward through GELU: dZ = (dY W) * gelu'(z), with W used transposed
    dy = torch.randn(M, N, device=cuda_device, generator=g).bfloat16()
    dz = torch.empty(M, K, device=cuda_device, dtype=torch.bfloat16)
    zin = torch.randn(M, K, device=cuda_device, generator=g)
    colsum = torch.zeros(K, device=cuda_device)
    gemm(dy, (N, 1), w, (1, K), M, K, N, EPI_GELU_GRAD, out_bf16=dz, z=zin, col_sum=colsum)
    zz = zin.clone().requires_grad_(True)
    torch.nn.functional.gelu(zz, approximate="tanh").backward(dy.float() @ w.float())
    assert rel(dz.float(), zz.grad) < 1e-2
    # fused bias gradient: column sums of the stored BF16 output
    assert rel(colsum, dz.float().sum(0)) < 1e-5


def test_tensor_core_wait_time_out_is_reported(cuda_device):
    """The bounded mbarrier wait's error path: with one K stage's MMAs and
    commit left out (first, middle and last of four stages) the wait on that
    stage runs out after 1024 polls; every CTA latches the error flag and
    returns without its epilogue (C keeps its NaN fill), and the stream and
    the regular GEMM still work afterwards."""
    M, N, K = 256, 256, 256
    g = torch.Generator(device=cuda_device).manual_seed(11)
    a = torch.randn(M, K, device=cuda_device, generator=g).bfloat16()
    b = torch.randn(N, K, device=cuda_device, generator=g).bfloat16()
    err = torch.zeros(1, dtype=torch.int32, device=cuda_device)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for skip in (0, 1, 3):
        out = torch.full((M, N), float("nan"), device=cuda_device)
        err.zero_()
        check(lib.gsv_mlp_gemm_test_timeout(_p(a), _p(b), M, N, K, _p(out), skip, 1 << 10, _p(err), st),
              "gsv_mlp_gemm_test_timeout")
        torch.cuda.synchronize()
        assert int(err.item()) == 1, skip
        assert bool(torch.isnan(out).all()), skip
    # out-of-range hooks are refused before any launch
    for skip, limit in ((4, 1024), (-1, 1024), (0, 0), (0, (1 << 26) + 1)):
        assert lib.gsv_mlp_gemm_test_timeout(_p(a), _p(b), M, N, K, _p(out), skip, limit, _p(err), st) != 0
    out = torch.empty(M, N, device=cuda_device)
    gemm(a, (K, 1), b, (K, 1), M, N, K, EPI_F32, out_f32=out)
    assert rel(out, a.float() @ b.float().t()) < 1e-5
