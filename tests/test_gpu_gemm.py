"""tgl_gemm_bf16: tensor-core BF16 products against an f32 PyTorch reference.

The products of bf16 inputs are exact in f32, so the only difference from
the reference is the f32 summation order: tolerance 1e-5 relative to the
sum of |terms| (written in `check`).
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class Gemm(ctypes.Structure):
    _fields_ = [
        ("a", ctypes.c_void_p), ("b", ctypes.c_void_p), ("lda", ctypes.c_int64), ("ldb", ctypes.c_int64),
        ("m", ctypes.c_int32), ("n", ctypes.c_int32), ("k", ctypes.c_int64), ("a_mn", ctypes.c_int32),
        ("b_mn", ctypes.c_int32), ("k_split", ctypes.c_int64), ("bias", ctypes.c_void_p),
        ("relu", ctypes.c_int32), ("reserved", ctypes.c_int32), ("mask", ctypes.c_void_p),
        ("ld_mask", ctypes.c_int64), ("residual", ctypes.c_void_p), ("ld_res", ctypes.c_int64), ("out_f32", ctypes.c_void_p),
        ("ldo", ctypes.c_int64), ("out_bf16", ctypes.c_void_p), ("ldo_bf16", ctypes.c_int64),
        ("error", ctypes.c_void_p),
    ]


def run(lib, torch, a, b, m, n, k, a_mn, b_mn, bias=None, relu=False, k_split=0, want_bf16=False):
    dev = a.device
    splits = 1 if k_split == 0 else (k + k_split - 1) // k_split
    out = torch.full((splits, m, n), float("nan"), dtype=torch.float32, device=dev)
    out_bf16 = torch.empty((m, n), dtype=torch.bfloat16, device=dev) if want_bf16 else None
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    g = Gemm(a.data_ptr(), b.data_ptr(), a.shape[1], b.shape[1], m, n, k, a_mn, b_mn, k_split,
             bias.data_ptr() if bias is not None else None, int(relu), 0, None, 0, None, 0, out.data_ptr(), n,
             out_bf16.data_ptr() if want_bf16 else None, n, err.data_ptr())
    fn = lib.tgl_gemm_bf16
    fn.argtypes = [ctypes.POINTER(Gemm), ctypes.c_void_p]
    fn.restype = ctypes.c_int
    rc = fn(ctypes.byref(g), torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.tgl_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return out.sum(0), out_bf16


def check(torch, got, a_kmaj, b_kmaj, bias=None, relu=False):
    A, B = a_kmaj.float(), b_kmaj.float()
    ref = A @ B.T
    scale = A.abs() @ B.abs().T
    if bias is not None:
        ref = ref + bias
        scale = scale + bias.abs()
    if relu:
        ref = torch.clamp(ref, min=0.0)
    err = (got - ref).abs()
    assert bool((err <= 1.0e-5 * scale + 1.0e-30).all()), float((err / (scale + 1e-30)).max())


@pytest.mark.parametrize("m,n,k", [(300, 64, 80), (128, 16, 16), (1000, 192, 192), (77, 256, 64), (513, 48, 136)])
def test_k_major(m, n, k, cuda_lib):
    import torch

    g = torch.Generator(device="cuda").manual_seed(m * 7 + n)
    a = torch.randn(m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    got, _ = run(cuda_lib, torch, a, b, m, n, k, 0, 0)
    check(torch, got, a, b)


def test_bias_relu_and_bf16_output(cuda_lib):
    import torch

    m, n, k = 260, 64, 192
    a = torch.randn(m, k, device="cuda").to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda").to(torch.bfloat16)
    bias = torch.randn(n, device="cuda")
    got, got_bf16 = run(cuda_lib, torch, a, b, m, n, k, 0, 0, bias=bias, relu=True, want_bf16=True)
    check(torch, got, a, b, bias, relu=True)
    assert torch.equal(got_bf16, got.to(torch.bfloat16))


@pytest.mark.parametrize("k,k_split", [(1000, 256), (64, 0), (4097, 1024)])
def test_mn_major_split_k_weight_gradient(k, k_split, cuda_lib):
    """dW^T = dY^T X with both operands MN-major (rows = samples)."""
    import torch

    m, n = 64, 80
    dy = torch.randn(k, m, device="cuda").to(torch.bfloat16)   # [samples][out]
    x = torch.randn(k, n, device="cuda").to(torch.bfloat16)    # [samples][in]
    got, _ = run(cuda_lib, torch, dy, x, m, n, k, 1, 1, k_split=k_split)
    check(torch, got, dy.T.contiguous(), x.T.contiguous())


def test_mixed_majors(cuda_lib):
    import torch

    m, n, k = 200, 32, 96
    a = torch.randn(m, k, device="cuda").to(torch.bfloat16)
    b_t = torch.randn(k, n, device="cuda").to(torch.bfloat16)  # B MN-major
    got, _ = run(cuda_lib, torch, a, b_t, m, n, k, 0, 1)
    check(torch, got, a, b_t.T.contiguous())


def test_rejects_bad_shapes(cuda_lib):
    import torch

    a = torch.zeros(16, 16, device="cuda", dtype=torch.bfloat16)
    out = torch.zeros(16, 24, device="cuda")
    g = Gemm(a.data_ptr(), a.data_ptr(), 16, 16, 16, 24, 16, 0, 0, 0, None, 0, 0, None, 0, None, 0, out.data_ptr(), 24,
             None, 0, None)
    fn = cuda_lib.tgl_gemm_bf16
    fn.argtypes = [ctypes.POINTER(Gemm), ctypes.c_void_p]
    fn.restype = ctypes.c_int
    assert fn(ctypes.byref(g), None) == 1  # n = 24 is not a multiple of 16


def test_mask_and_residual_epilogue(cuda_lib):
    import torch

    m, n, k = 300, 64, 64
    a = torch.randn(m, k, device="cuda").to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda").to(torch.bfloat16)
    mask = torch.randn(m, n, device="cuda").to(torch.bfloat16)
    res = torch.randn(m, n, device="cuda")
    out = torch.full((m, n), float("nan"), device="cuda")
    g = Gemm(a.data_ptr(), b.data_ptr(), k, k, m, n, k, 0, 0, 0, None, 0, 0, mask.data_ptr(), n, res.data_ptr(), n,
             out.data_ptr(), n, None, 0, None)
    fn = cuda_lib.tgl_gemm_bf16
    fn.argtypes = [ctypes.POINTER(Gemm), ctypes.c_void_p]
    fn.restype = ctypes.c_int
    assert fn(ctypes.byref(g), torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    ref = (a.float() @ b.float().T) * (mask.float() > 0) + res
    scale = (a.float().abs() @ b.float().abs().T) + res.abs()
    assert bool(((out - ref).abs() <= 1.0e-5 * scale + 1e-30).all())


@pytest.mark.parametrize("m,n,k", [(40000, 64, 1024), (20000, 256, 200), (70001, 16, 8)])
def test_persistent_kernel_wraps_its_stages_and_accumulators(m, n, k, cuda_lib, monkeypatch):
    """K-major products take the persistent TMA kernel: more 128-row tiles
    than CTAs (each CTA alternates its two accumulators) and contractions of
    many 64-wide chunks (the four pipeline stages wrap around). Against the
    f32 reference, and equal to the staged kernel (the same tensor-core
    products summed in the same chunk order)."""
    import torch

    g = torch.Generator(device="cuda").manual_seed(m + n + k)
    a = torch.randn(m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(n, device="cuda", generator=g)
    got, got_bf16 = run(cuda_lib, torch, a, b, m, n, k, 0, 0, bias=bias, relu=True, want_bf16=True)
    check(torch, got, a, b, bias, relu=True)
    monkeypatch.setenv("TGL_GEMM_STAGED", "1")
    staged, staged_bf16 = run(cuda_lib, torch, a, b, m, n, k, 0, 0, bias=bias, relu=True, want_bf16=True)
    assert torch.equal(got, staged) and torch.equal(got_bf16, staged_bf16)
