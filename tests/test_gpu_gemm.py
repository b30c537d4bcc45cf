"""The tcgen05 BF16 GEMM (culda_gemm_bf16) against an FP64 product of the same
BF16 operands.  FP32 accumulation of exact BF16 products differs from it only
by summation rounding: relative error below 1e-5 of the row's magnitude."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

import culda_cgs_b200 as cb
from culda_cgs_b200 import _ffi

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _gelu(x):
    import torch

    return 0.5 * x * (1.0 + torch.erf(x / math.sqrt(2.0)))


def _gelu_grad(x):
    import torch

    return 0.5 * (1.0 + torch.erf(x / math.sqrt(2.0))) + x * torch.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def _operands(m, n, k, lda, ldb, seed):
    import torch

    g = torch.Generator(device="cpu").manual_seed(seed)
    a = torch.randn(m, lda, generator=g).to(torch.bfloat16)
    b = torch.randn(n, ldb, generator=g).to(torch.bfloat16)
    ref = a[:, :k].double() @ b[:, :k].double().T
    return a.cuda(), b.cuda(), ref


def _run(args):
    import torch

    rc = cb.lib().culda_gemm_bf16(C.byref(args), None)
    torch.cuda.synchronize()
    return rc


@pytest.mark.parametrize("m,n,k,pad", [(128, 128, 64, 0), (256, 384, 320, 0), (384, 256, 1024, 64),
                                       (128, 1024, 512, 8)])
def test_gemm_f32_matches_fp64(m, n, k, pad):
    import torch

    lda = ldb = k + pad
    a, b, ref = _operands(m, n, k, lda, ldb, seed=m + n + k)
    bias = torch.randn(n, dtype=torch.float32, device="cuda")
    out = torch.full((m, n), float("nan"), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    args = _ffi.GemmArgs(m=m, n=n, k=k, a=_ptr(a), lda=lda, b=_ptr(b), ldb=ldb, epilogue=_ffi.CULDA_GEMM_F32,
                         alpha=0.5, out_f32=_ptr(out), ldo=n, bias=_ptr(bias), error=_ptr(err))
    assert _run(args) == 0
    assert int(err.item()) == 0
    want = 0.5 * ref + bias.cpu().double()
    got = out.cpu().double()
    scale = ref.abs().max().item()
    assert torch.isfinite(got).all()
    assert (got - want).abs().max().item() <= 1e-5 * scale


def test_gemm_bias_gelu_and_transpose():
    import torch

    m, n, k = 256, 256, 192
    a, b, ref = _operands(m, n, k, k, k, seed=5)
    bias = torch.randn(n, dtype=torch.float32, device="cuda")
    pre = torch.zeros(m, n, dtype=torch.float32, device="cuda")
    h = torch.zeros(m, n, dtype=torch.bfloat16, device="cuda")
    ht = torch.zeros(n, m + 128, dtype=torch.bfloat16, device="cuda")
    args = _ffi.GemmArgs(m=m, n=n, k=k, a=_ptr(a), lda=k, b=_ptr(b), ldb=k, epilogue=_ffi.CULDA_GEMM_BIAS_GELU,
                         out_f32=_ptr(pre), out_bf16=_ptr(h), out_bf16_t=_ptr(ht), ldo=n, ld_t=m + 128,
                         bias=_ptr(bias))
    assert _run(args) == 0
    want_pre = ref + bias.cpu().double()
    assert (pre.cpu().double() - want_pre).abs().max().item() <= 1e-5 * ref.abs().max().item()
    # the activation is GELU of the FP32 pre-activation, rounded once to BF16
    act = _gelu(pre.cpu().double())
    assert (h.cpu().double() - act).abs().max().item() <= 2.0 ** -7 * max(1.0, act.abs().max().item())
    assert torch.equal(ht[:, :m].cpu(), h.cpu().T)


def test_gemm_gelu_backward_and_bias_gradient():
    import torch

    m, n, k = 384, 128, 256
    a, b, ref = _operands(m, n, k, k, k, seed=9)
    pre = torch.randn(m, n, dtype=torch.float32, device="cuda")
    g = torch.zeros(m, n, dtype=torch.bfloat16, device="cuda")
    gt = torch.zeros(n, m, dtype=torch.bfloat16, device="cuda")
    colsum = torch.zeros(n, dtype=torch.float32, device="cuda")
    args = _ffi.GemmArgs(m=m, n=n, k=k, a=_ptr(a), lda=k, b=_ptr(b), ldb=k, epilogue=_ffi.CULDA_GEMM_GELU_BWD,
                         out_bf16=_ptr(g), out_bf16_t=_ptr(gt), ldo=n, ld_t=m, pre=_ptr(pre), colsum=_ptr(colsum))
    assert _run(args) == 0
    want = ref * _gelu_grad(pre.cpu().double())
    scale = want.abs().max().item()
    assert (g.cpu().double() - want).abs().max().item() <= 2.0 ** -7 * scale
    assert torch.equal(gt.cpu(), g.cpu().T)
    assert (colsum.cpu().double() - want.sum(0)).abs().max().item() <= 1e-4 * want.abs().sum(0).max().item()


def test_gemm_rejects_bad_shapes():
    import torch

    a = torch.zeros(128, 64, dtype=torch.bfloat16, device="cuda")
    out = torch.zeros(128, 128, dtype=torch.float32, device="cuda")
    bad = _ffi.GemmArgs(m=100, n=128, k=64, a=_ptr(a), lda=64, b=_ptr(a), ldb=64, epilogue=_ffi.CULDA_GEMM_F32,
                        alpha=1.0, out_f32=_ptr(out), ldo=128)
    assert cb.lib().culda_gemm_bf16(C.byref(bad), None) == _ffi.CULDA_ERR_INVALID_ARG
    bad.m, bad.k = 128, 48
    assert cb.lib().culda_gemm_bf16(C.byref(bad), None) == _ffi.CULDA_ERR_INVALID_ARG


@pytest.mark.parametrize("m,n,k,splits", [(128, 128, 512, 2), (256, 384, 1024, 5), (512, 256, 4096, 16),
                                          (128, 256, 192, 3)])
def test_gemm_split_k_accumulates(m, n, k, splits):
    """k cut into slices whose partial products are added with atomics into
    out_f32 (zeros, or a value to add to); bias once; same 1e-5 bound."""
    import torch

    a, b, ref = _operands(m, n, k, k, k, seed=3 * m + k)
    bias = torch.randn(n, dtype=torch.float32, device="cuda")
    base = torch.randn(m, n, dtype=torch.float32, device="cuda")
    out = base.clone()
    args = _ffi.GemmArgs(m=m, n=n, k=k, a=_ptr(a), lda=k, b=_ptr(b), ldb=k, epilogue=_ffi.CULDA_GEMM_F32,
                         alpha=1.0, out_f32=_ptr(out), ldo=n, bias=_ptr(bias), k_splits=splits)
    assert _run(args) == 0
    want = base.cpu().double() + ref + bias.cpu().double()
    assert (out.cpu().double() - want).abs().max().item() <= 1e-5 * max(1.0, ref.abs().max().item())


def test_gemm_split_k_rejects_bad_splits():
    import torch

    a = torch.zeros(128, 128, dtype=torch.bfloat16, device="cuda")
    out = torch.zeros(128, 128, dtype=torch.float32, device="cuda")
    g = torch.zeros(128, 128, dtype=torch.bfloat16, device="cuda")
    bad = _ffi.GemmArgs(m=128, n=128, k=128, a=_ptr(a), lda=128, b=_ptr(a), ldb=128,
                        epilogue=_ffi.CULDA_GEMM_F32, alpha=1.0, out_f32=_ptr(out), ldo=128, k_splits=3)
    assert cb.lib().culda_gemm_bf16(C.byref(bad), None) == _ffi.CULDA_ERR_INVALID_ARG  # 3 > k / 64
    bad2 = _ffi.GemmArgs(m=128, n=128, k=128, a=_ptr(a), lda=128, b=_ptr(a), ldb=128,
                         epilogue=_ffi.CULDA_GEMM_GELU_BWD, out_bf16=_ptr(g), out_bf16_t=_ptr(g), ldo=128, ld_t=128,
                         pre=_ptr(out), k_splits=2)
    assert cb.lib().culda_gemm_bf16(C.byref(bad2), None) == _ffi.CULDA_ERR_INVALID_ARG
