"""GPU check of the tcgen05 split-BF16x3 Gram product (qsb_gram_bf16x3, C ABI)
against an FP64 product of the same FP32 / FP64 inputs.

Tolerance: max |T - T64| <= 2e-5 * max |T64| (split-BF16x3 keeps ~16 mantissa
bits per operand; FP32 accumulation inside a CTA, FP64 across CTAs)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 2e-5


def _gram(qsb, U, V, p, q, upper=0, products=3, kind=None):
    """kind None: split-BF16 with `products` products; "ozaki": INT8 slices."""
    import torch
    N = U.shape[-1]
    same = int(U.data_ptr() == V.data_ptr())
    nbytes = ctypes.c_size_t()
    wsq = qsb.lib.qsb_gram_ozaki_int8_workspace if kind == "ozaki" else qsb.lib.qsb_gram_bf16x3_workspace
    assert wsq(ctypes.c_int64(N), p, q, same, ctypes.byref(nbytes)) == 0
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device="cuda")
    T = torch.full((q, p), float("nan"), dtype=torch.float64, device="cuda")   # column-major p x q
    dt = 0 if U.dtype == torch.float64 else 1
    fn = qsb.lib.qsb_gram_bf16x3 if products == 3 else qsb.lib.qsb_gram_bf16x4
    if kind == "ozaki":
        fn = qsb.lib.qsb_gram_ozaki_int8
    st = fn(dt, ctypes.c_int64(N), p, q, ctypes.c_void_p(U.data_ptr()),
                                 ctypes.c_void_p(V.data_ptr()), ctypes.c_void_p(T.data_ptr()), p, upper,
                                 ctypes.c_void_p(ws.data_ptr()), ctypes.c_size_t(nbytes.value),
                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, qsb.lib.qsb_last_error()
    torch.cuda.synchronize()
    return T.t()   # p x q


@pytest.mark.parametrize("N,p,q,same,dtype", [
    (50021, 16, 16, True, "f32"),        # K tail not a multiple of 64, single tile
    (70000, 100, 37, False, "f32"),      # ragged rows and columns
    (65536, 256, 256, True, "f32"),      # 2 x 2 output tiles
    (40000, 130, 260, False, "f64"),     # 2 x 3 tiles, FP64 input
])
def test_gram_bf16x3_matches_fp64(qsb, N, p, q, same, dtype):
    import torch
    g = torch.Generator(device="cuda").manual_seed(7)
    dt = torch.float32 if dtype == "f32" else torch.float64
    U = (torch.rand(p, N, generator=g, device="cuda", dtype=torch.float64) - 0.5).to(dt)
    V = U if same else (torch.rand(q, N, generator=g, device="cuda", dtype=torch.float64) - 0.5).to(dt)
    T = _gram(qsb, U, V, p, q)
    ref = U.double() @ V.double().t()
    err = (T - ref).abs().max().item() / ref.abs().max().item()
    assert err < TOL, err
    assert qsb.device_status() == 0


def test_gram_bf16x3_upper_tiles(qsb):
    """upper = 1: every entry m <= n is the product; tiles strictly below the
    diagonal stay untouched (NaN here)."""
    import torch
    N, p = 60000, 300
    g = torch.Generator(device="cuda").manual_seed(8)
    U = (torch.rand(p, N, generator=g, device="cuda", dtype=torch.float64) - 0.5).float()
    T = _gram(qsb, U, U, p, p, upper=1)
    ref = U.double() @ U.double().t()
    iu = torch.triu_indices(p, p, device="cuda")
    err = (T[iu[0], iu[1]] - ref[iu[0], iu[1]]).abs().max().item() / ref.abs().max().item()
    assert err < TOL, err
    m = torch.arange(p, device="cuda")
    below = (m[:, None] // 128) > (m[None, :] // 128)
    assert torch.isnan(T[below]).all()
    assert qsb.device_status() == 0


def test_bf16_gram_diagonal_carries_the_accumulation_bias(qsb):
    """U^T U diagonal through the BF16 forms: the tensor core's FP32 accumulator
    rounds toward zero, so the same-sign diagonal sums come out low by an
    amount that grows with the K range one CTA accumulates (8192 points per
    CTA here: about -5e-5 relative).  This is the measurement behind the INT8
    default of the mixed-precision solver."""
    import torch
    N, p = 148 * 8192, 64
    g = torch.Generator(device="cuda").manual_seed(9)
    U = (torch.rand(p, N, generator=g, device="cuda", dtype=torch.float64) - 0.5).float()
    ref = (U.double() * U.double()).sum(1)
    for products in (3, 4):
        d = torch.diagonal(_gram(qsb, U, U, p, p, products=products))
        rel = ((d - ref) / ref).mean().item()
        assert -2e-4 < rel < -1e-5, (products, rel)
    assert qsb.device_status() == 0


@pytest.mark.parametrize("N,p,q,same,dtype,upper", [
    (50021, 16, 16, True, "f32", 0),         # K tail not a multiple of 128, single tile
    (70000, 100, 37, False, "f32", 0),       # ragged rows and columns
    (65536, 256, 256, True, "f32", 1),       # upper tiles of a 2 x 2 grid
    (40000, 130, 260, False, "f64", 0),      # 2 x 3 tiles, FP64 input
])
def test_gram_ozaki_int8_matches_fp64(qsb, N, p, q, same, dtype, upper):
    import torch
    g = torch.Generator(device="cuda").manual_seed(17)
    dt = torch.float32 if dtype == "f32" else torch.float64
    U = (torch.rand(p, N, generator=g, device="cuda", dtype=torch.float64) - 0.5).to(dt)
    V = U if same else (torch.rand(q, N, generator=g, device="cuda", dtype=torch.float64) - 0.5).to(dt)
    T = _gram(qsb, U, V, p, q, upper=upper, kind="ozaki")
    ref = U.double() @ V.double().t()
    if upper:
        iu = torch.triu_indices(p, q, device="cuda")
        err = (T[iu[0], iu[1]] - ref[iu[0], iu[1]]).abs().max().item()
    else:
        err = (T - ref).abs().max().item()
    assert err / ref.abs().max().item() < 5e-6, err
    assert qsb.device_status() == 0


def test_gram_ozaki_int8_has_no_diagonal_bias(qsb):
    """Same long-chain case as the BF16 bias test: integer accumulation leaves
    the diagonal unbiased (mean relative error below 2e-8) and every entry
    within 1e-6 of the FP64 product."""
    import torch
    N, p = 148 * 8192, 64
    g = torch.Generator(device="cuda").manual_seed(9)
    U = (torch.rand(p, N, generator=g, device="cuda", dtype=torch.float64) - 0.5).float()
    full = U.double() @ U.double().t()
    T = _gram(qsb, U, U, p, p, kind="ozaki")
    rel = ((torch.diagonal(T) - torch.diagonal(full)) / torch.diagonal(full)).mean().item()
    assert abs(rel) < 2e-8, rel
    assert (T - full).abs().max().item() / full.abs().max().item() < 1e-6
    assert qsb.device_status() == 0


@pytest.mark.parametrize("N,K,q", [
    (50021, 96, 40),       # ragged everything: grid tail, K < one stage, q < one tile
    (65536, 384, 256),     # the mixed LOBPCG shape: three K stages, two column tiles
    (70000, 200, 130),     # K tail inside a stage, column tail in the second tile
])
def test_rotation_ozaki_int8_matches_fp64(qsb, N, K, q):
    """OUT = U C on the INT8 tensor cores (MN-major A operand) against the FP64
    product: every element within 5e-6 of max|OUT|."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(21)
    U = (torch.rand(K, N, generator=g, device="cuda", dtype=torch.float64) - 0.5).float()
    U[K // 3] *= 1e-3                                    # columns of very different scale
    C = torch.randn(q, K, generator=g, device="cuda", dtype=torch.float64)   # column-major K x q
    nbytes = ctypes.c_size_t()
    assert qsb.lib.qsb_rotate_ozaki_int8_workspace(ctypes.c_int64(N), K, q, ctypes.byref(nbytes)) == 0
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device="cuda")
    out = torch.full((q, N), float("nan"), dtype=torch.float32, device="cuda")
    st = qsb.lib.qsb_rotate_ozaki_int8(1, ctypes.c_int64(N), K, q, ctypes.c_void_p(U.data_ptr()),
                                       ctypes.c_void_p(C.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                       ctypes.c_void_p(ws.data_ptr()), ctypes.c_size_t(nbytes.value),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, qsb.lib.qsb_last_error()
    torch.cuda.synchronize()
    ref = C @ U.double()                                 # q x N: column j of OUT is row j here
    err = (out.double() - ref).abs().max().item() / ref.abs().max().item()
    assert err < 5e-6, err
    assert qsb.device_status() == 0
