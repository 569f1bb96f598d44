"""GPU check of the tcgen05 split-BF16x3 Gram product (qsb_gram_bf16x3, C ABI)
against an FP64 product of the same FP32 / FP64 inputs.

Tolerance: max |T - T64| <= 2e-5 * max |T64| (split-BF16x3 keeps ~16 mantissa
bits per operand; FP32 accumulation inside a CTA, FP64 across CTAs)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 2e-5


def _gram(qsb, U, V, p, q, upper=0):
    import torch
    N = U.shape[-1]
    same = int(U.data_ptr() == V.data_ptr())
    nbytes = ctypes.c_size_t()
    assert qsb.lib.qsb_gram_bf16x3_workspace(ctypes.c_int64(N), p, q, same, ctypes.byref(nbytes)) == 0
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device="cuda")
    T = torch.full((q, p), float("nan"), dtype=torch.float64, device="cuda")   # column-major p x q
    dt = 0 if U.dtype == torch.float64 else 1
    st = qsb.lib.qsb_gram_bf16x3(dt, ctypes.c_int64(N), p, q, ctypes.c_void_p(U.data_ptr()),
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
