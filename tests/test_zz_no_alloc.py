"""The allocation-free nonlocal apply (qsb_ham_nonlocal_apply_static), called
through the C ABI, against the regular entry point (qsb_ham_nonlocal_apply).

Some callers must not allocate device memory while they run (codes that keep
all device memory in their own arena, loops that cannot take cudaMalloc's
device-wide synchronization); this entry point serves them from a fixed 4 MiB
device array.  Two calls in a row with different inputs, each compared with
the regular path at the FP64 H.psi tolerance, show that the shared array's left
over contents do not leak into a result.  This file is collected last."""
import ctypes

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
TOL64 = 1e-12


def _call(qsb, fn, H, psi, hpsi, cplx, g):
    import torch
    nb = psi.numel() // ((2 if cplx else 1) * H.N)
    st = fn(H._h, 0, int(cplx), nb, ctypes.c_void_p(psi.data_ptr()), ctypes.c_void_p(hpsi.data_ptr()),
            ctypes.c_double(g[0]), ctypes.c_double(g[1]), ctypes.c_double(g[2]),
            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    if st != 0:
        raise qsb.QsbError(st, qsb.lib.qsb_last_error().decode())
    torch.cuda.synchronize()
    return hpsi


def _rel(a, b):
    return float((a - b).norm() / b.norm())


def test_static_scratch_matches_regular_nonlocal_apply_twice(qsb):
    import torch
    n = 24
    h = 6.0 / n
    H = qsb.Hamiltonian(n, n, n, h, h, h)
    H.set_potential(O.seeded_potential(3, n ** 3))
    pos = O.bcc_positions(6.0, 1) + 0.07
    H.set_gth_projectors(pos, [0, 0], [2], [O.GTH_BCC["r"]], [O.GTH_BCC["h"]], O.RCUT_FACTOR)
    cases = [(False, (0.0, 0.0, 0.0), 6, 31), (True, (0.26, 0.52, -0.1), 3, 32)]
    for cplx, g, nb, seed in cases:                 # two calls in a row, different inputs
        psi = torch.from_numpy(O.seeded_psi(seed, nb, n ** 3, cplx)).cuda()
        base = torch.from_numpy(O.seeded_psi(seed + 1, nb, n ** 3, cplx)).cuda()
        want = _call(qsb, qsb.lib.qsb_ham_nonlocal_apply, H, psi, base.clone(), cplx, g) - base
        got = _call(qsb, qsb.lib.qsb_ham_nonlocal_apply_static, H, psi, base.clone(), cplx, g) - base
        assert want.norm().item() > 0
        assert _rel(got, want) < TOL64


def test_static_scratch_rejects_oversized_requests(qsb):
    import torch
    n = 16
    h = 6.0 / n
    H = qsb.Hamiltonian(n, n, n, h, h, h)
    H.set_potential(O.seeded_potential(4, n ** 3))
    H.set_gth_projectors(O.bcc_positions(6.0, 1), [0, 0], [2], [O.GTH_BCC["r"]], [O.GTH_BCC["h"]], O.RCUT_FACTOR)
    # 2 atoms of one chunk each, 4 projectors: 128 B of scratch per column, so
    # 40000 real bands need 5 MB > 4 MiB.  The size check comes before any
    # device access, so one small buffer stands in for both bundles.
    nb = 40000
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    ptr = ctypes.c_void_p(buf.data_ptr())
    st = qsb.lib.qsb_ham_nonlocal_apply_static(H._h, 0, 0, nb, ptr, ptr, ctypes.c_double(0.0), ctypes.c_double(0.0),
                                               ctypes.c_double(0.0),
                                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 1                                   # QSB_ERR_INVALID
    assert "static scratch holds" in qsb.lib.qsb_last_error().decode()
    torch.cuda.synchronize()
    assert buf.abs().sum().item() == 0.0             # nothing was touched
