"""The batched H psi of independent systems (qsb_ham_apply_batch: the FD8 + V
part of all systems in one persistent launch) and the autotuner
(qsb_set_autotune / qsb_autotune_report), through the C ABI.

Systems in the manner of config 4's independent-system part: cubic cells with
edges drawn from {32, 40, 48, 56, 64} (h = 0.25 bohr), 5 to 24 bands and 1 to 4
GTH atoms at seeded positions (seed 4).  Bars: FP64 batched = each system's own
qsb_ham_apply (itself pinned to the reference) to 1e-12 relative L2, FP32
batched = FP64 to 2e-5; tuned applies equal untuned ones to 1e-12, and the
decision log names the shapes it timed."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _systems(qsb, n_sys=6, seed=4):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_sys):
        n = int(rng.choice([32, 40, 48, 56, 64]))
        nb = int(rng.integers(5, 25))
        na = int(rng.integers(1, 5))
        h = 0.25
        L = n * h
        pos = rng.uniform(0, L, (na, 3))
        H = qsb.Hamiltonian(n, n, n, h, h, h)
        H.set_potential(O.seeded_potential(seed + i, n ** 3))
        H.set_gth_projectors(pos, [0] * na, [O.GTH_BCC["nl"]], [O.GTH_BCC["r"]], [O.GTH_BCC["h"]], O.RCUT_FACTOR)
        psi = O.seeded_psi(seed + 10 * i, nb, n ** 3)
        out.append((H, psi))
    return out


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_batched_apply_equals_per_system_apply(qsb, dtype):
    import torch
    dt = torch.float64 if dtype == "f64" else torch.float32
    systems = _systems(qsb)
    hams = [H for H, _ in systems]
    psis = [torch.from_numpy(p).to("cuda", dt) for _, p in systems]
    got = [torch.zeros_like(p) for p in psis]
    qsb.apply_batch(hams, psis, got)
    for (H, p64), g, p in zip(systems, got, psis):
        ref = torch.empty(p64.shape, dtype=torch.float64, device="cuda")
        H.apply(torch.from_numpy(p64).cuda(), ref)
        assert _rel(g.double().cpu().numpy(), ref.cpu().numpy()) < (1e-12 if dtype == "f64" else 2e-5)
    assert qsb.device_status() == 0


def test_autotuned_applies_equal_untuned_and_are_logged(qsb):
    import torch
    systems = _systems(qsb, n_sys=3, seed=9)
    hams = [H for H, _ in systems]
    psis = [torch.from_numpy(p).cuda() for _, p in systems]
    want = [torch.zeros_like(p) for p in psis]
    for H, p, w in zip(hams, psis, want):
        H.apply(p, w)
    want_b = [torch.zeros_like(p) for p in psis]
    qsb.apply_batch(hams, psis, want_b)
    qsb.set_autotune(True)
    try:
        for rep in range(2):                          # the first call tunes, the second uses the choice
            for H, p, w in zip(hams, psis, want):
                got = torch.zeros_like(p)
                H.apply(p, got)
                assert _rel(got.cpu().numpy(), w.cpu().numpy()) < 1e-12
            got_b = [torch.zeros_like(p) for p in psis]
            qsb.apply_batch(hams, psis, got_b)
            for g, w in zip(got_b, want_b):
                assert _rel(g.cpu().numpy(), w.cpu().numpy()) < 1e-12
        log = qsb.autotune_report()
    finally:
        qsb.set_autotune(False)
    for H, p in systems:
        n = round(len(p[0]) ** (1 / 3))
        assert f"stencil {n}x{n}x{n} real" in log, log
    assert "ham_apply_batch 3 systems" in log and "->" in log, log
    assert qsb.device_status() == 0
