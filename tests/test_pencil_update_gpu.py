"""The steady-state pencil update of the FP64 complex LOBPCG (NextMatrix_z,
source/lobpcg_z_multi_mpi.h:579-794, and the skipped blocks of
MakeMatrix_z_blas, :2091-2101), called through the C ABI.

Between full recomputes (every 6 iterations and the first of each call) only
the R blocks of the Rayleigh-Ritz pencil are formed from the bundles; the X/P
blocks come from the previous pencil.  The update is exact arithmetic on the
same subspace, so the solver with it follows the solver that forms every block
from the bundles: eigenvalues after every call to 1e-9 Ha, and both reach the
reference's own trajectory (tests/golden/lobpcg_z_ref.npz) to 1e-7 Ha."""
import os

import numpy as np
import pytest

import oracle as O
from cases import EIG_G, EIG_NB, eig_inputs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _setup(qsb, mode):
    import torch
    inp = eig_inputs(0, True)
    nx, ny, nz, dx, dy, dz = inp["grid"]
    H = qsb.Hamiltonian(nx, ny, nz, dx, dy, dz)
    H.set_potential(inp["V"])
    sp = inp["sp"][0]
    H.set_gth_projectors(inp["pos"], [0] * len(inp["pos"]), [sp["nl"]], [sp["r"]], [sp["h"]], O.RCUT_FACTOR)
    es = qsb.EigenSolver(nx * ny * nz, EIG_NB, True)
    es.set_hamiltonian(H, EIG_G)
    es.set_pencil_update(mode)
    X = torch.from_numpy(inp["X"].copy()).cuda()
    return inp, H, es, X, torch.zeros_like(X)


def _run(es, inp, X, keep, calls, iter_max):
    ev = np.zeros(EIG_NB)
    out, stats, nf = [], [], 0
    for step in range(calls):
        nf = es.lobpcg_z(inp["dV"], EIG_NB, iter_max, ev, X, keep, nf, 1e-4, step)
        out.append(np.concatenate([ev, [nf]]))
        stats.append(es.pencil_stats() + es.last_stats())
    return np.array(out), stats


def test_steady_state_follows_full_pencils_and_the_reference(qsb):
    inp, H, es, X, keep = _setup(qsb, 1)
    steady, st1 = _run(es, inp, X, keep, 3, 4)
    inp, H0, es0, X0, keep0 = _setup(qsb, 0)
    full, st0 = _run(es0, inp, X0, keep0, 3, 4)
    # per call of 4 iterations: the first pencil in full, three by the update
    # (no rollback in this run); mode 0 forms all four in full
    assert st1 == [(1, 3, 4, 0)] * 3
    assert st0 == [(4, 0, 4, 0)] * 3
    np.testing.assert_array_equal(steady[:, 8], full[:, 8])
    np.testing.assert_allclose(steady[:, :8], full[:, :8], rtol=0, atol=1e-9)
    ref = np.load(os.path.join(GOLD, "lobpcg_z_ref.npz"))["out"]
    np.testing.assert_array_equal(steady[:, 8], ref[:, 8])
    np.testing.assert_allclose(steady[:, :8], ref[:, :8], rtol=0, atol=1e-7)
    # the states agree as well: X normalized, same span
    import torch
    assert torch.allclose(X, X0, rtol=0, atol=1e-6)


def test_full_recompute_every_sixth_iteration(qsb):
    inp, H, es, X, keep = _setup(qsb, 1)
    traj, stats = _run(es, inp, X, keep, 10, 8)
    # iterations 0 and 6 of each call form the whole pencil (S_MAT_REST_LIMIT = 6),
    # the other six are updated; a call that rolls back ends early
    assert stats[:2] == [(2, 6, 8, 0)] * 2
    for full, steady, iters, rolled in stats:
        assert full >= 1 and full + steady == iters
    exact = np.load(os.path.join(GOLD, "eig_exact_z.npz"))["out"]
    np.testing.assert_allclose(traj[-1][:6], exact[:6], rtol=0, atol=1e-6)
