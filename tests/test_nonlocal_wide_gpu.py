"""GPU parity of the nonlocal kernels at projector widths 5-16 per atom (the
forms UPF species with d and f channels use: the kernels' WM = 9 and WM = 16
instantiations), against the oracle's C restatement, through the C ABI.
Seeded synthetic tables: voxel spheres around three atoms with seeded values,
widths (5, 13, 16) and (8, 2, 9); FP64 1e-12 relative L2 (the H.psi bar) for
H.psi, the nonlocal increment, the projections and the nonlocal energy and
forces."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def _tables(grid, pos, widths, radius, seed):
    nx, ny, nz, dx, dy, dz = grid
    rng = np.random.default_rng(seed)
    npts, coords, beta, energy, dbeta = [], [], [], [], []
    for R, w in zip(pos, widths):
        pts = []
        r = int(np.ceil(radius / min(dx, dy, dz)))
        c = np.round(np.array(R) / np.array([dx, dy, dz])).astype(int)
        for k in range(-r, r + 1):
            for j in range(-r, r + 1):
                for i in range(-r, r + 1):
                    p = c + np.array([i, j, k])
                    if np.sum(((p * np.array([dx, dy, dz])) - R) ** 2) <= radius ** 2:
                        pts.append(p)
        pts = np.array(pts, np.int32)
        npts.append(len(pts))
        coords.append(pts.ravel())
        beta.append(rng.uniform(-1, 1, len(pts) * w))
        dbeta.append(rng.uniform(-1, 1, 3 * len(pts) * w))
        energy.append(rng.uniform(-2, 2, w))
    return ((np.array(npts, np.int32), np.array(widths, np.int32), np.concatenate(coords).astype(np.int32),
             np.concatenate(beta), np.concatenate(energy)), np.concatenate(dbeta))


@pytest.mark.parametrize("widths", [(5, 13, 16), (8, 2, 9)])
@pytest.mark.parametrize("cplx", [False, True])
def test_wide_projector_sets_vs_oracle(qsb, widths, cplx):
    import torch
    grid = (20, 18, 16, 0.3, 0.3, 0.3)
    nx, ny, nz = grid[:3]
    N = nx * ny * nz
    g = (0.3, -0.2, 0.5) if cplx else (0.0, 0.0, 0.0)
    pos = [(1.1, 1.0, 0.9), (3.9, 4.2, 2.5), (5.4, 1.2, 4.3)]    # the first sphere wraps around the cell
    tab, dbeta = _tables(grid, pos, widths, 1.6, 41)
    V = O.seeded_potential(41, N)
    nb = 6
    psi = O.seeded_psi(41, nb, N, cplx)
    H = qsb.Hamiltonian(*grid)
    H.set_potential(V)
    H.set_projectors(*tab)
    H.set_projector_gradients(dbeta)
    p = torch.from_numpy(np.ascontiguousarray(psi)).cuda()
    hp = torch.empty_like(p)
    H.apply(p, hp, cplx, g)
    assert rel(hp.cpu().numpy(), O.hamiltonian(grid, V, tab, psi, nb, cplx, g)) < 1e-12
    base = O.seeded_psi(42, nb, N, cplx)
    inc = torch.from_numpy(base.copy()).cuda()
    H.nonlocal_apply(p, inc, cplx, g)
    ref = O.nonlocal_apply(grid, tab, psi, nb, cplx, g, hp=base.copy())
    assert rel(inc.cpu().numpy() - base, ref - base) < 1e-12
    assert rel(H.nonlocal_project(p, cplx, g), O.nonlocal_project(grid, tab, psi, nb, cplx, g)) < 1e-12
    occ = np.linspace(2.0, 0.5, nb)
    e, f = H.nonlocal_energy_force(p, occ, len(pos), cplx, g)
    e_o, f_o = O.nonlocal_energy_force(grid, tab, dbeta, psi, nb, occ, cplx, g)
    assert abs(e - e_o) <= 1e-12 * abs(e_o)
    assert rel(np.asarray(f).reshape(-1, 3), f_o) < 1e-12
    assert qsb.device_status() == 0
