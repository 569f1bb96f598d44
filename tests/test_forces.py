"""Nonlocal energy and forces (EnergyPPnonlocal_bundle / ForceNonlocal_bundle,
source/PseudoPotNonlocal_SvF2_kpoint.h:5033-5135, :3629-3731) — CPU checks of
the oracle: its restatement against the reference's own code built from its
sources, and its forces against central finite differences of its energy.

Tolerances: oracle vs reference 1e-12 relative (same tables, same order of
operations up to summation order).  Finite differences (projector cutoff
9 r_l so that no projector value jumps at the sphere edge): central
differences with delta = 1e-3 bohr within the stated force bar 1e-5 Ha/bohr,
and their Richardson extrapolation from delta and delta/2 (error O(delta^4))
within 1e-6 of the largest force component."""
import numpy as np
import pytest

import oracle as O


def _case(n=16, a=6.0, shift=0.07):
    h = a / n
    grid = (n, n, n, h, h, h)
    pos = O.bcc_positions(a, 1) + shift
    return grid, pos, [dict(O.GTH_BCC)] * len(pos)


@pytest.mark.parametrize("cplx,g", [(False, (0.0, 0.0, 0.0)), (True, (0.3, 0.2, -0.1))])
def test_oracle_energy_force_matches_reference(cplx, g):
    grid, pos, sps = _case()
    n = grid[0]
    cube = O.gth_cube_tables(pos, sps, n, n, n, *grid[3:])
    nb = 3
    psi = O.seeded_psi(5, nb, n ** 3, cplx)
    occ = np.array([2.0, 1.5, 0.5])
    soa = psi if cplx else np.stack([psi, np.zeros_like(psi)], 1).reshape(2 * nb, -1)
    e_ref, f_ref = O.ref_nonlocal_energy_force(grid, cube, soa, nb, occ, g)
    tables = (cube["npts"], cube["widths"], cube["coords"], cube["proj"], cube["energy"])
    e, f = O.nonlocal_energy_force(grid, tables, cube["grad"], psi, nb, occ, cplx, g)
    assert abs(e - e_ref) <= 1e-12 * abs(e_ref)
    np.testing.assert_allclose(f, f_ref, rtol=0, atol=1e-12 * np.abs(f_ref).max())


def _energy(grid, pos, sps, psi, nb, occ, cplx, g, rcut):
    tables = O.gth_tables(pos, sps, *grid[3:], rcut_factor=rcut)
    dbeta = O.gth_gradient_tables(pos, sps, *grid[3:], tables, rcut_factor=rcut)
    return O.nonlocal_energy_force(grid, tables, dbeta, psi, nb, occ, cplx, g)


@pytest.mark.parametrize("cplx,g", [(False, (0.0, 0.0, 0.0)), (True, (0.25, -0.4, 0.1))])
def test_oracle_force_is_minus_the_energy_gradient(cplx, g):
    grid, pos, sps = _case(n=20)
    n = grid[0]
    nb = 2
    psi = O.seeded_psi(7, nb, n ** 3, cplx)
    occ = np.array([2.0, 1.0])
    rcut, delta = 9.0, 1e-3
    _, f = _energy(grid, pos, sps, psi, nb, occ, cplx, g, rcut)

    def central(d):
        fd = np.zeros_like(f)
        for a in range(len(pos)):
            for k in range(3):
                p1, p2 = pos.copy(), pos.copy()
                p1[a, k] += d
                p2[a, k] -= d
                e1, _ = _energy(grid, p1, sps, psi, nb, occ, cplx, g, rcut)
                e2, _ = _energy(grid, p2, sps, psi, nb, occ, cplx, g, rcut)
                fd[a, k] = -(e1 - e2) / (2 * d)
        return fd

    fd1, fd2 = central(delta), central(delta / 2)
    assert np.abs(f).max() > 1e-2
    np.testing.assert_allclose(f, fd1, rtol=0, atol=1e-5)
    np.testing.assert_allclose(f, (4 * fd2 - fd1) / 3, rtol=0, atol=1e-6 * np.abs(f).max())
