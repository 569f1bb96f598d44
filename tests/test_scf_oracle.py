"""CPU checks of the SCF oracle (oracle/scf_oracle.py): its LDA and Fermi
occupations against the reference's own Calc_XC_LDA (source/Vxc.h:43-75) and
SetOccupancy (source/SetOccupancy.h:7-18) compiled from its sources, the
restated pieces against properties of the mathematics, and the committed
SCF fixture against its inputs.

Tolerances: LDA 1e-14 relative (same formulas, libm vs numpy cbrt/log);
occupations 1e-14 relative + 1e-15 absolute (libm vs numpy exp); the bcc
translation symmetry of V_loc and V_H 1e-12 relative; the bordered solve
against LAPACK 1e-12."""
import os

import numpy as np
import pytest

import oracle as O
import scf_oracle as S
from cases import SCF_C0, scf_inputs

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


@needs_ref
def test_lda_matches_reference():
    rho = np.concatenate([np.logspace(-12, 3, 4000), [0.0, 1e-8, 0.99e-8, 0.238732414637843]])
    e1, v1 = S.lda_pz(rho)
    e2, v2 = S.ref_lda_pz(rho)
    np.testing.assert_allclose(e1, e2, rtol=1e-14, atol=0)
    np.testing.assert_allclose(v1, v2, rtol=1e-14, atol=0)


@needs_ref
def test_fermi_occupations_match_reference():
    rng = np.random.default_rng(3)
    eig = np.sort(rng.uniform(-0.5, 0.5, 24))
    for n_el, kbt in ((12.0, 0.01), (17.0, 0.05), (3.0, 0.002)):
        occ, mu = S.fermi_occupations(eig, n_el, kbt)
        np.testing.assert_allclose(occ, S.ref_occupancy(eig, mu, kbt, 2.0), rtol=1e-14, atol=1e-15)
        assert abs(occ.sum() - n_el) < 1e-6


def test_bordered_solve_equals_lapack():
    rng = np.random.default_rng(1)
    R = rng.standard_normal((5, 40))
    B = R @ R.T
    M = np.zeros((6, 6))
    M[:5, :5] = B / B.diagonal().max()
    M[:5, 5] = M[5, :5] = 1.0
    rhs = np.zeros(6)
    rhs[5] = 1.0
    np.testing.assert_allclose(S.solve_bordered(M, rhs), np.linalg.solve(M, rhs), rtol=1e-12, atol=1e-12)


def test_local_and_hartree_potentials_have_the_bcc_symmetry():
    """Translation by (a/2)(1,1,1) maps the bcc cell's two atoms onto each other:
    V_loc, and V_H of a density with that symmetry, are invariant under it."""
    n, a = 24, 6.0
    h = a / n
    grid = (n, n, n, h, h, h)
    pos = O.bcc_positions(a, 1)
    v = S.gth_local_potential(grid, pos, [dict(O.GTH_BCC)] * 2).reshape(n, n, n)
    shift = np.roll(v, (n // 2, n // 2, n // 2), axis=(0, 1, 2))
    assert np.abs(shift - v).max() <= 1e-12 * np.abs(v).max()
    # the cell average of V_loc is the finite G = 0 part per volume
    sp = O.GTH_BCC
    r = sp["rloc"]
    g0 = 2 * (2 * np.pi * sp["zion"] * r * r + (2 * np.pi) ** 1.5 * r ** 3 * (sp["c1"] + 3 * sp["c2"])) / a ** 3
    assert abs(v.mean() - g0) < 1e-12 * abs(g0)
    rho = np.exp(-np.abs(v) / np.abs(v).max())
    vh, eh = S.hartree(rho.reshape(-1), grid)
    vh = vh.reshape(n, n, n)
    assert np.abs(np.roll(vh, (n // 2,) * 3, axis=(0, 1, 2)) - vh).max() <= 1e-12 * np.abs(vh).max()
    assert eh > 0.0 and abs(vh.mean()) < 1e-12 * np.abs(vh).max()


def test_scf_fixture_matches_its_inputs():
    f = np.load(os.path.join(GOLD, "scf_c0.npz"))
    inp = scf_inputs()
    np.testing.assert_allclose(f["checksum"], [float(np.sum(v)) for v in inp["checked"]], rtol=1e-15)
    assert bool(f["converged"])
    e = f["energies"]
    assert abs(e[-1] - e[-2]) / 2 < SCF_C0["params"]["tol_per_atom"]
    assert abs(f["occ"].sum() - SCF_C0["n_el"]) < 1e-6
    assert abs(f["rho"].sum() * (SCF_C0["a"] / SCF_C0["n"]) ** 3 - SCF_C0["n_el"]) < 1e-6


def test_local_forces_are_minus_the_local_energy_gradient():
    """gth_local_forces against central differences (delta 1e-4 bohr) of
    E_loc(R) = dV sum rho V_loc(R) with the density frozen: 1e-7 of the largest
    component (the Fourier series is smooth in R; error O(delta^2))."""
    n, a = 24, 6.0
    h = a / n
    grid = (n, n, n, h, h, h)
    pos = O.bcc_positions(a, 1) + np.array([[0.13, -0.07, 0.21], [-0.11, 0.05, 0.02]])
    sps = [dict(O.GTH_BCC)] * 2
    rng = np.random.default_rng(9)
    rho = 0.05 + 0.02 * rng.uniform(size=n ** 3)
    f = S.gth_local_forces(rho, grid, pos, sps)
    d = 1e-4
    fd = np.zeros_like(f)
    for at in range(2):
        for k in range(3):
            p1, p2 = pos.copy(), pos.copy()
            p1[at, k] += d
            p2[at, k] -= d
            e1 = float(np.dot(rho, S.gth_local_potential(grid, p1, sps))) * h ** 3
            e2 = float(np.dot(rho, S.gth_local_potential(grid, p2, sps))) * h ** 3
            fd[at, k] = -(e1 - e2) / (2 * d)
    assert np.abs(f).max() > 1e-3
    np.testing.assert_allclose(f, fd, rtol=0, atol=1e-7 * np.abs(f).max())
