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


def test_ewald_is_independent_of_the_splitting_and_its_forces_are_exact():
    """The Ewald energy does not depend on the splitting alpha (1e-10
    relative); the forces equal central differences of the energy (delta 1e-4,
    1e-7 relative); the NaCl-like check: a rocksalt cell's energy per ion pair
    gives the Madelung constant 1.7475646 (1e-7)."""
    rng = np.random.default_rng(2)
    cell = (7.0, 8.0, 9.0)
    pos = rng.uniform(0, 7, (3, 3))
    Z = np.array([6.0, 1.0, 1.0])
    e1, f1 = S.ewald(pos, Z, cell, alpha=0.5)
    e2, f2 = S.ewald(pos, Z, cell, alpha=0.9)
    assert abs(e1 - e2) < 1e-10 * abs(e1)
    np.testing.assert_allclose(f1, f2, rtol=0, atol=1e-9 * np.abs(f1).max())
    d = 1e-4
    for a in range(3):
        for k in range(3):
            p1, p2 = pos.copy(), pos.copy()
            p1[a, k] += d
            p2[a, k] -= d
            fd = -(S.ewald(p1, Z, cell)[0] - S.ewald(p2, Z, cell)[0]) / (2 * d)
            assert abs(fd - f1[a, k]) < 1e-7 * np.abs(f1).max()
    # rocksalt: conventional cell of edge 2 (nearest neighbour 1), 4 Na+ and 4 Cl-
    fcc = np.array([[0, 0, 0], [0, 1, 1], [1, 0, 1], [1, 1, 0]], float)
    pos = np.vstack([fcc, fcc + np.array([1.0, 0, 0])])
    Z = np.array([1.0] * 4 + [-1.0] * 4)
    e, _ = S.ewald(pos, Z, (2.0, 2.0, 2.0), alpha=2.0)
    assert abs(-e / 4 - 1.74756459463) < 1e-7


def test_library_ewald_matches_the_oracle():
    """qsb_ewald (host code in the C-ABI library) against the oracle's Ewald sum:
    energy 1e-12 relative, forces 1e-10 of the largest; the rocksalt Madelung
    constant to 1e-9."""
    import qsb
    rng = np.random.default_rng(5)
    for cell, Z in (((7.0, 8.0, 9.0), [6.0, 1.0, 1.0]), ((20.0, 20.0, 20.0), [6.0, 1.0, 1.0]),
                    ((12.0, 12.0, 12.0), [6.0] * 16)):
        pos = rng.uniform(0, min(cell), (len(Z), 3))
        e, f = qsb.ewald(pos, Z, cell)
        eo, fo = S.ewald(pos, np.array(Z), cell)
        assert abs(e - eo) <= 1e-12 * abs(eo)
        np.testing.assert_allclose(f, fo, rtol=0, atol=1e-10 * np.abs(fo).max())
    fcc = np.array([[0, 0, 0], [0, 1, 1], [1, 0, 1], [1, 1, 0]], float)
    e, _ = qsb.ewald(np.vstack([fcc, fcc + np.array([1.0, 0, 0])]), [1.0] * 4 + [-1.0] * 4, (2.0, 2.0, 2.0))
    assert abs(-e / 4 - 1.74756459463) < 1e-9
