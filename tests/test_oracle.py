"""CPU tests of the oracle: the C restatement against golden outputs of the
reference's own code (tests/golden, made by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import oracle as O
from cases import CASES

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", sorted(n for n in CASES if CASES[n]["oracle"] is not None))
def test_restatement_matches_reference_golden(name):
    case = CASES[name]
    inp = case["inputs"]()
    gold = np.load(os.path.join(GOLD, name + ".npz"))
    # the seeded inputs are the ones the fixture was made from
    np.testing.assert_array_equal(gold["checksum"], np.array([float(np.sum(v)) for v in inp["checked"]]))
    out = case["oracle"](inp)
    ref = gold["out"]
    assert out.shape == ref.shape
    if name.startswith("lap_"):
        # same operations in the same order: bit-exact
        np.testing.assert_array_equal(out, ref)
    else:
        # H.psi: sphere vs cube projector layout and BLAS summation order differ
        assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < 1e-14


@pytest.mark.skipif(not O.ref_available(), reason="reference oracle library not built here")
@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_reproduces_golden(name):
    case = CASES[name]
    inp = case["inputs"]()
    gold = np.load(os.path.join(GOLD, name + ".npz"))
    np.testing.assert_array_equal(gold["checksum"], np.array([float(np.sum(v)) for v in inp["checked"]]))
    out = case["reference"](inp)
    if name.startswith("eig_exact"):
        np.testing.assert_allclose(out, gold["out"], rtol=0, atol=1e-12)   # LAPACK eigvalsh
    else:
        np.testing.assert_array_equal(out, gold["out"])


def test_reference_lobpcg_fixtures_approach_exact_eigenvalues():
    """The reference solver trajectories stored as fixtures head for the exact
    (dense) eigenvalues: the lowest band gains with every SCF call."""
    for kind in ("z", "d"):
        traj = np.load(os.path.join(GOLD, f"lobpcg_{kind}_ref.npz"))["out"][:, :8]
        exact = np.load(os.path.join(GOLD, f"eig_exact_{kind}.npz"))["out"]
        err = np.abs(traj - exact[None, :])
        assert np.all(np.diff(err[:, 0]) < 0)
        assert np.all(traj >= exact[None, :] - 1e-12)     # Ritz values bound from above


def test_oracle_hamiltonian_is_symmetric():
    """<phi|H psi> = <H phi|psi> for the real Gamma-point H (FD8 + V + KB projectors)."""
    nx = ny = nz = 16
    h = 6.0 / 16
    grid = (nx, ny, nz, h, h, h)
    pos = O.bcc_positions(6.0, 1)
    tab = O.gth_tables(pos, [O.GTH_BCC] * 2, h, h, h)
    V = O.seeded_potential(7, nx * ny * nz)
    a = O.seeded_psi(8, 1, nx * ny * nz)
    b = O.seeded_psi(9, 1, nx * ny * nz)
    Ha = O.hamiltonian(grid, V, tab, a, 1)
    Hb = O.hamiltonian(grid, V, tab, b, 1)
    lhs, rhs = float(np.dot(b.ravel(), Ha.ravel())), float(np.dot(Hb.ravel(), a.ravel()))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_kinetic_plane_wave_eigenvalue():
    """FD8 on exp(iG.r) is diagonal with the closed-form 8th-order symbol."""
    nx, ny, nz = 16, 12, 10
    dx, dy, dz = 0.3, 0.35, 0.4
    N = nx * ny * nz
    m = (3, 2, 1)
    x = np.arange(nx)[None, None, :] * dx
    y = np.arange(ny)[None, :, None] * dy
    z = np.arange(nz)[:, None, None] * dz
    G = [2 * np.pi * m[0] / (nx * dx), 2 * np.pi * m[1] / (ny * dy), 2 * np.pi * m[2] / (nz * dz)]
    f = np.cos(G[0] * x + G[1] * y + G[2] * z).ravel()
    out = np.zeros(N)
    O.laplacian8th(nx, ny, nz, out, f, 1.0, dx, dy, dz)
    w = [8064.0, -1008.0, 128.0, -9.0]

    def symbol(Gd, hd):
        return (-14350.0 + 2 * sum(w[k] * np.cos((k + 1) * Gd * hd) for k in range(4))) / (5040.0 * hd * hd)

    lam = symbol(G[0], dx) + symbol(G[1], dy) + symbol(G[2], dz)
    np.testing.assert_allclose(out, lam * f, rtol=0, atol=1e-11 * abs(lam))


def test_gth_sphere_equals_reference_cube_layout():
    """Voxel-sphere tables give the same V_NL psi as the reference's cube blocks
    (including periodic self-images: the p sphere is wider than the 6 bohr cell)."""
    if not O.ref_available():
        pytest.skip("reference oracle library not built here")
    n = 20
    h = 6.0 / n
    grid = (n, n, n, h, h, h)
    pos = O.bcc_positions(6.0, 1) + 0.1
    sp = [O.GTH_BCC] * 2
    tab = O.gth_tables(pos, sp, h, h, h)
    cube = O.gth_cube_tables(pos, sp, n, n, n, h, h, h)
    tabc = (cube["npts"], cube["widths"], cube["coords"], cube["proj"], cube["energy"])
    psi = O.seeded_psi(11, 2, n ** 3)
    a = O.nonlocal_apply(grid, tab, psi, 2)
    b = O.nonlocal_apply(grid, tabc, psi, 2)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-14
    # the sphere is wider than the cell, so folded points repeat
    c = tab[2].reshape(-1, 3)[: tab[0][0]]
    folded = (c[:, 0] % n) + n * ((c[:, 1] % n) + n * (c[:, 2] % n))
    assert len(np.unique(folded)) < len(folded)
