"""GPU checks of the nonlocal energy and forces (qsb_ham_nonlocal_energy,
qsb_ham_nonlocal_energy_force; EnergyPPnonlocal_bundle / ForceNonlocal_bundle,
source/PseudoPotNonlocal_SvF2_kpoint.h:5033-5135, :3629-3731) through the C ABI.

Tolerances: against the oracle (pinned to the reference in test_forces.py)
1e-12 relative in FP64 and 2e-5 relative in FP32; against central finite
differences of the library's own energies (delta = 1e-3 bohr, cutoff 9 r_l)
the stated bar 1e-5 Ha/bohr, and 1e-6 relative after Richardson extrapolation."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _setup(qsb, n, pos, rcut=O.RCUT_FACTOR, a=6.0):
    h = a / n
    H = qsb.Hamiltonian(n, n, n, h, h, h)
    H.set_potential(O.seeded_potential(3, n ** 3))
    H.set_gth_projectors(pos, [0] * len(pos), [2], [O.GTH_BCC["r"]], [O.GTH_BCC["h"]], rcut)
    return H, (n, n, n, h, h, h)


@pytest.mark.parametrize("cplx,g", [(False, (0.0, 0.0, 0.0)), (True, (0.3, 0.2, -0.1))])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_energy_force_match_oracle(qsb, cplx, g, dtype):
    import torch
    n, nb = 24, 5
    pos = O.bcc_positions(6.0, 1) + np.array([0.07, -0.03, 0.11])
    H, grid = _setup(qsb, n, pos)
    sps = [dict(O.GTH_BCC)] * len(pos)
    tables = O.gth_tables(pos, sps, *grid[3:])
    dbeta = O.gth_gradient_tables(pos, sps, *grid[3:], tables)
    psi = O.seeded_psi(9, nb, n ** 3, cplx)
    occ = np.array([2.0, 2.0, 1.2, 0.6, 0.0])
    e_o, f_o = O.nonlocal_energy_force(grid, tables, dbeta, psi, nb, occ, cplx, g)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    P = torch.from_numpy(psi).to(tdt).cuda()
    e, f = H.nonlocal_energy_force(P, occ, len(pos), cplx, g)
    e_only = H.nonlocal_energy(P, occ, cplx, g)
    tol = 1e-12 if dtype == "f64" else 2e-5
    assert abs(e - e_o) <= tol * abs(e_o), (e, e_o)
    assert abs(e_only - e) <= 1e-14 * abs(e)
    np.testing.assert_allclose(f, f_o, rtol=0, atol=tol * np.abs(f_o).max())
    assert qsb.device_status() == 0


def test_user_gradient_tables_equal_the_gth_path(qsb):
    """Point-list projectors with caller-supplied gradients give the same
    energy and forces as qsb_ham_set_gth_projectors (which builds both)."""
    import torch
    n, nb = 20, 3
    pos = O.bcc_positions(6.0, 1) + 0.05
    H, grid = _setup(qsb, n, pos)
    sps = [dict(O.GTH_BCC)] * len(pos)
    tables = O.gth_tables(pos, sps, *grid[3:])
    H2 = qsb.Hamiltonian(n, n, n, *grid[3:])
    H2.set_projectors(*tables)
    P = torch.from_numpy(O.seeded_psi(4, nb, n ** 3, False)).cuda()
    occ = np.array([2.0, 2.0, 1.0])
    with pytest.raises(qsb.QsbError) as err:            # forces need gradients
        H2.nonlocal_energy_force(P, occ, len(pos))
    assert err.value.status == 4
    H2.set_projector_gradients(O.gth_gradient_tables(pos, sps, *grid[3:], tables))
    e1, f1 = H.nonlocal_energy_force(P, occ, len(pos))
    e2, f2 = H2.nonlocal_energy_force(P, occ, len(pos))
    assert abs(e1 - e2) <= 1e-13 * abs(e1)
    np.testing.assert_allclose(f2, f1, rtol=0, atol=1e-13 * np.abs(f1).max())


@pytest.mark.parametrize("cplx,g", [(False, (0.0, 0.0, 0.0)), (True, (0.25, -0.4, 0.1))])
def test_forces_are_minus_the_energy_gradient(qsb, cplx, g):
    """End to end on the device: analytic projector gradients contracted with
    the adjoint of the projection against finite differences of the energy,
    the atoms moved through qsb_ham_set_gth_projectors."""
    import torch
    n, nb, rcut, delta = 20, 2, 9.0, 1e-3
    pos = O.bcc_positions(6.0, 1) + np.array([0.07, -0.03, 0.11])
    psi = torch.from_numpy(O.seeded_psi(7, nb, n ** 3, cplx)).cuda()
    occ = np.array([2.0, 1.0])
    H, grid = _setup(qsb, n, pos, rcut)
    _, f = H.nonlocal_energy_force(psi, occ, len(pos), cplx, g)

    def energy(p):
        H.set_gth_projectors(p, [0] * len(p), [2], [O.GTH_BCC["r"]], [O.GTH_BCC["h"]], rcut)
        return H.nonlocal_energy(psi, occ, cplx, g)

    def central(d):
        fd = np.zeros_like(f)
        for a in range(len(pos)):
            for k in range(3):
                p1, p2 = pos.copy(), pos.copy()
                p1[a, k] += d
                p2[a, k] -= d
                fd[a, k] = -(energy(p1) - energy(p2)) / (2 * d)
        return fd

    fd1, fd2 = central(delta), central(delta / 2)
    assert np.abs(f).max() > 1e-2
    np.testing.assert_allclose(f, fd1, rtol=0, atol=1e-5)
    np.testing.assert_allclose(f, (4 * fd2 - fd1) / 3, rtol=0, atol=1e-6 * np.abs(f).max())
    assert qsb.device_status() == 0
