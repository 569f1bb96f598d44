"""Local parts from radial tables in the device SCF (qsb_scf_set_radial_local),
through the C ABI: the route a UPF's local potential takes (its radius,
v_local and z_valence through qsb_radial_local_table, which the CPU tests pin
to the analytic GTH transform to 1e-9 and check on the reference's shipped
PseudoDojo files).  Here the table of a GTH local potential tabulated on a log
grid must reproduce the analytic GTH path of the same driver: V_loc on the
grid to 1e-8 Ha (of ~10 Ha), the local forces from a density to 1e-7 Ha/bohr, and the SCF
energies of both runs step by step to 1e-8 Ha / atom."""
import math

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

GTH = O.GTH_BCC
A = 6.0


def _gth_radial_table(qsb, dg, n_g, sigma):
    from scipy.special import erf
    Z, rl, c1, c2 = GTH["zion"], GTH["rloc"], GTH["c1"], GTH["c2"]
    r = np.exp(-9 + np.arange(2000) * (math.log(15.0) + 9) / 2000)
    x = r / rl
    V = -Z * erf(r / (math.sqrt(2) * rl)) / r + np.exp(-0.5 * x * x) * (c1 + c2 * x * x)
    return qsb.radial_local_table(r, V, Z, n_g, dg, sigma)


def _scf(qsb, n, nb, pos, local):
    import torch
    h = A / n
    H = qsb.Hamiltonian(n, n, n, h, h, h)
    na = len(pos)
    H.set_gth_projectors(pos, [0] * na, [GTH["nl"]], [GTH["r"]], [GTH["h"]], O.RCUT_FACTOR)
    es = qsb.EigenSolver(n ** 3, nb, False)
    es.set_hamiltonian(H)
    scf = qsb.SCF(H, es, nb, GTH["zion"] * na)
    if local == "gth":
        scf.set_gth_local(pos, [0] * na, [GTH["zion"]], [GTH["rloc"]], [GTH["c1"]], [GTH["c2"]])
    else:
        dg, sigma = 0.01, 0.45
        gmax = math.sqrt(3) * math.pi / h
        n_g = int(gmax / dg) + 8
        tab = _gth_radial_table(qsb, dg, n_g, sigma)
        scf.set_radial_local(pos, [0] * na, [GTH["zion"]], [sigma], dg, tab[None, :])
    X = torch.from_numpy(O.orthonormal_psi(5, nb, n ** 3, h ** 3)).cuda()
    return H, es, scf, X


def test_radial_table_local_parts_equal_the_analytic_gth_path(qsb):
    import torch
    n, nb = 24, 8
    pos = O.bcc_positions(A, 1) + np.array([0.11, -0.07, 0.05])
    pos[1] += np.array([0.13, 0.02, -0.09])
    runs = {}
    for local in ("gth", "table"):
        H, es, scf, X = _scf(qsb, n, nb, pos, local)
        vloc = scf.field(1).cpu().numpy()
        rho = torch.from_numpy(np.abs(O.seeded_potential(3, n ** 3)) * 0.1).cuda()
        f_rho = scf.local_forces(rho)
        keep = torch.zeros_like(X)
        e, ev, occ = scf.run(X, keep, lobpcg_iters=4, max_steps=12, tol_per_atom=1e-12)
        f_out = scf.local_forces()
        runs[local] = dict(vloc=vloc, f_rho=f_rho, e=e, ev=ev, f_out=f_out)
        scf.close()
        es.close()
        H.close()
    a, b = runs["gth"], runs["table"]
    # the table's v(G) is the analytic transform to ~1e-9 (Simpson on the log
    # grid); V_loc ~ 10 Ha on this grid
    assert np.abs(a["vloc"] - b["vloc"]).max() < 1e-8
    assert np.abs(a["f_rho"] - b["f_rho"]).max() < 1e-7
    assert len(a["e"]) == len(b["e"])
    assert np.abs(a["e"] - b["e"]).max() / len(pos) < 1e-8
    assert np.abs(a["ev"] - b["ev"]).max() < 1e-8
    assert np.abs(a["f_out"] - b["f_out"]).max() < 1e-7


def test_radial_local_rejects_a_table_that_stops_short(qsb):
    n, nb = 24, 8
    h = A / n
    pos = O.bcc_positions(A, 1)
    H = qsb.Hamiltonian(n, n, n, h, h, h)
    es = qsb.EigenSolver(n ** 3, nb, False)
    es.set_hamiltonian(H)
    scf = qsb.SCF(H, es, nb, 12.0)
    tab = _gth_radial_table(qsb, 0.02, 200, 0.45)      # ends at 4 bohr^-1, the grid reaches 21.8
    with pytest.raises(qsb.QsbError, match="table ends"):
        scf.set_radial_local(pos, [0, 0], [GTH["zion"]], [0.45], 0.02, tab[None, :])
    scf.close()
    es.close()
    H.close()
