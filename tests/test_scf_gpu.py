"""GPU checks of the device SCF (qsb_scf_*, qsb_density, qsb_lda_pz) through
the C ABI against the SCF oracle (oracle/scf_oracle.py; fixture
tests/golden/scf_c0.npz made by tests/golden/make_golden.py with the
reference's own LOBPCG as its eigensolver).

Config 0: 2-atom bcc, 32^3, 16 bands, 12 electrons, LDA, Fermi 0.01 Ha, 4
LOBPCG iterations per step, Kerker-DIIS, |dE| < 1e-6 Ha / atom.

Tolerances: LDA and density 1e-13 relative; V_loc 1e-12 of its range (cuFFT
vs numpy FFT); the FP64 SCF trajectory follows the oracle's within 1e-6 Ha per
step over the first 8 steps (the device LOBPCG follows the reference's to 1e-7
per call) and ends within 1e-6 Ha / atom of it; converged to |dE| < 1e-8 Ha /
atom, the mixed-precision SCF's energy is within 1e-6 Ha / atom of the FP64
device SCF's (the stated total-energy bar), its occupied band energies within
5e-5 Ha."""
import os

import numpy as np
import pytest

import oracle as O
import scf_oracle as S
from cases import SCF_C0, scf_inputs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _scf(qsb, precision, tol=None, max_steps=None):
    import torch
    inp = scf_inputs()
    nx, ny, nz, dx, dy, dz = inp["grid"]
    N = nx * ny * nz
    H = qsb.Hamiltonian(nx, ny, nz, dx, dy, dz)
    sp = inp["sp"][0]
    H.set_gth_projectors(inp["pos"], [0] * len(inp["pos"]), [sp["nl"]], [sp["r"]], [sp["h"]], O.RCUT_FACTOR)
    H.set_potential(np.zeros(N))
    es = qsb.EigenSolver(N, SCF_C0["nb"], False, precision)
    scf = qsb.SCF(H, es, SCF_C0["nb"], SCF_C0["n_el"])
    scf.set_gth_local(inp["pos"], [0] * len(inp["pos"]), [sp["zion"]], [sp["rloc"]], [sp["c1"]], [sp["c2"]])
    p = SCF_C0["params"]
    scf.set_mixing(p["amplitude"], p["q0"], p["depth"])
    scf.set_smearing(p["kbt"])
    X = torch.from_numpy(inp["X"].copy()).cuda()
    keep = torch.zeros_like(X)
    e, ev, occ = scf.run(X, keep, p["lobpcg_iters"], max_steps or p["max_steps"], tol or p["tol_per_atom"])
    return dict(H=H, es=es, scf=scf, e=e, ev=ev, occ=occ, X=X, inp=inp)


def test_lda_and_density_match_oracle(qsb):
    import torch
    rng = np.random.default_rng(5)
    rho = np.concatenate([np.logspace(-10, 2, 5000), [0.0, 1e-8]])
    exc, vxc = qsb.lda_pz(torch.from_numpy(rho).cuda())
    e_o, v_o = S.lda_pz(rho)
    np.testing.assert_allclose(exc.cpu().numpy(), e_o, rtol=1e-13, atol=0)
    np.testing.assert_allclose(vxc.cpu().numpy(), v_o, rtol=1e-13, atol=0)
    X = rng.uniform(-0.5, 0.5, (7, 3000))
    occ = np.array([2.0, 2.0, 1.5, 1.0, 0.5, 0.01, 0.0])
    rho_d = qsb.density(torch.from_numpy(X).cuda(), occ, 3000).cpu().numpy()
    np.testing.assert_allclose(rho_d, S.density(X, occ, 3000), rtol=1e-13, atol=0)


def test_fp64_scf_follows_the_oracle(qsb):
    r = _scf(qsb, "fp64")
    gold = np.load(os.path.join(GOLD, "scf_c0.npz"))
    ge = gold["energies"]
    vloc = r["scf"].field(1).cpu().numpy()
    assert np.abs(vloc - gold["vloc"]).max() <= 1e-12 * np.abs(gold["vloc"]).max()
    k = min(8, len(ge), len(r["e"]))
    np.testing.assert_allclose(r["e"][:k], ge[:k], rtol=0, atol=1e-6)
    n_atoms = len(r["inp"]["pos"])
    assert abs(r["e"][-1] - ge[-1]) / n_atoms < 1e-6, (r["e"][-1], ge[-1])
    assert abs(len(r["e"]) - len(ge)) <= 4, (len(r["e"]), len(ge))
    assert abs(r["occ"].sum() - SCF_C0["n_el"]) < 1e-6
    t = r["scf"].step_seconds()
    assert len(t) == len(r["e"]) and np.all(t > 0)
    rho = r["scf"].field(0).cpu().numpy()
    dV = (SCF_C0["a"] / SCF_C0["n"]) ** 3
    assert np.abs(rho - gold["rho"]).sum() * dV / SCF_C0["n_el"] < 1e-3
    assert qsb.device_status() == 0


def test_mixed_scf_reaches_the_fp64_energy(qsb):
    # both converged to |dE| < 1e-8 Ha / atom: the stopping rule at 1e-6 alone
    # leaves each run ~1e-6 from its own fixed point
    r64 = _scf(qsb, "fp64", 1e-8, 100)
    r32 = _scf(qsb, "mixed", 1e-8, 100)
    n_atoms = len(r64["inp"]["pos"])
    assert abs(r64["e"][-1] - r64["e"][-2]) / n_atoms < 1e-8
    assert abs(r32["e"][-1] - r64["e"][-1]) / n_atoms < 1e-6, (r32["e"][-1], r64["e"][-1])
    # band energies are first order in the remaining density error (the total
    # energy second order)
    occ_n = int(SCF_C0["n_el"] // 2)
    np.testing.assert_allclose(r32["ev"][:occ_n], r64["ev"][:occ_n], rtol=0, atol=5e-5)
    assert qsb.device_status() == 0


def _bcc(qsb, pos, X0=None):
    """Config 0's cell (2-atom bcc, 32^3, 16 bands, 12 electrons, Fermi 0.01 Ha)
    with displaced atoms, converged to |dE| < 1e-11 Ha / atom and
    int |rho_out - rho_in| / N_e < 1e-10; projector cutoff 9 r_l so that no
    projector value jumps at the sphere edge when an atom moves."""
    import torch
    n, a = SCF_C0["n"], SCF_C0["a"]
    h = a / n
    N = n ** 3
    sp = O.GTH_BCC
    H = qsb.Hamiltonian(n, n, n, h, h, h)
    H.set_gth_projectors(pos, [0, 0], [sp["nl"]], [sp["r"]], [sp["h"]], 9.0)
    H.set_potential(np.zeros(N))
    es = qsb.EigenSolver(N, 16, False, "fp64")
    scf = qsb.SCF(H, es, 16, 12.0)
    scf.set_gth_local(pos, [0, 0], [sp["zion"]], [sp["rloc"]], [sp["c1"]], [sp["c2"]])
    scf.set_density_tolerance(1e-10)
    X = torch.from_numpy(O.orthonormal_psi(0, 16, N, h ** 3)).cuda() if X0 is None else X0.clone()
    keep = torch.zeros_like(X)
    e, ev, occ = scf.run(X, keep, 4, 300, 1e-11)
    return dict(H=H, es=es, scf=scf, e=e, ev=ev, occ=occ, X=X)


def _ts(occ, kbt=0.01):
    """kBT S of spin-paired Fermi-Dirac occupations (S = -2 sum f ln f + (1-f) ln(1-f), f = occ / 2)."""
    f = np.clip(np.asarray(occ) / 2.0, 1e-300, 1.0 - 1e-16)
    return kbt * 2.0 * float(np.sum(-(f * np.log(f) + (1.0 - f) * np.log1p(-f))))


def test_forces_are_minus_the_free_energy_gradient(qsb):
    """Adjoint forces (local part from the output density, qsb_scf_local_forces;
    nonlocal part from the projections on the analytic projector gradients,
    qsb_ham_nonlocal_energy_force) against central differences (delta = 1e-3
    bohr) of the converged SCF free energy F = E - kBT S (the variational
    functional with Fermi smearing; the cell's Fermi level sits in a partly
    filled triplet): every component within 1e-6 Ha / bohr (the stated bar is
    1e-5), and within 1e-8 after Richardson extrapolation from delta / 2."""
    pos = O.bcc_positions(SCF_C0["a"], 1) + np.array([[0.13, -0.07, 0.21], [-0.11, 0.05, 0.02]])
    r0 = _bcc(qsb, pos)
    assert 0.01 < _ts(r0["occ"])                                # smearing matters here (kBT S ~ 0.04 Ha)
    f = r0["scf"].local_forces() + np.asarray(r0["H"].nonlocal_energy_force(r0["X"], r0["occ"], 2)[1]).reshape(2, 3)
    assert np.abs(f).max() > 0.05
    for at in range(2):
        for k in range(3):
            fds = []
            for d in (1e-3, 5e-4):
                fe = []
                for sgn in (1.0, -1.0):
                    p = pos.copy()
                    p[at, k] += sgn * d
                    r = _bcc(qsb, p, r0["X"])
                    fe.append(r["e"][-1] - _ts(r["occ"]))
                fds.append(-(fe[0] - fe[1]) / (2 * d))
            assert abs(f[at, k] - fds[0]) < 1e-6, (at, k, f[at, k], fds[0])
            assert abs(f[at, k] - (4 * fds[1] - fds[0]) / 3) < 1e-8, (at, k, f[at, k], fds)
    assert qsb.device_status() == 0


def test_local_forces_match_the_oracle_on_a_molecule(qsb):
    """Config 1 (O + 2 H in a 20 bohr box, 112^3): the device local force on the
    converged SCF density equals the oracle's to 1e-10 relative (Nyquist planes
    left out by both)."""
    import torch
    n, L = 112, 20.0
    h = L / n
    N = n ** 3
    pos = np.array([[0.0, 0.0, 0.0], [1.43, 1.11, 0.0], [-1.43, 1.11, 0.0]])
    pos = pos + np.random.default_rng(1).normal(0.0, 0.05, pos.shape)
    H = qsb.Hamiltonian(n, n, n, h, h, h)
    H.set_gth_projectors(pos, [0, 1, 1], [1, 0], [[O.GTH_O["r"][0], 0.0], [0.0, 0.0]],
                         [[O.GTH_O["h"][0], 0.0], [0.0, 0.0]], 9.0)
    H.set_potential(np.zeros(N))
    es = qsb.EigenSolver(N, 8, False, "fp64")
    scf = qsb.SCF(H, es, 8, 8.0)
    sps = [O.GTH_O, O.GTH_H]
    scf.set_gth_local(pos, [0, 1, 1], [s["zion"] for s in sps], [s["rloc"] for s in sps], [s["c1"] for s in sps],
                      [s["c2"] for s in sps])
    X = torch.from_numpy(O.orthonormal_psi(1, 8, N, h ** 3)).cuda()
    e, ev, occ = scf.run(X, torch.zeros_like(X), 4, 200, 1e-8)
    rho = scf.field(0)
    f = scf.local_forces()
    f_o = S.gth_local_forces(rho.cpu().numpy(), (n, n, n, h, h, h), pos, [O.GTH_O, O.GTH_H, O.GTH_H])
    np.testing.assert_allclose(f, f_o, rtol=0, atol=1e-10 * np.abs(f_o).max())
    assert np.abs(f).max() > 0.1


def test_lbfgs_relaxes_the_molecule(qsb):
    """Config 1 relaxed by qsb_relax_lbfgs (free energy E - kBT S + Ewald; forces
    local + nonlocal + Ewald) to max |F| < 1e-4 Ha / bohr: the energy never
    rises by more than the SCF noise, the returned forces equal the ones
    assembled afresh at the returned geometry from the parts (1e-6), and the
    two O-H bonds come out equal (the molecule's mirror symmetry; the grid
    breaks it only by its egg-box ripple, 1e-2 bohr)."""
    import torch
    n, L = 112, 20.0
    h = L / n
    N = n ** 3
    pos = np.array([[0.0, 0.0, 0.0], [1.43, 1.11, 0.0], [-1.43, 1.11, 0.0]])
    pos = pos + np.random.default_rng(1).normal(0.0, 0.05, pos.shape) + L / 2
    sps = [O.GTH_O, O.GTH_H]
    species = [0, 1, 1]
    proj = ([1, 0], [[O.GTH_O["r"][0], 0.0], [0.0, 0.0]], [[O.GTH_O["h"][0], 0.0], [0.0, 0.0]], 9.0)
    local = ([s["zion"] for s in sps], [s["rloc"] for s in sps], [s["c1"] for s in sps], [s["c2"] for s in sps])
    H = qsb.Hamiltonian(n, n, n, h, h, h)
    H.set_gth_projectors(pos, species, *proj)
    H.set_potential(np.zeros(N))
    es = qsb.EigenSolver(N, 8, False, "fp64")
    scf = qsb.SCF(H, es, 8, 8.0)
    scf.set_gth_local(pos, species, *local)
    scf.set_density_tolerance(1e-7)
    X = torch.from_numpy(O.orthonormal_psi(1, 8, N, h ** 3)).cuda()
    keep = torch.zeros_like(X)
    p, e, f = scf.relax(X, keep, pos, species, proj, local, scf_tol=1e-9, max_iter=40, fmax=1e-4)
    assert np.linalg.norm(f, axis=1).max() < 1e-4, f
    assert len(e) >= 3 and e[-1] < e[0] - 1e-3
    assert np.all(np.diff(e) < 10 * 1e-9 * 3 + 1e-12), np.diff(e)
    # forces afresh from the parts at the returned geometry (states and density of the last evaluation)
    e_run, ev, occ = scf.run(X, keep, 4, 200, 1e-9)
    f2 = scf.local_forces() + np.asarray(H.nonlocal_energy_force(X, occ, 3)[1]).reshape(3, 3)
    f2 += qsb.ewald(p, [6.0, 1.0, 1.0], (L, L, L))[1]
    np.testing.assert_allclose(f2, f, rtol=0, atol=1e-6)
    b1, b2 = np.linalg.norm(p[1] - p[0]), np.linalg.norm(p[2] - p[0])
    assert abs(b1 - b2) < 1e-2, (b1, b2)
    assert qsb.device_status() == 0
