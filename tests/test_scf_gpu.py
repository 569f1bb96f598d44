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
