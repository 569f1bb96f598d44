"""GPU gates on the force and precision bars of the device SCF, through the C ABI.

* Config 1 (O + 2 H in a 20 bohr box, 112^3 grid, GTH O with one s projector,
  H local only, 4 occupied + 4 empty bands; atoms jittered by N(0, 0.05 bohr)
  from seed 1, projector cutoff 9 r_l): the adjoint forces (local part from the
  output density, nonlocal part from the projector-gradient projections, Ewald)
  against central differences (delta = 1e-3 bohr) of the converged SCF free
  energy F = E - kBT S + E_ewald, every component within 1e-5 Ha / bohr, and
  against their Richardson extrapolation from delta / 2 within 1e-6.  The LDA
  is Perdew-Zunger with the high-density correlation branch made continuous
  at rs = 1 (qsb_scf_set_xc variant 1): with the published constants (the
  reference's Calc_XC_LDA) eps_c jumps by 3.2e-5 Ha there, every grid point
  whose density crosses 3 / (4 pi) as O moves steps the converged energy by
  (3 / 4 pi) dV 3.2e-5 = 4.36e-8 Ha, and central differences of the O in-plane
  force scatter by 2e-5 to 9e-5 Ha / bohr while the adjoint forces stay the
  exact derivative of every position-dependent term.  Both
  sides need the density converged: the Hellmann-Feynman forces carry the
  remaining density error to first order, the energy only to second, so each
  SCF here runs to int |rho_out - rho_in| / N_e < 1e-10 and |dE| < 1e-11 Ha / atom.
* Mixed precision (FP32 H.psi, INT8-Ozaki Gram, FP64 pencil) with its FP64 polish
  (qsb_scf_set_polish) against the FP64 drop-in on a displaced 16-atom bcc cell
  (2x2x2 of the a = 6 bohr cell, 96^3, 128 bands, atoms displaced N(0, 0.1 bohr)
  from seed 2), both converged to |dE| < 1e-9 Ha / atom and a density
  residual below 1e-9 (the stopping error of either run stays below the
  comparison): forces on every atom within 1e-5 Ha / bohr, occupied band
  energies within 1e-6 Ha, energy within 1e-6 Ha / atom."""
import math

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _ts(occ, kbt=0.01):
    """kBT S of spin-paired Fermi-Dirac occupations (S = -2 sum f ln f + (1-f) ln(1-f), f = occ / 2)."""
    f = np.clip(np.asarray(occ) / 2.0, 1e-300, 1.0 - 1e-16)
    return kbt * 2.0 * float(np.sum(-(f * np.log(f) + (1.0 - f) * np.log1p(-f))))


WATER_L, WATER_N = 20.0, 112
# Projector spheres of 9 r_l: at 6 r_l the GTH s projector of O still has
# exp(-18) of its peak at the sphere edge, and grid points entering or leaving
# the sphere as the atom moves step the energy by ~1e-9 Ha each (measured: the
# O central differences at delta = 1e-3 move by ~1e-6 Ha / bohr between 6 and
# 9 r_l); at 9 r_l the edge value is exp(-40.5).
WATER_RCUT = 9.0
WATER_SPECIES = [0, 1, 1]
WATER_ZION = [O.GTH_O["zion"], O.GTH_H["zion"], O.GTH_H["zion"]]


def _water_positions():
    pos = np.array([[0.0, 0.0, 0.0], [1.43, 1.11, 0.0], [-1.43, 1.11, 0.0]])
    return pos + np.random.default_rng(1).normal(0.0, 0.05, pos.shape) + WATER_L / 2


def _water(qsb, pos, X0=None, pz_variant=1):
    import torch
    n, L = WATER_N, WATER_L
    h = L / n
    N = n ** 3
    sps = [O.GTH_O, O.GTH_H]
    H = qsb.Hamiltonian(n, n, n, h, h, h)
    H.set_gth_projectors(pos, WATER_SPECIES, [1, 0], [[O.GTH_O["r"][0], 0.0], [0.0, 0.0]],
                         [[O.GTH_O["h"][0], 0.0], [0.0, 0.0]], WATER_RCUT)
    H.set_potential(np.zeros(N))
    es = qsb.EigenSolver(N, 8, False, "fp64")
    scf = qsb.SCF(H, es, 8, 8.0)
    scf.set_gth_local(pos, WATER_SPECIES, [s["zion"] for s in sps], [s["rloc"] for s in sps],
                      [s["c1"] for s in sps], [s["c2"] for s in sps])
    scf.set_density_tolerance(1e-10)
    scf.set_xc(pz_variant)
    X = torch.from_numpy(O.orthonormal_psi(1, 8, N, h ** 3)).cuda() if X0 is None else X0.clone()
    keep = torch.zeros_like(X)
    e, ev, occ = scf.run(X, keep, 4, 400, 1e-11)
    assert len(e) < 400, "SCF did not converge"
    ee, fe = qsb.ewald(pos, WATER_ZION, (L, L, L))
    F = e[-1] - _ts(occ) + ee
    return dict(H=H, es=es, scf=scf, e=e, occ=occ, X=X, F=F, ewald_f=fe)


def test_config1_adjoint_forces_match_central_differences(qsb):
    pos = _water_positions()
    r0 = _water(qsb, pos)
    f = (r0["scf"].local_forces() + np.asarray(r0["H"].nonlocal_energy_force(r0["X"], r0["occ"], 3)[1]).reshape(3, 3)
         + r0["ewald_f"])
    assert np.abs(f).max() > 0.02                      # a jittered, unrelaxed molecule
    fd = {}
    for d in (1e-3, 5e-4):
        fd[d] = np.zeros((3, 3))
        for at in range(3):
            for k in range(3):
                fe = []
                for sgn in (1.0, -1.0):
                    p = pos.copy()
                    p[at, k] += sgn * d
                    fe.append(_water(qsb, p, r0["X"])["F"])
                fd[d][at, k] = -(fe[0] - fe[1]) / (2 * d)
    rich = (4 * fd[5e-4] - fd[1e-3]) / 3
    print("adjoint forces\n", f)
    for d, v in fd.items():
        print("central differences, delta", d, "\n", v, "\n|difference|\n", np.abs(f - v))
    print("Richardson\n", rich, "\n|difference|\n", np.abs(f - rich))
    assert np.abs(f - rich).max() < 1e-6, np.abs(f - rich).max()
    assert np.abs(f - fd[1e-3]).max() < 1e-5, np.abs(f - fd[1e-3]).max()
    assert qsb.device_status() == 0


def _bcc16(qsb, prec, pos, X0):
    import torch
    n, a = 96, 12.0
    h = a / n
    N = n ** 3
    na = len(pos)
    sp = O.GTH_BCC
    H = qsb.Hamiltonian(n, n, n, h, h, h)
    H.set_gth_projectors(pos, [0] * na, [sp["nl"]], [sp["r"]], [sp["h"]], O.RCUT_FACTOR)
    H.set_potential(np.zeros(N))
    es = qsb.EigenSolver(N, 128, False, prec)
    scf = qsb.SCF(H, es, 128, 6.0 * na)
    scf.set_gth_local(pos, [0] * na, [sp["zion"]], [sp["rloc"]], [sp["c1"]], [sp["c2"]])
    es64 = None
    if prec == "mixed":
        es64 = qsb.EigenSolver(N, 128, False, "fp64")
        scf.set_polish(es64, 100, 1e-9, 1e-9)   # mixed loop to |dE| < 1e-8 Ha / atom, then FP64
    else:
        scf.set_density_tolerance(1e-9)
    X = X0.clone()
    keep = torch.zeros_like(X)
    e, ev, occ = scf.run(X, keep, 4, 250, 1e-8 if prec == "mixed" else 1e-9)
    res = scf.step_residuals()
    print(prec, "steps", len(e), "density residuals every 10 steps", res[::10], "last", res[-1])
    assert len(e) < 250, "SCF did not converge"
    polish = scf.polish_stats()
    f = scf.local_forces() + np.asarray(H.nonlocal_energy_force(X, occ, na)[1]).reshape(na, 3)
    out = dict(e=e, ev=ev, occ=occ, f=f, polish=polish)
    scf.close()
    es.close()
    if es64 is not None:
        es64.close()
    H.close()
    del X, keep
    torch.cuda.empty_cache()
    return out


def test_mixed_form_with_fp64_polish_meets_the_fp64_bars(qsb):
    import torch
    pos = O.bcc_positions(6.0, 2, jitter=0.1, seed=2)
    na = len(pos)
    n = 96
    N = n ** 3
    dV = (12.0 / n) ** 3
    gen = torch.Generator(device="cuda").manual_seed(2)
    psi = torch.rand(128, N, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    X0 = torch.linalg.qr(psi.t())[0].t().contiguous() / math.sqrt(dV)
    del psi
    r64 = _bcc16(qsb, "fp64", pos, X0)
    r32 = _bcc16(qsb, "mixed", pos, X0)
    first, steps = r32["polish"]
    print("steps: fp64", len(r64["e"]), "mixed", first, "+ polish", steps)
    assert first > 0 and 1 <= steps < 100, r32["polish"]
    assert abs(r32["e"][-1] - r64["e"][-1]) / na < 1e-6, (r32["e"][-1], r64["e"][-1])
    occupied = r64["occ"] > 1e-6
    ev_err = np.abs(r32["ev"] - r64["ev"])[occupied].max()
    f_err = np.abs(r32["f"] - r64["f"]).max()
    print("max |F|", np.abs(r64["f"]).max(), "force error", f_err, "eigenvalue error", ev_err)
    assert np.abs(r64["f"]).max() > 1e-3
    assert f_err < 1e-5, f_err
    assert ev_err < 1e-6, ev_err
    assert qsb.device_status() == 0
