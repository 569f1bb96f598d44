"""Seeded golden cases shared by make_golden.py and the tests.

Each case: inputs() -> dict of arrays (regenerated from seeds), reference(inp)
-> output of the reference's own code, oracle(inp) -> output of the C
restatement, and "checked" arrays whose sums are stored as checksums.
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402

SMALL = (12, 10, 8, 0.3, 0.25, 0.35)          # non-cubic, non-tile-multiple grid
TINY = (5, 4, 6, 0.4, 0.5, 0.45)              # dimensions smaller than the stencil reach
C0_24 = (24, 24, 24, 0.25, 0.25, 0.25)        # config-0 bcc cell (a = 6 bohr) on a 24^3 grid
C0_20 = (20, 20, 20, 0.3, 0.3, 0.3)           # same cell on a 20^3 grid (complex case)
A_BCC = 6.0


def _lap_inputs(grid, seed, nb, cplx=False):
    nx, ny, nz = grid[:3]
    N = nx * ny * nz
    p = O.seeded_psi(seed, nb, N, cplx)
    out0 = O.seeded_psi(seed + 50, nb, N, cplx)        # non-zero initial out: tests "+="
    return dict(grid=grid, p=p, out0=out0, checked=[p, out0])


def _lap_ref(inp, fn):
    nx, ny, nz, dx, dy, dz = inp["grid"]
    out = inp["out0"].copy()
    fn(nx, ny, nz, out, inp["p"], -0.5, dx, dy, dz)
    return out


def _kp_ref(inp, g, fn):
    nx, ny, nz, dx, dy, dz = inp["grid"]
    out = inp["out0"].copy()
    fn(nx, ny, nz, out, inp["p"], -0.5, dx, dy, dz, g)
    return out


def _ham_inputs(grid, seed, nb, cplx):
    nx, ny, nz, dx, dy, dz = grid
    N = nx * ny * nz
    pos = O.bcc_positions(A_BCC, 1) + np.array([0.11, -0.07, 0.05])   # off-grid atoms
    sp = [O.GTH_BCC] * len(pos)
    psi = O.seeded_psi(seed, nb, N, cplx)
    V = O.seeded_potential(seed, N)
    return dict(grid=grid, pos=pos, sp=sp, psi=psi, V=V, nb=nb, checked=[psi, V])


def _ham_ref(inp, cplx, g):
    nx, ny, nz, dx, dy, dz = inp["grid"]
    cube = O.gth_cube_tables(inp["pos"], inp["sp"], nx, ny, nz, dx, dy, dz)
    return O.ref_hamiltonian(inp["grid"], inp["V"], cube, inp["psi"], inp["nb"], cplx, g)


def _ham_oracle(inp, cplx, g):
    nx, ny, nz, dx, dy, dz = inp["grid"]
    tab = O.gth_tables(inp["pos"], inp["sp"], dx, dy, dz)
    return O.hamiltonian(inp["grid"], inp["V"], tab, inp["psi"], inp["nb"], cplx, g)


def _fft_inputs(grid, seed, nb, cplx):
    N = grid[0] * grid[1] * grid[2]
    psi = O.seeded_psi(seed, nb, N, cplx)
    V = O.seeded_potential(seed, N)
    return dict(grid=grid, psi=psi, V=V, nb=nb, checked=[psi, V])


def _fft_ref(inp, cplx, ks, ki):
    return O.ref_hamiltonian_fft(inp["grid"], inp["V"], inp["psi"], inp["nb"], cplx, ks, ki)


def _fft_oracle(inp, cplx, ks, ki):
    g = O.kpoint_vector(inp["grid"], ks, ki)
    nb, N = inp["nb"], inp["V"].size
    vpsi = (inp["psi"].reshape(-1, N) * inp["V"][None, :]).reshape(inp["psi"].shape)
    return O.kinetic_fft(inp["grid"], inp["psi"], nb, cplx, g) + vpsi


GGA_GRID = (20, 18, 16, 0.3, 0.33, 0.375)


def gga_density(grid=GGA_GRID):
    """A smooth positive periodic density with three points below the GGA cut."""
    nx, ny, nz, dx, dy, dz = grid
    x, y, z = np.arange(nx) * dx, np.arange(ny) * dy, np.arange(nz) * dz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    L = (nx * dx, ny * dy, nz * dz)
    rho = 0.02 + 0.3 * np.exp(np.cos(2 * np.pi * X / L[0]) + np.sin(2 * np.pi * Y / L[1]) * np.cos(4 * np.pi * Z / L[2]))
    rho[0, 0, :3] = 1e-9
    return rho.ravel()


def _gga_inputs():
    rho = gga_density()
    return dict(grid=GGA_GRID, rho=rho, checked=[rho])


def _gga_ref(inp):
    import scf_oracle as S
    v, ex, ec = S.ref_gga_pbe(inp["grid"], inp["rho"])
    return np.concatenate([v, [ex, ec]])


def _gga_oracle(inp):
    import scf_oracle as S
    _, v, ex, ec = S.gga_pbe(inp["grid"], inp["rho"])
    return np.concatenate([v, [ex, ec]])


HARTREE_ODD = (15, 12, 9, 0.4, 0.5, 0.6)


def _hartree_inputs(grid, seed):
    nx, ny, nz = grid[:3]
    rho = gga_density(grid) if seed is None else np.random.default_rng(seed).uniform(0.0, 1.0, nx * ny * nz)
    return dict(grid=grid, rho=rho, checked=[rho])


def _hartree_ref(inp):
    import scf_oracle as S
    return S.ref_hartree(inp["grid"], inp["rho"], 2)


def _hartree_oracle(inp):
    import scf_oracle as S
    return S.hartree(inp["rho"], inp["grid"])[0]


# the FFT-kinetic cases: k-point sampling and index of each (the reference's k)
FFT_GRID_EVEN = (24, 20, 16, 0.25, 0.3, 0.375)
FFT_GRID_ODD = (15, 12, 9, 0.4, 0.5, 0.6)
FFT_KPT = {"ham_fft_real_c0": ((1, 1, 1), (0, 0, 0)),
           "ham_fft_kpt_even": ((2, 4, 2), (1, -1, 1)),
           "ham_fft_kpt_odd": ((4, 3, 2), (1, 2, 1))}

G_KP = (0.3, 0.0, -0.2)
G_SMALL = (1.0e-9, 0.4, 0.1)    # |gx| below the 1e-8 dispatch threshold
G_C0 = (2 * math.pi / A_BCC * 0.25, 2 * math.pi / A_BCC * 0.5, 0.0)

CASES = {
    "lap_real_small": dict(inputs=lambda: _lap_inputs(SMALL, 0, 2),
                           reference=lambda i: _lap_ref(i, O.ref_laplacian8th),
                           oracle=lambda i: _lap_ref(i, O.laplacian8th)),
    "lap_real_tiny": dict(inputs=lambda: _lap_inputs(TINY, 3, 1),
                          reference=lambda i: _lap_ref(i, O.ref_laplacian8th),
                          oracle=lambda i: _lap_ref(i, O.laplacian8th)),
    "lap_kpoint_small": dict(inputs=lambda: _lap_inputs(SMALL, 1, 2, True),
                             reference=lambda i: _kp_ref(i, G_KP, O.ref_laplacian_kpoint8th),
                             oracle=lambda i: _kp_ref(i, G_KP, O.laplacian_kpoint8th)),
    "lap_kpoint_thresh": dict(inputs=lambda: _lap_inputs(SMALL, 2, 1, True),
                              reference=lambda i: _kp_ref(i, G_SMALL, O.ref_laplacian_kpoint8th),
                              oracle=lambda i: _kp_ref(i, G_SMALL, O.laplacian_kpoint8th)),
    "lap_kpoint_gamma": dict(inputs=lambda: _lap_inputs(TINY, 4, 1, True),
                             reference=lambda i: _kp_ref(i, (0.0, 0.0, 0.0), O.ref_laplacian_kpoint8th),
                             oracle=lambda i: _kp_ref(i, (0.0, 0.0, 0.0), O.laplacian_kpoint8th)),
    "ham_real_c0": dict(inputs=lambda: _ham_inputs(C0_24, 0, 3, False),
                        reference=lambda i: _ham_ref(i, False, (0.0, 0.0, 0.0)),
                        oracle=lambda i: _ham_oracle(i, False, (0.0, 0.0, 0.0))),
    "ham_cplx_c0": dict(inputs=lambda: _ham_inputs(C0_20, 5, 2, True),
                        reference=lambda i: _ham_ref(i, True, G_C0),
                        oracle=lambda i: _ham_oracle(i, True, G_C0)),
    # FFT kinetic + V (the reference's default operator, run by its own code)
    "ham_fft_real_c0": dict(inputs=lambda: _fft_inputs(C0_24, 7, 3, False),
                            reference=lambda i: _fft_ref(i, False, *FFT_KPT["ham_fft_real_c0"]),
                            oracle=lambda i: _fft_oracle(i, False, *FFT_KPT["ham_fft_real_c0"])),
    "ham_fft_kpt_even": dict(inputs=lambda: _fft_inputs(FFT_GRID_EVEN, 8, 3, True),
                             reference=lambda i: _fft_ref(i, True, *FFT_KPT["ham_fft_kpt_even"]),
                             oracle=lambda i: _fft_oracle(i, True, *FFT_KPT["ham_fft_kpt_even"])),
    # GGA-PBE exchange-correlation: V_xc on the grid, then E_x, E_c (the reference's own mSetPotentialVxc)
    "gga_pbe": dict(inputs=_gga_inputs, reference=_gga_ref, oracle=_gga_oracle),
    # Hartree potential: the reference's mSetPotentialVhart (Poisson on its 2x high-resolution grid)
    "hartree_even": dict(inputs=lambda: _hartree_inputs(GGA_GRID, None), reference=_hartree_ref,
                         oracle=_hartree_oracle),
    "hartree_odd": dict(inputs=lambda: _hartree_inputs(HARTREE_ODD, 13), reference=_hartree_ref,
                        oracle=_hartree_oracle),
    "ham_fft_kpt_odd": dict(inputs=lambda: _fft_inputs(FFT_GRID_ODD, 9, 2, True),
                            reference=lambda i: _fft_ref(i, True, *FFT_KPT["ham_fft_kpt_odd"]),
                            oracle=lambda i: _fft_oracle(i, True, *FFT_KPT["ham_fft_kpt_odd"])),
}


# ---------------------------------------------------------------------------
# LOBPCG: the reference's solvers on the reference Hamiltonian, 12^3 bcc cell
# ---------------------------------------------------------------------------
EIG_GRID = (12, 12, 12, 0.5, 0.5, 0.5)
EIG_NB = 8
EIG_G = (2 * math.pi / A_BCC * 0.25, 2 * math.pi / A_BCC * 0.5, 0.0)


def eig_inputs(seed=0, cplx=False):
    nx, ny, nz, dx, dy, dz = EIG_GRID
    N = nx * ny * nz
    dV = dx * dy * dz
    pos = O.bcc_positions(A_BCC, 1) + 0.1
    sp = [O.GTH_BCC] * len(pos)
    V = 0.3 * O.seeded_potential(seed, N)
    X = O.orthonormal_psi(seed, EIG_NB, N, dV, cplx)
    return dict(grid=EIG_GRID, pos=pos, sp=sp, V=V, X=X, dV=dV, checked=[V, X])


def eig_ref_z(inp, calls=3, iter_max=4, g=EIG_G):
    """Sequence of Eigen_z_multi_mpi calls (SCF steps 0..calls-1): eigenvalues after each."""
    nx, ny, nz, dx, dy, dz = inp["grid"]
    cube = O.gth_cube_tables(inp["pos"], inp["sp"], nx, ny, nz, dx, dy, dz)
    X = inp["X"].copy()
    keep = np.zeros_like(X)
    ev = np.zeros(EIG_NB)
    out, nf = [], 0
    for step in range(calls):
        nf = O.ref_lobpcg_z(inp["grid"], inp["V"], cube, X, keep, EIG_NB, iter_max, ev, nf, 1e-4, step, g)
        out.append(np.concatenate([ev, [nf]]))
    return np.array(out)


def eig_ref_d(inp, calls=3, iter_max=4):
    nx, ny, nz, dx, dy, dz = inp["grid"]
    cube = O.gth_cube_tables(inp["pos"], inp["sp"], nx, ny, nz, dx, dy, dz)
    X = inp["X"].copy()
    keep = np.zeros_like(X)
    ev = np.zeros(EIG_NB)
    out = []
    for step in range(calls):
        O.ref_lobpcg_d(inp["grid"], inp["V"], cube, X, keep, EIG_NB, iter_max, ev, step == 0)
        out.append(ev.copy())
    return np.array(out)


def eig_exact(inp, cplx, g=EIG_G):
    nx, ny, nz, dx, dy, dz = inp["grid"]
    tab = O.gth_tables(inp["pos"], inp["sp"], dx, dy, dz)
    return O.dense_eigenvalues(inp["grid"], inp["V"], tab, EIG_NB, cplx, g if cplx else (0.0, 0.0, 0.0))


CASES.update({
    "lobpcg_z_ref": dict(inputs=lambda: eig_inputs(0, True), reference=eig_ref_z, oracle=None),
    "lobpcg_d_ref": dict(inputs=lambda: eig_inputs(0, False), reference=eig_ref_d, oracle=None),
    "eig_exact_z": dict(inputs=lambda: eig_inputs(0, True), reference=lambda i: eig_exact(i, True), oracle=None),
    "eig_exact_d": dict(inputs=lambda: eig_inputs(0, False), reference=lambda i: eig_exact(i, False), oracle=None),
})


# SCF of config 0: 2-atom bcc (a = 6 bohr), 32^3 grid (h = 0.1875), GTH
# (Z 6, r_loc 0.45, C1 -4, C2 0.6; s + p projectors), LDA, 16 bands, 12
# electrons, Fermi 0.01 Ha, 4 LOBPCG iterations per step, Kerker (q0 0.8
# bohr^-1, A 0.5) + DIIS depth 6, |dE| < 1e-6 Ha / atom.
SCF_C0 = dict(n=32, a=A_BCC, nb=16, n_el=12.0, seed=0,
              params=dict(kbt=0.01, lobpcg_iters=4, max_steps=60, tol_per_atom=1e-6, amplitude=0.5, q0=0.8,
                          depth=6))


def scf_inputs():
    n, a = SCF_C0["n"], SCF_C0["a"]
    h = a / n
    grid = (n, n, n, h, h, h)
    pos = O.bcc_positions(a, 1)
    sp = [dict(O.GTH_BCC)] * len(pos)
    X = O.orthonormal_psi(SCF_C0["seed"], SCF_C0["nb"], n ** 3, h ** 3)
    return dict(grid=grid, pos=pos, sp=sp, X=X, checked=[X, pos])


# ---------------------------------------------------------------------------
# Shapes of the larger configurations, pinned to the reference's own solvers:
#   C4K: one k-point of config 4's k part -- the config-0 cell (a = 6 bohr) on a
#        48^3 grid (h = 0.125), 24 complex bands, k = (1, 2, 3) / 4 of the
#        reciprocal vectors (a point of the 4 x 4 x 4 Gamma-centred mesh);
#   C0D: config 0's real shape -- 32^3 grid, 16 bands.
# Potentials are the seeded V of the other LOBPCG cases (0.3 U[-1, 1]), atoms
# off-grid, GTH s + p projectors (cutoff 6 r_l).
# ---------------------------------------------------------------------------
C4K_GRID = (48, 48, 48, 0.125, 0.125, 0.125)
C4K_NB = 24
C4K_G = tuple(2 * math.pi / A_BCC * f for f in (0.25, 0.5, 0.75))
C0D_GRID = (32, 32, 32, 0.1875, 0.1875, 0.1875)
C0D_NB = 16


def big_eig_inputs(grid, nb, seed, cplx):
    nx, ny, nz, dx, dy, dz = grid
    N = nx * ny * nz
    dV = dx * dy * dz
    pos = O.bcc_positions(A_BCC, 1) + np.array([0.11, -0.07, 0.05])
    sp = [O.GTH_BCC] * len(pos)
    V = 0.3 * O.seeded_potential(seed, N)
    X = O.orthonormal_psi(seed, nb, N, dV, cplx)
    return dict(grid=grid, pos=pos, sp=sp, V=V, X=X, dV=dV, nb=nb, checked=[V, X])


def big_eig_ref(inp, cplx, calls=3, iter_max=4, g=(0.0, 0.0, 0.0)):
    """Reference solver calls (SCF steps 0..calls-1): eigenvalues (and num_fix) after each."""
    nx, ny, nz, dx, dy, dz = inp["grid"]
    nb = inp["nb"]
    cube = O.gth_cube_tables(inp["pos"], inp["sp"], nx, ny, nz, dx, dy, dz)
    X = inp["X"].copy()
    keep = np.zeros_like(X)
    ev = np.zeros(nb)
    out, nf = [], 0
    for step in range(calls):
        if cplx:
            nf = O.ref_lobpcg_z(inp["grid"], inp["V"], cube, X, keep, nb, iter_max, ev, nf, 1e-4, step, g)
            out.append(np.concatenate([ev, [nf]]))
        else:
            O.ref_lobpcg_d(inp["grid"], inp["V"], cube, X, keep, nb, iter_max, ev, step == 0)
            out.append(ev.copy())
    return np.array(out)


CASES.update({
    "lobpcg_z_c4k": dict(inputs=lambda: big_eig_inputs(C4K_GRID, C4K_NB, 4, True),
                         reference=lambda i: big_eig_ref(i, True, g=C4K_G), oracle=None),
    "lobpcg_d_c0": dict(inputs=lambda: big_eig_inputs(C0D_GRID, C0D_NB, 0, False),
                        reference=lambda i: big_eig_ref(i, False), oracle=None),
    "ham_cplx_c4k": dict(inputs=lambda: _ham_inputs(C4K_GRID, 6, 1, True),
                         reference=lambda i: _ham_ref(i, True, C4K_G),
                         oracle=lambda i: _ham_oracle(i, True, C4K_G)),
})


# k-point SCF: the config-0 cell (2-atom bcc, a = 6 bohr) on a 20^3 grid, the
# 2 x 2 x 2 Gamma-centred k mesh (8 points, weight 1/8 each, no symmetry
# reduction), 10 complex bands per k-point, 12 electrons, GTH as config 0, LDA,
# Fermi 0.01 Ha, 4 LOBPCG iterations per step, Kerker-DIIS, |dE| < 1e-6 Ha / atom.
SCF_KPT = dict(n=20, a=A_BCC, nb=10, n_el=12.0,
               params=dict(kbt=0.01, lobpcg_iters=4, max_steps=60, tol_per_atom=1e-6, amplitude=0.5, q0=0.8,
                           depth=6))


def scf_kpt_inputs():
    n, a = SCF_KPT["n"], SCF_KPT["a"]
    h = a / n
    grid = (n, n, n, h, h, h)
    pos = O.bcc_positions(a, 1) + np.array([0.05, -0.03, 0.02])
    sp = [dict(O.GTH_BCC)] * len(pos)
    b = 2 * math.pi / a
    kvecs = np.array([[i * b / 2, j * b / 2, k * b / 2] for i in range(2) for j in range(2) for k in range(2)])
    weights = np.full(len(kvecs), 1.0 / len(kvecs))
    Xs = [O.orthonormal_psi(10 + k, SCF_KPT["nb"], n ** 3, h ** 3, True) for k in range(len(kvecs))]
    return dict(grid=grid, pos=pos, sp=sp, kvecs=kvecs, weights=weights, Xs=Xs, checked=Xs + [pos, kvecs])
