"""CPU oracle of the self-consistent-field loop (test infrastructure only).

Gamma point, spin-unpolarised, LDA (Perdew-Zunger), analytic GTH local part,
Fermi-Dirac occupations, Kerker-preconditioned DIIS density mixing, and the
reference's own real LOBPCG (EigenLOBPCG_d_multi through oracle/_ref) as the
eigensolver.  The step order is QUMASUN_KPOINT::Execute's
(source/qumasun_kpoint.scfloop.h:61-230): eigensolver -> occupations ->
density -> mixing -> potentials -> energy -> |dE| test.

Pinned pieces: lda_pz against the reference's Calc_XC_LDA (source/Vxc.h:43-75)
and fermi_occupations against its SetOccupancy (source/SetOccupancy.h:7-18)
with the bisection of mSetOccupancyTemperature
(source/qumasun_base1.occupancy.h:76-170), both compiled from the reference
sources into oracle/_ref; the loop refines the bisection's mu by Newton steps
to the exact electron count (fermi_occupations_exact).  Restated from the mathematics (no reference
counterpart on this path): the GTH local potential in G space, the FFT Poisson
solve, the Kerker-preconditioned DIIS mixer and the Kohn-Sham energy of the
output density; SCF-level parity with the reference is therefore unpinned
(its local potential goes through core charges and a Poisson solve on a finer
grid, source/qumasun_base1.core.h), and the device SCF is checked against
this oracle.
"""
import contextlib
import math
import ctypes
import os
import sys

import numpy as np

import oracle as O

_C2 = (3.0 / (4.0 * np.pi)) ** (1.0 / 3.0)
_C3 = -(3.0 / (4.0 * np.pi)) * (9.0 * np.pi / 4.0) ** (1.0 / 3.0)


def lda_pz(rho):
    """(rho * eps_xc, v_xc) of the Perdew-Zunger LDA, zero below rho = 1e-8
    (Calc_XC_LDA, source/Vxc.h:43-75; PZ81 parameters of calc_LSDA_ge1/_lt1)."""
    rho = np.asarray(rho, np.float64)
    exc = np.zeros_like(rho)
    vxc = np.zeros_like(rho)
    m = rho >= 1.0e-8
    r = rho[m]
    rs = _C2 / np.cbrt(r)
    ex = _C3 / rs
    ec = np.empty_like(rs)
    ndec = np.empty_like(rs)
    ge = rs >= 1.0
    s = np.sqrt(rs[ge])
    g, b1, b2 = -0.1423, 1.0529, 0.3334
    ec[ge] = g / (1.0 + b1 * s + b2 * rs[ge])
    ndec[ge] = ec[ge] * ec[ge] * (b1 * 0.5 * s + b2 * rs[ge]) / (3.0 * g)
    lt = ~ge
    A, B, C, D = 0.0311, -0.0480, 0.0020, -0.0116
    lr = np.log(rs[lt])
    ec[lt] = B + A * lr + D * rs[lt] + C * rs[lt] * lr
    ndec[lt] = -(A + (D + C) * rs[lt] + C * rs[lt] * lr) / 3.0
    exc[m] = r * ex + r * ec
    vxc[m] = (ex + ex / 3.0) + (ec + ndec)
    return exc, vxc


def _fd8_d1(f, axis, h):
    """Eighth-order central first derivative along a numpy axis (periodic),
    GridGradient8th.h:23-26,65: c4 (f+4 - f-4) + c3 (..) + c2 (..) + c1 (..)."""
    c = {4: -3.0 / (840.0 * h), 3: 32.0 / (840.0 * h), 2: -168.0 / (840.0 * h), 1: 672.0 / (840.0 * h)}
    out = None
    for m in (4, 3, 2, 1):
        t = c[m] * (np.roll(f, -m, axis=axis) - np.roll(f, m, axis=axis))
        out = t if out is None else out + t
    return out


def gga_pbe(grid, rho):
    """Spin-unpolarised GGA-PBE as the reference's mSetPotentialVxc forms it
    (source/qumasun_base1.potential.h:383-470, 585-640, XC_IMPLE_VER2):
    exchange on rho_s = rho / 2 per spin channel (GGA_PBE::Potential_X_test3,
    source/xc_gga_pbe.h:326-356), correlation on rho (EnergyDensityPotential_C_test3
    :525-594 with LDA_PW92 :7-76 at zeta = 0), FD8 gradients and divergences.
    Returns (exc energy density, vxc, E_x, E_c); grid = (nx, ny, nz, dx, dy, dz),
    rho with x fastest."""
    nx, ny, nz, dx, dy, dz = grid
    r = np.asarray(rho, np.float64).reshape(nz, ny, nx)
    rs_ = r / 2.0
    hs = (dz, dy, dx)
    g = [_fd8_d1(rs_, ax, hs[ax]) for ax in (2, 1, 0)]          # d/dx, d/dy, d/dz
    kappa, mu, beta, gamma = 0.804, 0.21951, 0.066725, 0.031091
    cut = 1.0e-8
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        # exchange
        s2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2]
        r13 = np.cbrt(rs_)
        r43 = r13 * rs_
        c6 = np.cbrt(6.0 / math.pi)
        c62 = (6.0 * math.pi) / c6
        qm = 4.0 * c62 * r43 * r43
        q = s2 / qm
        den = 1.0 + q * mu / kappa
        F = 1.0 + kappa - kappa / den
        dF = mu / (den * den)
        dq = -(8.0 / 3.0) * q / rs_
        okx = rs_ >= cut
        ex = np.where(okx, -(3.0 / 4.0) * c6 * r43 * F, 0.0)
        vx = np.where(okx, -c6 * (r13 * F + (3.0 / 4.0) * r43 * dF * dq), 0.0)
        px = np.where(okx, -(3.0 / 4.0) * c6 * r43 * dF * (1.0 / qm), 0.0)
        # correlation
        G = [2.0 * gi for gi in g]
        s2c = G[0] * G[0] + G[1] * G[1] + G[2] * G[2]
        A, al, b1, b2, b3, b4 = 0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294
        rsw = np.cbrt(3.0 / (4.0 * math.pi * r))
        sq = np.sqrt(rsw)
        mother = 2.0 * A * (b1 * sq + b2 * rsw + b3 * rsw * sq + b4 * rsw * rsw)
        lnt = np.log(1.0 + 1.0 / mother)
        el = -2.0 * A * (1.0 + al * rsw) * lnt
        dmo = 2.0 * A * (b1 / (2.0 * sq) + b2 + (3.0 / 2.0) * b3 * sq + 2.0 * b4 * rsw)
        dln = -dmo / ((mother + 1.0) * mother)
        de = -2.0 * A * (al * lnt + (1.0 + al * rsw) * dln)
        vl = el - (1.0 / 3.0) * rsw * de
        ee = np.exp(-el / gamma)
        alpha = ee - 1.0
        C = (beta / gamma) * np.cbrt(math.pi / 3.0) / 16.0
        cr = np.cbrt(r)
        Y = C * s2c
        r73 = r * r * cr
        B = alpha * r73
        BeY = np.maximum(B + ee * Y, 1e-30)
        BY = np.maximum(B + Y, 1e-30)
        lg = np.log(BeY / BY)
        H = gamma * lg
        dexp = np.where(0.5 * r < cut, 0.0, -(ee / gamma) * (vl - el) / r)
        dB = (7.0 / 3.0) * alpha * cr * r + r73 * dexp
        vH = H + r * gamma * ((-alpha * Y / (BeY * BY)) * dB + Y / BeY * dexp)
        okc = r >= cut
        ec = np.where(okc, el + H, 0.0)
        vc = np.where(okc, vl + vH, 0.0)
        pc = np.where(okc, r * gamma * (alpha * B / (BeY * BY)) * C, 0.0)
    dV = dx * dy * dz
    E_x = 2.0 * float(np.sum(ex)) * dV
    E_c = float(np.sum(r * ec)) * dV
    vxc = vx + vc
    for ax, gi in zip((2, 1, 0), g):
        vxc = vxc - _fd8_d1((2.0 * px + 4.0 * pc) * gi, ax, hs[ax])
    exc = 2.0 * ex + r * ec
    return exc.ravel(), vxc.ravel(), E_x, E_c


def ref_gga_pbe(grid, rho):
    """The reference's own GGA branch of mSetPotentialVxc on its QUMASUN_BASE1
    object (oracle/_ref/libqsref_fft.so): (vxc, E_x, E_c)."""
    nx, ny, nz, dx, dy, dz = grid
    lib = ctypes.CDLL(O.LIB_REF_FFT)
    rho = np.ascontiguousarray(rho, np.float64)
    vxc = np.zeros_like(rho)
    e = np.zeros(2)
    dp = ctypes.POINTER(ctypes.c_double)
    with contextlib.redirect_stdout(None):
        rc = lib.qsref_gga_pbe(nx, ny, nz, ctypes.c_double(nx * dx), ctypes.c_double(ny * dy), ctypes.c_double(nz * dz),
                               rho.ctypes.data_as(dp), vxc.ctypes.data_as(dp), e.ctypes.data_as(dp))
    assert rc == 0
    return vxc, float(e[0]), float(e[1])


def ref_hartree(grid, rho, hr=2):
    """The reference's own Hartree potential (QUMASUN_BASE1::mSetPotentialVhart on its
    object in oracle/_ref/libqsref_fft.so; high-resolution ratio hr, the
    reference's default 2)."""
    nx, ny, nz, dx, dy, dz = grid
    lib = ctypes.CDLL(O.LIB_REF_FFT)
    rho = np.ascontiguousarray(rho, np.float64)
    vh = np.zeros_like(rho)
    dp = ctypes.POINTER(ctypes.c_double)
    rc = lib.qsref_hartree(nx, ny, nz, ctypes.c_double(nx * dx), ctypes.c_double(ny * dy), ctypes.c_double(nz * dz),
                           int(hr), rho.ctypes.data_as(dp), vh.ctypes.data_as(dp))
    assert rc == 0
    return vh


def ref_lda_pz(rho):
    """The reference's Calc_XC_LDA, compiled from its sources."""
    lib = O.ref_lib()
    rho = np.ascontiguousarray(rho, np.float64)
    exc = np.zeros_like(rho)
    vxc = np.zeros_like(rho)
    lib.qsref_lda_pz(rho.size, O._d(rho), O._d(exc), O._d(vxc))
    return exc, vxc


def _occupancy(eig, mu, kbt, weight):
    # SetOccupancy (source/SetOccupancy.h:7-18): coef / (exp(min(beta (e - mu), 80)) + 1)
    p = np.minimum((eig - mu) / kbt, 80.0)
    return weight / (np.exp(p) + 1.0)


def fermi_occupations(eig, n_el, kbt, weight=2.0, occupancy=_occupancy):
    """Occupations at the chemical potential found by the bisection of
    mSetOccupancyTemperature (source/qumasun_base1.occupancy.h:76-170): mu in
    [min eig, max eig], halved until the bracket is below 1e-9 or the electron
    count is met exactly."""
    eig = np.asarray(eig, np.float64)
    mu_min, mu_max = float(eig.min()), float(eig.max())
    mu = 0.5 * (mu_min + mu_max)
    go = abs(mu_max - mu_min) > 1.0e-9
    occ = occupancy(eig, mu, kbt, weight)
    mu_occ = mu
    while go:
        occ = occupancy(eig, mu, kbt, weight)
        mu_occ = mu
        ne = float(np.sum(occ))
        if ne < n_el:
            mu_min = mu
        elif ne > n_el:
            mu_max = mu
        else:
            break
        mu = 0.5 * (mu_min + mu_max)
        go = abs(mu_max - mu_min) > 1.0e-9
    # the occupations are those of the last evaluated mu (as the reference leaves them)
    return occ, mu_occ


def fermi_occupations_exact(eig, n_el, kbt, weight=2.0):
    """fermi_occupations refined by Newton steps on sum f(mu) = N_e (the
    bisection's 1e-9 bracket leaves the count off by dN/dmu 1e-9, ~1e-7
    electrons at a partly filled Fermi level); the device driver's form."""
    occ, mu = fermi_occupations(eig, n_el, kbt, weight)
    eig = np.asarray(eig, np.float64)
    for _ in range(8):
        occ = _occupancy(eig, mu, kbt, weight)
        r = float(np.sum(occ)) - n_el
        dn = float(np.sum(occ * (1.0 - occ / weight))) / kbt
        if abs(r) <= 1e-14 * n_el or not dn > 1e-300:
            break
        mu -= r / dn
    return _occupancy(eig, mu, kbt, weight), mu


def ref_occupancy(eig, mu, kbt, weight):
    lib = O.ref_lib()
    lib.qsref_set_occupancy.restype = ctypes.c_double
    eig = np.ascontiguousarray(eig, np.float64)
    occ = np.zeros_like(eig)
    lib.qsref_set_occupancy(ctypes.c_double(weight), ctypes.c_double(kbt), eig.size, O._d(eig), ctypes.c_double(mu),
                            O._d(occ))
    return occ


def zero_temperature_occupations(nb, n_el, weight=2.0):
    """Lowest bands filled with `weight` electrons each (mSetOccupancyZero's
    filling, source/qumasun_base1.occupancy.h:35-66), used for the initial density."""
    occ = np.zeros(nb)
    left = float(n_el)
    for n in range(nb):
        occ[n] = min(weight, left)
        left -= occ[n]
        if left <= 0.0:
            break
    return occ


def nyquist_mask(nx, ny, nz):
    """True off the Nyquist planes (k = n/2 of an even n): there G and -G are the
    same grid point and a structure-factor phase exp(-i G.R) has no real-field
    representation, so the local part leaves them out."""
    def ok(n):
        m = np.ones(n, bool)
        if n % 2 == 0:
            m[n // 2] = False
        return m
    return ok(nz)[:, None, None] & ok(ny)[None, :, None] & ok(nx)[None, None, :]


def g_squared(nx, ny, nz, dx, dy, dz):
    """|G|^2 on the FFT grid, array [z][y][x] (x fastest, as the grid layout)."""
    gx = 2.0 * np.pi * np.fft.fftfreq(nx, dx)
    gy = 2.0 * np.pi * np.fft.fftfreq(ny, dy)
    gz = 2.0 * np.pi * np.fft.fftfreq(nz, dz)
    return gz[:, None, None] ** 2 + gy[None, :, None] ** 2 + gx[None, None, :] ** 2, (gx, gy, gz)


def gth_local_potential(grid, pos, species_params):
    """V_loc(r) = sum over atoms and periodic images of the GTH local part
    v(r) = -Z/r erf(r / (sqrt(2) r_loc)) + exp(-(r/r_loc)^2 / 2) (C1 + C2 (r/r_loc)^2)
    through its Fourier series: v(G) = -4 pi Z exp(-G^2 r^2 / 2) / G^2 + (2 pi)^(3/2)
    r^3 exp(-G^2 r^2 / 2) (C1 + C2 (3 - G^2 r^2)); at G = 0 the Coulomb tail is
    neutralised by the electrons' Hartree G = 0 term and the finite remainder
    2 pi Z r^2 + (2 pi)^(3/2) r^3 (C1 + 3 C2) is kept; Nyquist planes left out
    (nyquist_mask)."""
    nx, ny, nz, dx, dy, dz = grid
    omega = nx * ny * nz * dx * dy * dz
    G2, (gx, gy, gz) = g_squared(nx, ny, nz, dx, dy, dz)
    VG = np.zeros((nz, ny, nx), np.complex128)
    nz0 = G2 > 0
    safe = np.where(nz0, G2, 1.0)
    for (X, Y, Z), sp in zip(np.asarray(pos, np.float64), species_params):
        r, zion, c1, c2 = sp["rloc"], sp["zion"], sp["c1"], sp["c2"]
        e = np.exp(-0.5 * G2 * r * r)
        coul = np.where(nz0, -4.0 * np.pi * zion * e / safe, 2.0 * np.pi * zion * r * r)
        short = (2.0 * np.pi) ** 1.5 * r ** 3 * e * (c1 + c2 * (3.0 - G2 * r * r))
        phase = np.exp(-1j * (gz[:, None, None] * Z + gy[None, :, None] * Y + gx[None, None, :] * X))
        VG += (coul + short) * phase
    VG *= nyquist_mask(nx, ny, nz) / omega
    return (np.fft.ifftn(VG) * (nx * ny * nz)).real.reshape(-1)


def gth_local_forces(rho, grid, pos, species_params):
    """F_a = -d/dR_a (dV sum_r rho(r) V_loc(r)) for V_loc = gth_local_potential:
    sum over G of G v_a(G) [sin(G.R_a) Re rho_G + cos(G.R_a) Im rho_G],
    rho_G = FFT(rho) / N (the G = 0 term carries no force; Nyquist planes out
    as in gth_local_potential)."""
    nx, ny, nz, dx, dy, dz = grid
    G2, (gx, gy, gz) = g_squared(nx, ny, nz, dx, dy, dz)
    rg = np.fft.fftn(np.asarray(rho, np.float64).reshape(nz, ny, nx)) / (nx * ny * nz)
    safe = np.where(G2 > 0, G2, 1.0)
    out = np.zeros((len(pos), 3))
    for a, ((X, Y, Z), sp) in enumerate(zip(np.asarray(pos, np.float64), species_params)):
        r, zion, c1, c2 = sp["rloc"], sp["zion"], sp["c1"], sp["c2"]
        e = np.exp(-0.5 * G2 * r * r)
        v = np.where(G2 > 0, -4.0 * np.pi * zion * e / safe, 0.0) + (2.0 * np.pi) ** 1.5 * r ** 3 * e * (
            c1 + c2 * (3.0 - G2 * r * r))
        v = np.where((G2 > 0) & nyquist_mask(nx, ny, nz), v, 0.0)
        th = gz[:, None, None] * Z + gy[None, :, None] * Y + gx[None, None, :] * X
        t = v * (np.sin(th) * rg.real + np.cos(th) * rg.imag)
        out[a] = [float(np.sum(gx[None, None, :] * t)), float(np.sum(gy[None, :, None] * t)),
                  float(np.sum(gz[:, None, None] * t))]
    return out


def hartree(rho, grid):
    """V_H solving lap V_H = -4 pi rho (G = 0 removed) through the FFT, and
    E_H = 1/2 int V_H rho."""
    nx, ny, nz, dx, dy, dz = grid
    G2, _ = g_squared(nx, ny, nz, dx, dy, dz)
    rg = np.fft.fftn(np.asarray(rho, np.float64).reshape(nz, ny, nx))
    vg = np.where(G2 > 0, 4.0 * np.pi * rg / np.where(G2 > 0, G2, 1.0), 0.0)
    vh = np.fft.ifftn(vg).real.reshape(-1)
    return vh, 0.5 * float(np.dot(vh, rho)) * dx * dy * dz


def kerker(res, grid, amplitude, q0):
    """A G^2 / (G^2 + q0^2) applied to a density residual (G = 0 removed)."""
    nx, ny, nz, dx, dy, dz = grid
    G2, _ = g_squared(nx, ny, nz, dx, dy, dz)
    rg = np.fft.fftn(np.asarray(res, np.float64).reshape(nz, ny, nx))
    rg *= amplitude * G2 / (G2 + q0 * q0)
    return np.fft.ifftn(rg).real.reshape(-1)


class KerkerDIIS:
    """Pulay (DIIS) density mixing with a Kerker preconditioner.

    History of (rho_in_i, R_i = rho_out_i - rho_in_i) over the last `depth`
    steps; coefficients a (sum a = 1) minimise |sum a_i R_i|^2 (grid inner
    product), solved as the bordered system [B 1; 1 0][a; l] = [0; 1] with B
    scaled by its largest diagonal; the next input density is
    sum a_i rho_in_i + P[sum a_i R_i], P = Kerker(amplitude, q0).  The
    reference's MixingDIIS (source/mixing_DIIS.h) is the unpreconditioned form
    of the same bordered system."""

    def __init__(self, grid, amplitude, q0, depth):
        self.grid, self.A, self.q0, self.depth = grid, amplitude, q0, depth
        self.rin, self.res = [], []

    def coefficients(self):
        m = len(self.res)
        B = np.array([[float(np.dot(a, b)) for b in self.res] for a in self.res])
        s = max(float(np.max(np.diag(B))), 1e-300)
        M = np.zeros((m + 1, m + 1))
        M[:m, :m] = B / s
        M[:m, m] = 1.0
        M[m, :m] = 1.0
        rhs = np.zeros(m + 1)
        rhs[m] = 1.0
        return solve_bordered(M, rhs)[:m]

    def next(self, rho_in, rho_out):
        self.rin.append(np.array(rho_in, np.float64))
        self.res.append(np.asarray(rho_out, np.float64) - rho_in)
        if len(self.res) > self.depth:
            self.rin.pop(0)
            self.res.pop(0)
        a = self.coefficients()
        rin = sum(ai * r for ai, r in zip(a, self.rin))
        res = sum(ai * r for ai, r in zip(a, self.res))
        return rin + kerker(res, self.grid, self.A, self.q0)


def solve_bordered(M, rhs):
    """Gaussian elimination with partial pivoting (the device driver's host
    solve, restated so both sides take the same steps)."""
    M = np.array(M, np.float64)
    b = np.array(rhs, np.float64)
    n = len(b)
    for k in range(n):
        p = k + int(np.argmax(np.abs(M[k:, k])))
        if p != k:
            M[[k, p]] = M[[p, k]]
            b[[k, p]] = b[[p, k]]
        if M[k, k] == 0.0:
            continue
        for i in range(k + 1, n):
            f = M[i, k] / M[k, k]
            M[i, k:] -= f * M[k, k:]
            b[i] -= f * b[k]
    x = np.zeros(n)
    for i in range(n - 1, -1, -1):
        x[i] = (b[i] - np.dot(M[i, i + 1:], x[i + 1:])) / M[i, i] if M[i, i] != 0.0 else 0.0
    return x


@contextlib.contextmanager
def _quiet_stdout():
    """The reference's LOBPCG prints per band and iteration (printf); route the
    process's stdout to /dev/null meanwhile."""
    sys.stdout.flush()
    saved = os.dup(1)
    null = os.open(os.devnull, os.O_WRONLY)
    try:
        os.dup2(null, 1)
        yield
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(null)


def density(X, occ, N):
    """rho = sum_n occ_n psi_n^2 (SetDensityOne, source/qumasun_SetDensityOne.h),
    psi normalised as int |psi|^2 dV = 1."""
    X = np.asarray(X).reshape(len(occ), N)
    return np.einsum("n,ni->i", np.asarray(occ, np.float64), X * X)


def xc_of(grid, rho, xc):
    """(energy density, v_xc) of the LDA-PZ (xc "lda") or the GGA-PBE ("pbe")."""
    if xc == "pbe":
        exc, vxc, _, _ = gga_pbe(grid, rho)
        return exc, vxc
    return lda_pz(rho)


def scf(grid, pos, species_params, nb, n_el, X0, kbt=0.01, lobpcg_iters=4, max_steps=60, tol_per_atom=1e-6,
        amplitude=0.5, q0=0.8, depth=6, rcut_factor=O.RCUT_FACTOR, xc="lda"):
    """The oracle SCF.  Returns a dict with the per-step total energies,
    final Rayleigh quotients, occupations, density and wavefunctions.
    xc: "lda" (PZ) or "pbe" (GGA-PBE, gga_pbe)."""
    nx, ny, nz, dx, dy, dz = grid
    N = nx * ny * nz
    dV = dx * dy * dz
    n_atoms = len(pos)
    tables = O.gth_tables(pos, species_params, dx, dy, dz, rcut_factor=rcut_factor)
    cube = O.gth_cube_tables(pos, species_params, nx, ny, nz, dx, dy, dz, rcut_factor=rcut_factor)
    vloc = gth_local_potential(grid, pos, species_params)
    X = np.array(X0, np.float64).reshape(nb, N).copy()
    keep = np.zeros_like(X)
    ev = np.zeros(nb)
    rho_in = density(X, zero_temperature_occupations(nb, n_el), N)
    mixer = KerkerDIIS(grid, amplitude, q0, depth)
    energies, e_prev = [], None
    for step in range(max_steps):
        vh, _ = hartree(rho_in, grid)
        _, vxc = xc_of(grid, rho_in, xc)
        veff = vloc + vh + vxc
        with _quiet_stdout():
            O.ref_lobpcg_d(grid, veff, cube, X, keep, nb, lobpcg_iters, ev, step == 0)
        HX = O.hamiltonian(grid, veff, tables, X, nb).reshape(nb, N)
        rq = np.einsum("ni,ni->n", X, HX) / np.einsum("ni,ni->n", X, X)
        occ, mu = fermi_occupations_exact(rq, n_el, kbt)
        rho_out = density(X, occ, N)
        vh_out, eh = hartree(rho_out, grid)
        exc_out, _ = xc_of(grid, rho_out, xc)
        etot = float(np.dot(occ, rq)) - float(np.dot(vh + vxc, rho_out)) * dV + eh + float(np.sum(exc_out)) * dV
        energies.append(etot)
        done = e_prev is not None and abs(etot - e_prev) / n_atoms < tol_per_atom
        e_prev = etot
        if done:
            break
        rho_in = mixer.next(rho_in, rho_out)
    return dict(energies=np.array(energies), rq=rq, occ=occ, mu=mu, rho=rho_out, X=X, vloc=vloc, steps=len(energies),
                converged=done)


def ewald(pos, charge, cell, alpha=None, tol=1e-16):
    """Ewald energy and forces of point charges in an orthorhombic periodic cell
    with a neutralising background (the ion-ion term that goes with the G-space
    GTH local part, whose Coulomb tail -Z/r is that of a point charge):
    E = 1/2 sum' Z_a Z_b erfc(alpha r)/r + (2 pi/Omega) sum_{G!=0} exp(-G^2/4alpha^2)/G^2 |S(G)|^2
        - alpha/sqrt(pi) sum Z^2 - pi/(2 Omega alpha^2) (sum Z)^2,  S(G) = sum Z e^{iG.R}.
    Restated from the mathematics (the reference forms nucleus-nucleus terms from
    core charges on its finer grid, source/qumasun_base1.energy.h)."""
    from math import erfc, sqrt, pi, exp
    pos = np.asarray(pos, np.float64)
    Z = np.asarray(charge, np.float64)
    L = np.asarray(cell, np.float64)
    omega = float(np.prod(L))
    if alpha is None:
        alpha = 5.0 / float(L.min())
    rc = sqrt(-np.log(tol)) / alpha
    gc = 2.0 * alpha * sqrt(-np.log(tol))
    na = len(pos)
    E = 0.0
    F = np.zeros((na, 3))
    nimg = [int(np.ceil(rc / L[d])) + 1 for d in range(3)]
    for a in range(na):
        for b in range(na):
            d0 = pos[a] - pos[b]
            for i in range(-nimg[0], nimg[0] + 1):
                for j in range(-nimg[1], nimg[1] + 1):
                    for k in range(-nimg[2], nimg[2] + 1):
                        if a == b and i == 0 and j == 0 and k == 0:
                            continue
                        d = d0 + np.array([i, j, k]) * L
                        r = sqrt(float(d @ d))
                        if r > rc:
                            continue
                        E += 0.5 * Z[a] * Z[b] * erfc(alpha * r) / r
                        g = Z[a] * Z[b] * (erfc(alpha * r) / r + 2 * alpha / sqrt(pi) * exp(-alpha * alpha * r * r)) / (r * r)
                        F[a] += g * d
    m = [int(np.ceil(gc * L[d] / (2 * pi))) for d in range(3)]
    for i in range(-m[0], m[0] + 1):
        for j in range(-m[1], m[1] + 1):
            for k in range(-m[2], m[2] + 1):
                if i == 0 and j == 0 and k == 0:
                    continue
                G = 2 * pi * np.array([i / L[0], j / L[1], k / L[2]])
                g2 = float(G @ G)
                if g2 > gc * gc:
                    continue
                w = exp(-g2 / (4 * alpha * alpha)) / g2
                ph = pos @ G
                S = np.sum(Z * np.exp(1j * ph))
                E += 2 * pi / omega * w * abs(S) ** 2
                F += (4 * pi / omega * w * Z * np.imag(np.conj(S) * np.exp(1j * ph)))[:, None] * G[None, :]
    E += -alpha / sqrt(pi) * float(np.sum(Z * Z)) - pi / (2 * omega * alpha * alpha) * float(np.sum(Z)) ** 2
    return E, F


# --------------------------------------------------------------------------
# k-point SCF (complex Bloch bands): the loop of QUMASUN_KPOINT::Execute over k
# groups with the reference's own Eigen_z_multi_mpi (oracle/_ref) per k-point
# --------------------------------------------------------------------------
def fermi_occupancy_kpoints(eig, kweights, n_el, kbt):
    """mSetOccupancyTemperature over k groups (source/qumasun_base1.occupancy.h:76-170):
    occupancy_nk = SetOccupancy(2 w_k, ...) with one mu for all k, bisection on
    sum_nk occupancy_nk = N_e between the lowest and highest level, then Newton
    steps to the exact count (the device driver's refinement).  eig [n_k, nb];
    returns (occupancy [n_k, nb] including the weight, mu)."""
    eig = np.asarray(eig, np.float64)
    w = np.asarray(kweights, np.float64)[:, None] * np.ones_like(eig)

    def count(mu):
        occ = np.stack([_occupancy(eig[k], mu, kbt, 2.0 * w[k, 0]) for k in range(eig.shape[0])])
        return occ, float(occ.sum())
    mu_min, mu_max = float(eig.min()), float(eig.max())
    mu = 0.5 * (mu_min + mu_max)
    go = abs(mu_max - mu_min) > 1.0e-9
    mu_last = mu
    while go:
        occ, ne = count(mu)
        mu_last = mu
        if ne < n_el:
            mu_min = mu
        elif ne > n_el:
            mu_max = mu
        else:
            break
        mu = 0.5 * (mu_min + mu_max)
        go = abs(mu_max - mu_min) > 1.0e-9
    mu = mu_last
    for _ in range(8):
        occ, ne = count(mu)
        f = occ / w
        dn = float(np.sum(w * f * (1.0 - 0.5 * f))) / kbt
        r = ne - n_el
        if abs(r) <= 1e-14 * n_el or not dn > 1e-300:
            break
        mu -= r / dn
    return count(mu)[0], mu


def scf_kpoints(grid, pos, species_params, nb, n_el, X0s, kvecs, kweights, kbt=0.01, lobpcg_iters=4, max_steps=60,
                tol_per_atom=1e-6, amplitude=0.5, q0=0.8, depth=6, rcut_factor=O.RCUT_FACTOR):
    """The oracle k-point SCF: per step and k-point the reference's
    Eigen_z_multi_mpi (no soft locking), FP64 Rayleigh quotients of the complex
    bands with the restated H, occupations over all k (fermi_occupancy_kpoints),
    rho_out = sum_nk occupancy |psi|^2, the energy and the Kerker-DIIS mixing of
    the Gamma-point oracle."""
    nx, ny, nz, dx, dy, dz = grid
    N = nx * ny * nz
    dV = dx * dy * dz
    n_atoms = len(pos)
    nk = len(kweights)
    tables = O.gth_tables(pos, species_params, dx, dy, dz, rcut_factor=rcut_factor)
    cube = O.gth_cube_tables(pos, species_params, nx, ny, nz, dx, dy, dz, rcut_factor=rcut_factor)
    vloc = gth_local_potential(grid, pos, species_params)
    Xs = [np.array(x, np.float64).reshape(2 * nb, N).copy() for x in X0s]
    keeps = [np.zeros_like(x) for x in Xs]
    evs = [np.zeros(nb) for _ in range(nk)]
    f0 = zero_temperature_occupations(nb, n_el)

    def dens(Xk, occk):
        re, im = Xk[0::2], Xk[1::2]
        return np.einsum("n,ni->i", occk, re * re + im * im)

    rho_in = sum(dens(Xs[k], kweights[k] * f0) for k in range(nk))
    mixer = KerkerDIIS(grid, amplitude, q0, depth)
    energies, e_prev = [], None
    rq = np.zeros((nk, nb))
    occ = np.zeros((nk, nb))
    for step in range(max_steps):
        vh, _ = hartree(rho_in, grid)
        _, vxc = lda_pz(rho_in)
        veff = vloc + vh + vxc
        for k in range(nk):
            with _quiet_stdout():
                O.ref_lobpcg_z(grid, veff, cube, Xs[k], keeps[k], nb, lobpcg_iters, evs[k], 0, 0.0, step,
                               tuple(kvecs[k]))
            HX = O.hamiltonian(grid, veff, tables, Xs[k], nb, True, tuple(kvecs[k])).reshape(2 * nb, N)
            num = np.einsum("ni,ni->n", Xs[k], HX)
            den = np.einsum("ni,ni->n", Xs[k], Xs[k])
            rq[k] = (num[0::2] + num[1::2]) / (den[0::2] + den[1::2])
        occ, mu = fermi_occupancy_kpoints(rq, kweights, n_el, kbt)
        rho_out = sum(dens(Xs[k], occ[k]) for k in range(nk))
        vh_out, eh = hartree(rho_out, grid)
        exc_out, _ = lda_pz(rho_out)
        etot = float(np.sum(occ * rq)) - float(np.dot(vh + vxc, rho_out)) * dV + eh + float(np.sum(exc_out)) * dV
        energies.append(etot)
        if e_prev is not None and abs(etot - e_prev) / n_atoms < tol_per_atom:
            break
        e_prev = etot
        rho_in = mixer.next(rho_in, rho_out)
    return dict(energies=np.array(energies), rq=rq, occ=occ, rho=rho_out, steps=len(energies))
