"""Test oracle for the H.psi hot path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm may import this module; the product (libqumasun_b200.so and its binding)
never does.

It wraps two CPU libraries built by oracle/Makefile:
  * oracle/_build/libqsoracle.so — the C restatement (oracle/qsoracle.c);
  * oracle/_ref/libqsref.so      — the REFERENCE's own headers compiled from its
    source tree (oracle/ref_entry.cpp); present only where it was built.
and restates in numpy the analytic GTH projector tables (the reference has no
GTH support; the published GTH form is restated, see gth_tables) and the
seeded synthetic inputs.
"""
import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# Checkout of the reference project (its source/ and PP/ trees), read by the
# oracle/_ref build and by the CPU tests that compare with its shipped files.
# Set QSB_REFERENCE_ROOT where it lives elsewhere; absent, those tests skip.
REFERENCE_ROOT = os.environ.get("QSB_REFERENCE_ROOT", "/root/reference")
LIB_ORACLE = os.path.join(HERE, "_build", "libqsoracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libqsref.so")
LIB_REF_FFT = os.path.join(HERE, "_ref", "libqsref_fft.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


_oracle = None
_ref = None


def oracle_lib():
    """The C restatement (built on demand with make if missing)."""
    global _oracle
    if _oracle is None:
        if not os.path.exists(LIB_ORACLE):
            import subprocess
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        _oracle = ctypes.CDLL(LIB_ORACLE)
    return _oracle


def ref_available():
    return os.path.exists(LIB_REF)


def ref_lib():
    """The reference's own code (oracle/_ref/libqsref.so)."""
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(LIB_REF)
    return _ref


_ref_fft = None


def ref_fft_available():
    return os.path.exists(LIB_REF_FFT)


def ref_hamiltonian_fft(grid, V, psi, nb, is_complex=False, ksample=(1, 1, 1), kidx=(0, 0, 0)):
    """-1/2 (grad + i k)^2 psi + V psi by the reference's own FFT-kinetic
    Hamiltonian (QUMASUN_BASE1::mHamiltonianMatrix_ddm_bundle, algorithm 1,
    source/qumasun_base1.matrix.h:142-228, run on a reference object without
    nuclei: oracle/ref_fft.cpp, oracle/_ref/libqsref_fft.so), FFTW replaced by
    the DFT restated in oracle/ref_shim/fftw_dft.cpp.  k_d = kidx_d * 2 pi /
    (n_d h_d ksample_d), the reference's k-point indexing.  Real bands run as
    complex bands with zero imaginary part; the real part is returned."""
    global _ref_fft
    if _ref_fft is None:
        _ref_fft = ctypes.CDLL(LIB_REF_FFT)
        _ref_fft.qsref_ham_fft.restype = ctypes.c_int
    nx, ny, nz, dx, dy, dz = grid
    N = nx * ny * nz
    psi = np.asarray(psi, np.float64)
    if is_complex:
        z = np.ascontiguousarray(psi)
    else:
        z = np.zeros((nb, 2, N))
        z[:, 0] = psi.reshape(nb, N)
    out = np.zeros_like(z)
    ks = np.ascontiguousarray(ksample, np.int32)
    ki = np.ascontiguousarray(kidx, np.int32)
    V = np.ascontiguousarray(V, np.float64)
    rc = _ref_fft.qsref_ham_fft(nx, ny, nz, ctypes.c_double(nx * dx), ctypes.c_double(ny * dy),
                                ctypes.c_double(nz * dz), _i(ks), _i(ki), _d(V), nb, _d(z), _d(out))
    assert rc == 0, "qsref_ham_fft failed"
    if is_complex:
        return out.reshape(psi.shape)
    return np.ascontiguousarray(out.reshape(nb, 2, N)[:, 0]).reshape(psi.shape)


def kpoint_vector(grid, ksample, kidx):
    """The reference's k vector of k-point index kidx on a ksample grid:
    k_d = kidx_d * 2 pi / (L_d ksample_d) (qumasun_base1.constructor.h:34-36)."""
    nx, ny, nz, dx, dy, dz = grid
    return tuple(k * 2.0 * math.pi / (n * h * s) for k, n, h, s in zip(kidx, (nx, ny, nz), (dx, dy, dz), ksample))


# --------------------------------------------------------------------------
# configurations (BASELINE workloads), seeded inputs
# --------------------------------------------------------------------------
# GTH parameters used by the bcc cells (Z_ion = 6 element) and the water
# molecule (O, H); r_l / h_l per channel, channels s (l=0) and p (l=1).
GTH_BCC = dict(zion=6.0, rloc=0.45, c1=-4.0, c2=0.6, nl=2, r=(0.40, 0.55), h=(5.0, 1.5))
GTH_O = dict(zion=6.0, rloc=0.247, c1=-16.58, c2=2.40, nl=1, r=(0.222, 0.0), h=(18.27, 0.0))
GTH_H = dict(zion=1.0, rloc=0.2, c1=-4.18, c2=0.725, nl=0, r=(0.0, 0.0), h=(0.0, 0.0))
RCUT_FACTOR = 6.0


def bcc_positions(a, reps, jitter=0.0, seed=None):
    """bcc lattice of edge a (bohr) repeated reps^3 times; optional N(0, jitter) displacements."""
    pos = []
    for i in range(reps):
        for j in range(reps):
            for k in range(reps):
                base = np.array([i, j, k], dtype=float) * a
                pos.append(base)
                pos.append(base + 0.5 * a)
    pos = np.array(pos)
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        pos = pos + rng.normal(0.0, jitter, size=pos.shape)
    return pos


def gth_tables(pos, species_params, dx, dy, dz, rcut_factor=RCUT_FACTOR):
    """Voxel-sphere GTH projector tables in the C ABI's point-list format.

    Restates the GTH separable projector of one radial function per channel
    (Goedecker-Teter-Hutter PRB 54, 1703 (1996); HGH PRB 58, 3641 (1998)):
      p_l(r) = sqrt(2) r^l exp(-r^2/(2 r_l^2)) / (r_l^(l+3/2) sqrt(Gamma(l+3/2)))
    times real harmonics Y00 = 1/sqrt(4 pi), Y1 = sqrt(3/(4 pi)) (x, y, z)/r,
    zero beyond rcut_factor * r_l, on the points with |r - R| <= max_l rcut.
    Returns (npts, widths, coords, beta, energy) as numpy arrays.
    """
    npts, widths, coords, beta, energy = [], [], [], [], []
    for R, sp in zip(pos, species_params):
        nl = sp["nl"]
        w = (1 if nl >= 1 else 0) + (3 if nl >= 2 else 0)
        if w == 0:
            npts.append(0)
            widths.append(0)
            continue
        rl = sp["r"]
        rmax = max(rcut_factor * rl[l] for l in range(nl))
        ix = np.arange(math.floor((R[0] - rmax) / dx), math.ceil((R[0] + rmax) / dx) + 1)
        iy = np.arange(math.floor((R[1] - rmax) / dy), math.ceil((R[1] + rmax) / dy) + 1)
        iz = np.arange(math.floor((R[2] - rmax) / dz), math.ceil((R[2] + rmax) / dz) + 1)
        Z, Y, X = np.meshgrid(iz, iy, ix, indexing="ij")
        X = X.ravel(); Y = Y.ravel(); Z = Z.ravel()
        x = X * dx - R[0]; y = Y * dy - R[1]; z = Z * dz - R[2]
        r2 = x * x + y * y + z * z
        keep = r2 <= rmax * rmax
        X, Y, Z, x, y, z, r2 = X[keep], Y[keep], Z[keep], x[keep], y[keep], z[keep], r2[keep]
        r = np.sqrt(r2)
        cols = []
        pre0 = math.sqrt(2.0) / (rl[0] ** 1.5 * math.sqrt(math.sqrt(math.pi) / 2.0)) / math.sqrt(4.0 * math.pi)
        cols.append(np.where(r <= rcut_factor * rl[0], pre0 * np.exp(-r2 / (2.0 * rl[0] ** 2)), 0.0))
        en = [sp["h"][0]]
        if nl >= 2:
            pre1 = (math.sqrt(2.0) / (rl[1] ** 2.5 * math.sqrt(3.0 * math.sqrt(math.pi) / 4.0))
                    * math.sqrt(3.0 / (4.0 * math.pi)))
            e1 = np.where(r <= rcut_factor * rl[1], pre1 * np.exp(-r2 / (2.0 * rl[1] ** 2)), 0.0)
            cols += [e1 * x, e1 * y, e1 * z]
            en += [sp["h"][1]] * 3
        npts.append(len(X))
        widths.append(w)
        coords.append(np.stack([X, Y, Z], axis=1).astype(np.int32).ravel())
        beta.append(np.concatenate(cols))
        energy += en
    cat = lambda L, dt: np.ascontiguousarray(np.concatenate(L).astype(dt)) if L else np.zeros(0, dt)
    return (np.array(npts, np.int32), np.array(widths, np.int32), cat(coords, np.int32), cat(beta, np.float64),
            np.array(energy, np.float64))


def gth_gradient_columns(x, y, z, sp, rcut_factor=RCUT_FACTOR):
    """d beta_w / d(x, y, z) of the GTH projectors of gth_tables at offsets
    (x, y, z) = point - atom: grads[d][w] arrays.  Analytic derivatives:
      s:   d/dv_d exp(-r^2/(2 r0^2))      = -v_d / r0^2 * (the Gaussian)
      p_m: d/dv_d (v_m exp(-r^2/(2 r1^2))) = (delta_md - v_m v_d / r1^2) * (the Gaussian)
    (the same cutoffs as the projectors)."""
    nl, rl = sp["nl"], sp["r"]
    r2 = x * x + y * y + z * z
    r = np.sqrt(r2)
    v = (x, y, z)
    grads = [[], [], []]
    if nl >= 1:
        pre0 = math.sqrt(2.0) / (rl[0] ** 1.5 * math.sqrt(math.sqrt(math.pi) / 2.0)) / math.sqrt(4.0 * math.pi)
        b0 = np.where(r <= rcut_factor * rl[0], pre0 * np.exp(-r2 / (2.0 * rl[0] ** 2)), 0.0)
        for d in range(3):
            grads[d].append(-v[d] / rl[0] ** 2 * b0)
    if nl >= 2:
        pre1 = (math.sqrt(2.0) / (rl[1] ** 2.5 * math.sqrt(3.0 * math.sqrt(math.pi) / 4.0))
                * math.sqrt(3.0 / (4.0 * math.pi)))
        e1 = np.where(r <= rcut_factor * rl[1], pre1 * np.exp(-r2 / (2.0 * rl[1] ** 2)), 0.0)
        for m in range(3):
            for d in range(3):
                grads[d].append(e1 * ((1.0 if m == d else 0.0) - v[m] * v[d] / rl[1] ** 2))
    return grads


def gth_gradient_tables(pos, species_params, dx, dy, dz, tables, rcut_factor=RCUT_FACTOR):
    """Projector gradients for the point lists of gth_tables (same points, same
    order), in the C ABI's layout: per atom d/dx, d/dy, d/dz blocks, each
    npts x width column-major."""
    npts, widths, coords, _, _ = tables
    out, off = [], 0
    for a, (R, sp) in enumerate(zip(pos, species_params)):
        n = int(npts[a])
        if widths[a] == 0 or n == 0:
            off += n
            continue
        C = coords[3 * off: 3 * (off + n)].reshape(n, 3)
        g = gth_gradient_columns(C[:, 0] * dx - R[0], C[:, 1] * dy - R[1], C[:, 2] * dz - R[2], sp, rcut_factor)
        for d in range(3):
            out.append(np.concatenate(g[d]))
        off += n
    return np.ascontiguousarray(np.concatenate(out)) if out else np.zeros(0)


def nonlocal_energy_force(grid, tables, dbeta, psi, nb, occ, is_complex=False, g=(0.0, 0.0, 0.0)):
    """Restatement of EnergyPPnonlocal_bundle / ForceNonlocal_bundle
    (source/PseudoPotNonlocal_SvF2_kpoint.h:5033-5135, :3629-3731):
      c = dV <beta|psi>, d_k = dV <d beta/dk|psi> (qso_nonlocal_project on the
      beta and the gradient tables), E = sum occ E_w |c|^2,
      F_a,k = sum occ 2 E_w (c_re d_k,re + c_im d_k,im).
    Returns (energy, forces[n_atoms, 3])."""
    npts, widths, coords, beta, energy = tables
    c = nonlocal_project(grid, tables, psi, nb, is_complex, g)            # [ncol][P]
    d = []
    for k in range(3):
        parts = []
        off_g = 0
        for a in range(len(npts)):
            n, w = int(npts[a]), int(widths[a])
            parts.append(dbeta[off_g + k * n * w: off_g + (k + 1) * n * w])
            off_g += 3 * n * w
        tk = (npts, widths, coords, np.ascontiguousarray(np.concatenate(parts)) if parts else np.zeros(0), energy)
        d.append(nonlocal_project(grid, tk, psi, nb, is_complex, g))
    occ = np.asarray(occ, np.float64)
    occ_col = np.repeat(occ, 2) if is_complex else occ
    E = float((occ_col[:, None] * energy[None, :] * c * c).sum())
    F = np.zeros((len(npts), 3))
    p0 = 0
    for a in range(len(npts)):
        w = int(widths[a])
        sl = slice(p0, p0 + w)
        for k in range(3):
            F[a, k] = (2.0 * occ_col[:, None] * energy[None, sl] * c[:, sl] * d[k][:, sl]).sum()
        p0 += w
    return E, F


def gth_cube_tables(pos, species_params, nx, ny, nz, dx, dy, dz, rcut_factor=RCUT_FACTOR):
    """The same projectors on the reference's CUBE subgrid blocks (GetOverlapPeriodic,
    source/GridSubgrid.h:690-740), for the reference-side nonlocal.  Returns
    (cubes[6 per atom], widths, proj (block layout, column-major per atom), energy,
    point-list form (npts, coords) of the same blocks)."""
    lib = ref_lib()
    cubes, widths, proj, energy, npts, coords, grad = [], [], [], [], [], [], []
    blocks_buf = np.zeros(9 * 4096, np.int32)
    gsz = ctypes.c_int(0)
    for R, sp in zip(pos, species_params):
        nl = sp["nl"]
        w = (1 if nl >= 1 else 0) + (3 if nl >= 2 else 0)
        rl = sp["r"]
        rmax = max([rcut_factor * rl[l] for l in range(nl)] + [0.0])
        b = [math.floor((R[0] - rmax) / dx), math.floor((R[1] - rmax) / dy), math.floor((R[2] - rmax) / dz)]
        e = [math.ceil((R[0] + rmax) / dx) + 1, math.ceil((R[1] + rmax) / dy) + 1, math.ceil((R[2] + rmax) / dz) + 1]
        cube = np.array(b + e, np.int32)
        cubes.append(cube)
        nbk = lib.qsref_overlap_blocks(nx, ny, nz, _i(cube), _i(blocks_buf), 4096, ctypes.byref(gsz))
        assert nbk <= 4096
        pts = []
        for k in range(nbk):
            bx0, by0, bz0, bx1, by1, bz1, sx, sy, sz = blocks_buf[9 * k: 9 * k + 9]
            zz, yy, xx = np.meshgrid(np.arange(bz0, bz1), np.arange(by0, by1), np.arange(bx0, bx1), indexing="ij")
            pts.append(np.stack([xx.ravel() - sx, yy.ravel() - sy, zz.ravel() - sz], axis=1))
        P = np.concatenate(pts) if pts else np.zeros((0, 3), np.int64)
        assert len(P) == gsz.value
        x = P[:, 0] * dx - R[0]; y = P[:, 1] * dy - R[1]; z = P[:, 2] * dz - R[2]
        r2 = x * x + y * y + z * z
        r = np.sqrt(r2)
        cols = []
        if nl >= 1:
            pre0 = math.sqrt(2.0) / (rl[0] ** 1.5 * math.sqrt(math.sqrt(math.pi) / 2.0)) / math.sqrt(4.0 * math.pi)
            cols.append(np.where(r <= rcut_factor * rl[0], pre0 * np.exp(-r2 / (2.0 * rl[0] ** 2)), 0.0))
            energy.append(sp["h"][0])
        if nl >= 2:
            pre1 = (math.sqrt(2.0) / (rl[1] ** 2.5 * math.sqrt(3.0 * math.sqrt(math.pi) / 4.0))
                    * math.sqrt(3.0 / (4.0 * math.pi)))
            e1 = np.where(r <= rcut_factor * rl[1], pre1 * np.exp(-r2 / (2.0 * rl[1] ** 2)), 0.0)
            cols += [e1 * x, e1 * y, e1 * z]
            energy += [sp["h"][1]] * 3
        widths.append(w)
        if w:
            proj.append(np.concatenate(cols))
            gr = gth_gradient_columns(x, y, z, sp, rcut_factor)
            grad.append(np.concatenate([np.concatenate(gr[k]) for k in range(3)]))
        npts.append(len(P))
        coords.append(P.astype(np.int32).ravel())
    cat = lambda L, dt: np.ascontiguousarray(np.concatenate(L).astype(dt)) if L else np.zeros(0, dt)
    return dict(cubes=cat(cubes, np.int32), widths=np.array(widths, np.int32), proj=cat(proj, np.float64),
                energy=np.array(energy, np.float64), npts=np.array(npts, np.int32), coords=cat(coords, np.int32),
                grad=cat(grad, np.float64))


def seeded_psi(seed, nb, N, complex_=False, dtype=np.float64):
    """psi ~ U[-0.5, 0.5] from numpy PCG64(seed), layout of the reference bundle."""
    rng = np.random.default_rng(seed)
    return rng.uniform(-0.5, 0.5, size=(nb * (2 if complex_ else 1), N)).astype(dtype)


def seeded_potential(seed, N, scale=1.0):
    rng = np.random.default_rng(seed + 1000)
    return rng.uniform(-scale, scale, size=N)


# --------------------------------------------------------------------------
# C restatement wrappers
# --------------------------------------------------------------------------
def laplacian8th(nx, ny, nz, out, p, coef, dx, dy, dz):
    """out += coef * FD8 Laplacian(p) for every band row of p (restatement)."""
    lib = oracle_lib()
    N = nx * ny * nz
    p = np.ascontiguousarray(p, np.float64).reshape(-1, N)
    assert out.dtype == np.float64 and out.flags.c_contiguous
    o = out.reshape(-1, N)
    for b in range(p.shape[0]):
        lib.qso_laplacian8th(nx, ny, nz, _d(o[b]), _d(p[b]), ctypes.c_double(coef), ctypes.c_double(dx),
                             ctypes.c_double(dy), ctypes.c_double(dz))
    return out


def laplacian_kpoint8th(nx, ny, nz, out, src, coef, dx, dy, dz, g):
    lib = oracle_lib()
    N = nx * ny * nz
    s = np.ascontiguousarray(src, np.float64).reshape(-1, 2, N)
    o = out.reshape(-1, 2, N)
    for b in range(s.shape[0]):
        lib.qso_laplacian_kpoint8th(nx, ny, nz, _d(o[b, 0]), _d(o[b, 1]), _d(s[b, 0]), _d(s[b, 1]),
                                    *[ctypes.c_double(v) for v in (coef, dx, dy, dz, g[0], g[1], g[2])])
    return out


def hamiltonian(grid, V, tables, psi, nb, is_complex=False, g=(0.0, 0.0, 0.0)):
    """H psi (restatement of mHamiltonianMatrix_ddm), FP64."""
    return _hamiltonian_fd8(grid, V, tables, psi, nb, is_complex, g)


def _hamiltonian_fd8(grid, V, tables, psi, nb, is_complex=False, g=(0.0, 0.0, 0.0)):
    lib = oracle_lib()
    nx, ny, nz, dx, dy, dz = grid
    npts, widths, coords, beta, energy = tables
    psi = np.ascontiguousarray(psi, np.float64)
    hp = np.zeros_like(psi)
    V = np.ascontiguousarray(V, np.float64)
    lib.qso_hamiltonian(nx, ny, nz, *[ctypes.c_double(v) for v in (dx, dy, dz)], _d(V), len(npts), _i(npts),
                        _i(widths), _i(coords), _d(beta), _d(energy), nb, int(is_complex), _d(hp), _d(psi),
                        *[ctypes.c_double(v) for v in g])
    return hp


def nonlocal_apply(grid, tables, psi, nb, is_complex=False, g=(0.0, 0.0, 0.0), hp=None):
    lib = oracle_lib()
    nx, ny, nz, dx, dy, dz = grid
    npts, widths, coords, beta, energy = tables
    psi = np.ascontiguousarray(psi, np.float64)
    if hp is None:
        hp = np.zeros_like(psi)
    lib.qso_nonlocal_apply(nx, ny, nz, *[ctypes.c_double(v) for v in (dx, dy, dz)], len(npts), _i(npts), _i(widths),
                           _i(coords), _d(beta), _d(energy), nb, int(is_complex), _d(hp), _d(psi),
                           *[ctypes.c_double(v) for v in g])
    return hp


def nonlocal_project(grid, tables, psi, nb, is_complex=False, g=(0.0, 0.0, 0.0)):
    lib = oracle_lib()
    nx, ny, nz, dx, dy, dz = grid
    npts, widths, coords, beta, energy = tables
    P = int(widths.sum())
    ncol = 2 * nb if is_complex else nb
    out = np.zeros((ncol, P))
    psi = np.ascontiguousarray(psi, np.float64)
    lib.qso_nonlocal_project(nx, ny, nz, *[ctypes.c_double(v) for v in (dx, dy, dz)], len(npts), _i(npts),
                             _i(widths), _i(coords), _d(beta), nb, int(is_complex), _d(psi),
                             *[ctypes.c_double(v) for v in g], _d(out))
    return out


# --------------------------------------------------------------------------
# the reference's own code (oracle/_ref)
# --------------------------------------------------------------------------
def ref_nonlocal_energy_force(grid, cube, psi_soa, nb, occ, g=(0.0, 0.0, 0.0)):
    """The reference's nonlocal energy and forces (qsref_nonlocal_energy_force)
    on cube tables (gth_cube_tables) for nb complex SoA bands."""
    lib = ref_lib()
    nx, ny, nz, dx, dy, dz = grid
    e = ctypes.c_double()
    F = np.zeros(3 * len(cube["widths"]))
    psi = np.ascontiguousarray(psi_soa, np.float64)
    occ = np.ascontiguousarray(occ, np.float64)
    lib.qsref_nonlocal_energy_force(nx, ny, nz, *[ctypes.c_double(v) for v in (dx, dy, dz)], len(cube["widths"]),
                                    _i(cube["cubes"]), _i(cube["widths"]), _d(cube["proj"]), _d(cube["grad"]),
                                    _d(cube["energy"]), nb, _d(psi), _d(occ), *[ctypes.c_double(v) for v in g],
                                    ctypes.byref(e), _d(F))
    return e.value, F.reshape(-1, 3)


def ref_laplacian8th(nx, ny, nz, out, p, coef, dx, dy, dz):
    lib = ref_lib()
    N = nx * ny * nz
    p = np.ascontiguousarray(p, np.float64).reshape(-1, N)
    o = out.reshape(-1, N)
    for b in range(p.shape[0]):
        lib.qsref_laplacian8th(nx, ny, nz, _d(o[b]), _d(p[b]), *[ctypes.c_double(v) for v in (coef, dx, dy, dz)])
    return out


def ref_laplacian_kpoint8th(nx, ny, nz, out, src, coef, dx, dy, dz, g):
    lib = ref_lib()
    N = nx * ny * nz
    s = np.ascontiguousarray(src, np.float64).reshape(-1, 2, N)
    o = out.reshape(-1, 2, N)
    for b in range(s.shape[0]):
        lib.qsref_laplacian_kpoint8th(nx, ny, nz, _d(o[b, 0]), _d(o[b, 1]), _d(s[b, 0]), _d(s[b, 1]),
                                      *[ctypes.c_double(v) for v in (coef, dx, dy, dz, g[0], g[1], g[2])])
    return out


def ref_hamiltonian(grid, V, cube, psi, nb, is_complex=False, g=(0.0, 0.0, 0.0)):
    """H psi by the reference's own operators (mHamiltonianMatrix_ddm composition)."""
    lib = ref_lib()
    nx, ny, nz, dx, dy, dz = grid
    psi = np.ascontiguousarray(psi, np.float64)
    hp = np.zeros_like(psi)
    V = np.ascontiguousarray(V, np.float64)
    args = [nx, ny, nz, *[ctypes.c_double(v) for v in (dx, dy, dz)], _d(V), len(cube["widths"]), _i(cube["cubes"]),
            _i(cube["widths"]), _d(cube["proj"]), _d(cube["energy"]), nb, _d(hp), _d(psi)]
    if is_complex:
        lib.qsref_hamiltonian_complex(*args, *[ctypes.c_double(v) for v in g])
    else:
        lib.qsref_hamiltonian_real(*args)
    return hp


def ref_set_threads(n):
    ref_lib().qsref_set_threads(int(n))


# --------------------------------------------------------------------------
# eigensolver oracles
# --------------------------------------------------------------------------
def orthonormal_psi(seed, nb, N, dV, complex_=False):
    """Seeded psi ~ U[-0.5,0.5], orthonormalized with the dV-weighted inner product
    (the role of GramSchmidt_ddm, source/GramSchmidt_mpi.h:56-96: same span, done by QR)."""
    a = seeded_psi(seed, nb, N, complex_)
    if complex_:
        z = (a[0::2] + 1j * a[1::2]).T
        q, _ = np.linalg.qr(z)
        q = q.T / math.sqrt(dV)
        out = np.empty((2 * nb, N))
        out[0::2] = q.real
        out[1::2] = q.imag
        return out
    q, _ = np.linalg.qr(a.T)
    return np.ascontiguousarray(q.T / math.sqrt(dV))


def _cube_args(cube):
    return (len(cube["widths"]), _i(cube["cubes"]), _i(cube["widths"]), _d(cube["proj"]), _d(cube["energy"]))


def ref_lobpcg_z(grid, V, cube, X, keep, n, iter_max, eigen_values, num_fix, residual_threshold, scf_step,
                 g=(0.0, 0.0, 0.0)):
    """LOBPCG::Eigen_z_multi_mpi of the reference (in place on X, keep, eigen_values); returns num_fix."""
    lib = ref_lib()
    nx, ny, nz, dx, dy, dz = grid
    for a in (X, keep, eigen_values):
        assert a.dtype == np.float64 and a.flags.c_contiguous
    V = np.ascontiguousarray(V, np.float64)
    nf = ctypes.c_int(int(num_fix))
    lib.qsref_lobpcg_z(nx, ny, nz, *[ctypes.c_double(v) for v in (dx, dy, dz)], _d(V), *_cube_args(cube), n, iter_max,
                       _d(eigen_values), _d(X), _d(keep), ctypes.byref(nf), ctypes.c_double(residual_threshold),
                       int(scf_step), *[ctypes.c_double(v) for v in g])
    return nf.value


def ref_lobpcg_d(grid, V, cube, X, keep, n, iter_max, eigen_values, is_first_time):
    """EigenLOBPCG_d_multi of the reference (in place on X, keep, eigen_values)."""
    lib = ref_lib()
    nx, ny, nz, dx, dy, dz = grid
    N = nx * ny * nz
    V = np.ascontiguousarray(V, np.float64)
    work = np.zeros(5 * N * n)
    lib.qsref_lobpcg_d(nx, ny, nz, *[ctypes.c_double(v) for v in (dx, dy, dz)], _d(V), *_cube_args(cube), n, iter_max,
                       _d(eigen_values), _d(X), _d(keep), _d(work), int(is_first_time))


def ref_gram_schmidt(grid, X, nb, is_complex=False):
    """GramSchmidt_ddm of the reference (GramSchmidt_mpi.h:56-96), on a copy of X."""
    lib = ref_lib()
    nx, ny, nz, dx, dy, dz = grid
    out = np.ascontiguousarray(X, np.float64).copy()
    lib.qsref_gram_schmidt(nx, ny, nz, nb, int(is_complex), _d(out), ctypes.c_double(dx * dy * dz))
    return out


def dense_eigenvalues(grid, V, tables, k, is_complex=False, g=(0.0, 0.0, 0.0), fft=False):
    """Lowest k eigenvalues of H built column by column with the C restatement
    (fft: with the FFT kinetic of hamiltonian_fft; small grids only)."""
    hamiltonian = hamiltonian_fft if fft else _hamiltonian_fd8
    nx, ny, nz = grid[:3]
    N = nx * ny * nz
    if is_complex:
        M = np.zeros((N, N), complex)
        e = np.zeros((2, N))
        for j in range(N):
            e[:] = 0.0
            e[0, j] = 1.0
            h = hamiltonian(grid, V, tables, e.reshape(1, 2, N), 1, True, g).reshape(2, N)
            M[:, j] = h[0] + 1j * h[1]
        M = 0.5 * (M + M.conj().T)
    else:
        M = np.zeros((N, N))
        e = np.zeros((1, N))
        for j in range(N):
            e[:] = 0.0
            e[0, j] = 1.0
            M[:, j] = hamiltonian(grid, V, tables, e, 1)[0]
        M = 0.5 * (M + M.T)
    return np.linalg.eigvalsh(M)[:k]


def kinetic_fft(grid, psi, nb, is_complex=False, g=(0.0, 0.0, 0.0)):
    """-1/2 (grad + i k)^2 psi by FFT, FP64: the FFT kinetic of the reference's
    default Hamiltonian (mHamiltonianMatrix_ddm_bundle, algorithm 1,
    source/qumasun_base1.matrix.h:171-228, multiplier of
    OperateKineticInKspace_bundle :96-123): forward 3-D FFT of each band,
    times |G + k|^2 / 2 with G_d = 2 pi m / (n_d h_d) and m folded as
    (2m > n ? m - n : m) -- the Nyquist index of an even grid stays +n/2 --
    inverse FFT, times 1/N.  Real bands (k = 0): the same operator on psi as a
    complex field with zero imaginary part, real part returned."""
    nx, ny, nz, dx, dy, dz = grid
    psi = np.asarray(psi, np.float64)

    def axis(n, h, gk):
        m = np.arange(n)
        m = np.where(2 * m > n, m - n, m)
        return 2.0 * math.pi * m / (n * h) + gk

    kx, ky, kz = axis(nx, dx, g[0]), axis(ny, dy, g[1]), axis(nz, dz, g[2])
    mult = 0.5 * (kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2)
    if is_complex:
        f = psi.reshape(nb, 2, nz, ny, nx)
        c = f[:, 0] + 1j * f[:, 1]
    else:
        c = psi.reshape(nb, nz, ny, nx).astype(np.complex128)
    out = np.fft.ifftn(np.fft.fftn(c, axes=(-3, -2, -1)) * mult, axes=(-3, -2, -1))
    if is_complex:
        return np.stack([out.real, out.imag], axis=1).reshape(psi.shape)
    return out.real.reshape(psi.shape)


def hamiltonian_fft(grid, V, tables, psi, nb, is_complex=False, g=(0.0, 0.0, 0.0)):
    """H psi with the FFT kinetic (mHamiltonianMatrix_ddm_bundle, algorithm 1):
    FFT kinetic + V psi (mPotentialMatrixAdd_ddm_bundle) + nonlocal
    (ProjectionPP_bundle), FP64."""
    nx, ny, nz = grid[:3]
    N = nx * ny * nz
    psi = np.ascontiguousarray(psi, np.float64)
    hp = kinetic_fft(grid, psi, nb, is_complex, g)
    hp = hp + (psi.reshape(-1, N) * np.asarray(V, np.float64)[None, :]).reshape(psi.shape)
    return nonlocal_apply(grid, tables, psi, nb, is_complex, g, np.ascontiguousarray(hp))


def ref_cube_write(path, field, grid, axis, origin, Z, pos, comment=""):
    """The reference's CubeWriter::SaveCube (cube_writer.h:27-90) through oracle/_ref."""
    lib = ref_lib()
    nx, ny, nz = grid
    f = np.ascontiguousarray(field, np.float64).ravel()
    z = np.ascontiguousarray(Z, np.int32).ravel()
    p = np.ascontiguousarray(pos, np.float64).ravel()
    ax = np.ascontiguousarray(axis, np.float64).ravel()
    org = np.ascontiguousarray(origin, np.float64).ravel()
    lib.qsref_cube_write(os.fsencode(path), comment.encode(), nx, ny, nz, _d(ax), _d(org), int(z.size),
                         z.ctypes.data_as(_ip), _d(p), _d(f))


def ref_cube_read(path):
    """The reference's CubeReader3::LoadCube + GetMeshData (cube_reader3.h:38-124)."""
    lib = ref_lib()
    grid = np.zeros(3, np.int32)
    ax, org = np.zeros(9), np.zeros(3)
    lib.qsref_cube_read(os.fsencode(path), grid.ctypes.data_as(_ip), _d(ax), _d(org), None)
    f = np.zeros(int(np.prod(grid)))
    lib.qsref_cube_read(os.fsencode(path), grid.ctypes.data_as(_ip), _d(ax), _d(org), _d(f))
    return f, {"grid": tuple(int(v) for v in grid), "axis": ax.reshape(3, 3), "origin": org}


def ref_upf_load(path):
    """The reference's LoadUPF_ONCV (upf_oncv_loader.h:353-1050) through oracle/_ref:
    dict of its radial data (projectors are the up-spin copies)."""
    lib = ref_lib()
    info = np.zeros(3, np.int32)
    if not lib.qsref_upf_load(os.fsencode(path), info.ctypes.data_as(_ip), None, None, None, None, None, None, None):
        raise OSError(path)
    n, zv, ng = (int(v) for v in info)
    cut, xi = np.zeros(4), np.zeros(2)
    r, v = np.zeros(ng), np.zeros(ng)
    l, e = np.zeros(max(n, 1), np.int32), np.zeros(max(n, 1))
    pr = np.zeros(max(n, 1) * ng)
    lib.qsref_upf_load(os.fsencode(path), info.ctypes.data_as(_ip), _d(cut), _d(xi), _d(r), _d(v),
                       l.ctypes.data_as(_ip), _d(e), _d(pr))
    return {"n_projectors": n, "z_valence": zv, "n_grid": ng, "cutoff_l": cut, "xi": xi, "radius": r,
            "v_local": v, "l": l[:n], "energy": e[:n], "projectors": pr[: n * ng].reshape(n, ng)}
