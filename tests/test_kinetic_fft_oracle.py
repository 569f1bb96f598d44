"""CPU checks of the FFT-kinetic restatement (oracle.kinetic_fft /
hamiltonian_fft) of the reference's default Hamiltonian
(mHamiltonianMatrix_ddm_bundle, algorithm 1, source/qumasun_base1.matrix.h:171-228).

The restatement is pinned to the reference's own FFT-kinetic code by the
ham_fft_* golden cases (tests/test_oracle.py: the reference object built in
oracle/_ref/libqsref_fft.so with FFTW's documented DFT restated in
oracle/ref_shim/fftw_dft.cpp, 1e-14), and here by the operator's own
definition: plane waves exp(i G.r) are eigenfunctions with eigenvalue
|G + k|^2 / 2, the G of an even grid's Nyquist index taken as +n/2 (the fold of
OperateKineticInKspace_bundle, :96-123) -- 1e-12 relative; the operator is
Hermitian (1e-12); on a smooth periodic field it agrees with the reference's
own FD8 Laplacian (oracle/_ref) converges to it at eighth order."""
import math

import numpy as np
import pytest

import oracle as O

GRID = (8, 6, 5, 0.3, 0.4, 0.5)


def _plane(grid, m):
    nx, ny, nz, dx, dy, dz = grid
    G = [2 * math.pi * mi / (n * h) for mi, n, h in zip(m, (nx, ny, nz), (dx, dy, dz))]
    x, y, z = np.arange(nx) * dx, np.arange(ny) * dy, np.arange(nz) * dz
    return G[0] * x[None, None, :] + G[1] * y[None, :, None] + G[2] * z[:, None, None]


def _folded(grid, m):
    nx, ny, nz, dx, dy, dz = grid
    out = []
    for mi, n, h in zip(m, (nx, ny, nz), (dx, dy, dz)):
        r = mi % n
        out.append(2 * math.pi * ((r - n) if 2 * r > n else r) / (n * h))
    return out


@pytest.mark.parametrize("m", [(0, 0, 0), (4, 0, 0), (-4, 3, 0), (3, -2, 2), (-3, 3, -2), (1, 1, 1)])
@pytest.mark.parametrize("g", [(0.0, 0.0, 0.0), (0.3, -0.2, 0.1)])
def test_plane_waves_are_eigenfunctions(m, g):
    ph = _plane(GRID, m)
    psi = np.stack([np.cos(ph), np.sin(ph)])[None]
    out = O.kinetic_fft(GRID, psi.ravel(), 1, True, g).reshape(psi.shape)
    lam = 0.5 * sum((a + b) ** 2 for a, b in zip(_folded(GRID, m), g))
    assert np.abs(out - lam * psi).max() <= 1e-12 * max(lam, 1.0)


def test_real_bands_nyquist_cosine():
    # cos(pi x / h) lives on the x Nyquist index alone: eigenvalue (pi / h)^2 / 2
    ph = _plane(GRID, (4, 0, 0))
    psi = np.cos(ph)[None]
    out = O.kinetic_fft(GRID, psi.ravel(), 1).reshape(psi.shape)
    lam = 0.5 * (math.pi / GRID[3]) ** 2
    assert np.abs(out - lam * psi).max() <= 1e-12 * lam


def test_hermitian():
    rng = np.random.default_rng(4)
    nx, ny, nz = GRID[:3]
    N = nx * ny * nz
    a, b = rng.standard_normal((2, 1, 2, N))
    g = (0.3, -0.2, 0.1)
    ta = O.kinetic_fft(GRID, a.ravel(), 1, True, g).reshape(2, N)
    tb = O.kinetic_fft(GRID, b.ravel(), 1, True, g).reshape(2, N)
    ca, cb = a[0, 0] + 1j * a[0, 1], b[0, 0] + 1j * b[0, 1]
    cta, ctb = ta[0] + 1j * ta[1], tb[0] + 1j * tb[1]
    lhs, rhs = np.vdot(ca, ctb), np.vdot(cta, cb)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_the_reference_fd8_converges_to_it_at_eighth_order():
    """On a smooth periodic field the reference's FD8 kinetic approaches the
    FFT kinetic as h^8: halving h (L = 8 bohr, 32^3 -> 64^3) shrinks the gap by
    more than 2^8 / 2."""
    errs = []
    for n in (32, 64):
        L = 8.0
        h = L / n
        grid = (n, n, n, h, h, h)
        x = np.arange(n) * h
        f = np.exp(np.cos(2 * math.pi * x / L)[None, None, :] + 0.5 * np.sin(2 * math.pi * x / L)[None, :, None]
                   + 0.3 * np.cos(4 * math.pi * x / L)[:, None, None])
        psi = f.reshape(1, -1)
        t_fft = O.kinetic_fft(grid, psi, 1)
        t_fd = O.ref_laplacian8th(n, n, n, np.zeros_like(psi), psi, -0.5, h, h, h)
        errs.append(np.abs(t_fft - t_fd).max() / np.abs(t_fft).max())
    assert errs[0] < 1e-4 and errs[1] < errs[0] / 128, errs
