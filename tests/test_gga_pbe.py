"""CPU checks of the GGA-PBE restatement (oracle/scf_oracle.py gga_pbe): it is
pinned to the reference's own mSetPotentialVxc by the gga_pbe golden case
(tests/test_oracle.py, 1e-14); here, its potential is the exact derivative of
its discrete energy (the FD8 first derivative is antisymmetric, so the
divergence term is the adjoint of the gradient): central differences of
E_xc[rho + t d] equal dV sum V_xc d to 1e-8 relative, and the exchange part
alone reduces to the LDA exchange of a uniform density."""
import math

import numpy as np

import scf_oracle as S
from cases import GGA_GRID, gga_density


def test_potential_is_the_derivative_of_the_energy():
    rho = gga_density()
    rng = np.random.default_rng(3)
    nx, ny, nz, dx, dy, dz = GGA_GRID
    d = rng.uniform(-1.0, 1.0, rho.size) * rho * 0.1        # keeps rho + t d > 0
    d[rho < 1e-8] = 0.0
    _, vxc, _, _ = S.gga_pbe(GGA_GRID, rho)
    t = 1e-4
    ep = sum(S.gga_pbe(GGA_GRID, rho + t * d)[2:])
    em = sum(S.gga_pbe(GGA_GRID, rho - t * d)[2:])
    fd = (ep - em) / (2 * t)
    an = float(np.dot(vxc, d)) * dx * dy * dz
    assert abs(fd - an) <= 1e-8 * abs(an), (fd, an)


def test_uniform_density_exchange_is_the_lda_exchange():
    rho = np.full(GGA_GRID[0] * GGA_GRID[1] * GGA_GRID[2], 0.37)
    exc, vxc, ex, ec = S.gga_pbe(GGA_GRID, rho)
    dV = GGA_GRID[3] * GGA_GRID[4] * GGA_GRID[5]
    # no gradient: F = 1, e_x = -(3/4)(3/pi)^(1/3) rho^(4/3)
    lda_ex = -(3.0 / 4.0) * (3.0 / math.pi) ** (1.0 / 3.0) * 0.37 ** (4.0 / 3.0) * rho.size * dV
    assert abs(ex - lda_ex) <= 1e-12 * abs(lda_ex)
    assert np.ptp(vxc) <= 1e-12 * abs(vxc[0])
