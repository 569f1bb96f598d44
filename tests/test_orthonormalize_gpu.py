"""qsb_orthonormalize (Cholesky QR twice) against the reference's own
GramSchmidt_ddm (source/GramSchmidt_mpi.h:56-96, compiled into oracle/_ref) on
seeded U[-0.5, 0.5] bundles: real and complex SoA, the config-0 shape (32^3,
16 bands) among them.  Both give the Q factor of X = Q R with a positive
diagonal R, so the states agree to rounding: 1e-12 relative L2, and
dV <x_j|x_k> equals delta_jk to 1e-13."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not O.ref_available(), reason="needs oracle/_ref")
@pytest.mark.parametrize("shape,nb,cplx,seed", [((32, 32, 32), 16, False, 0), ((16, 12, 10), 8, False, 3),
                                                ((12, 10, 8), 6, True, 4), ((24, 24, 24), 24, True, 5)])
def test_orthonormalize_matches_reference_gram_schmidt(qsb, shape, nb, cplx, seed):
    import torch
    nx, ny, nz = shape
    N = nx * ny * nz
    h = 6.0 / nx
    grid = (nx, ny, nz, h, h, h)
    dV = h ** 3
    X = O.seeded_psi(seed, nb, N, cplx)
    want = O.ref_gram_schmidt(grid, X, nb, cplx)
    got = qsb.orthonormalize(torch.from_numpy(X).cuda(), N, dV, cplx).cpu().numpy()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-12
    if cplx:
        z = got[0::2] + 1j * got[1::2]
        S = (z.conj() @ z.T) * dV
    else:
        S = (got @ got.T) * dV
    assert np.abs(S - np.eye(nb)).max() < 1e-13


def test_orthonormalize_rejects_dependent_bands(qsb):
    import torch
    N = 4096
    X = np.random.default_rng(1).uniform(-0.5, 0.5, (4, N))
    X[3] = X[1]
    with pytest.raises(qsb.QsbError, match="linearly dependent"):
        qsb.orthonormalize(torch.from_numpy(X).cuda(), N, 0.01)
