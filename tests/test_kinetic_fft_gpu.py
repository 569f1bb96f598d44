"""GPU parity of the FFT-kinetic Hamiltonian (qsb_ham_set_kinetic(ham, 1): the
reference's default operator, mHamiltonianMatrix_ddm_bundle algorithm 1,
source/qumasun_base1.matrix.h:171-228) against the oracle's restatement
(oracle.hamiltonian_fft) and against fixtures made by the reference's own
FFT-kinetic code (tests/golden/ham_fft_*.npz), called through the C ABI.

Tolerances: FP64 1e-12 relative L2 (the H.psi bar); FP32 2e-5 relative L2
against the FP64 oracle; LOBPCG on the FFT operator reaches the dense
eigenvalues of the oracle's FFT Hamiltonian to 1e-8 Ha."""
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
TOL64 = 1e-12
TOL32 = 2e-5
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def _setup(qsb, grid, nb, cplx, seed, reps=1):
    nx, ny, nz, dx, dy, dz = grid
    pos = O.bcc_positions(nx * dx / reps, reps, 0.0, seed) + np.array([0.13, 0.02, -0.09])
    tab = O.gth_tables(pos, [O.GTH_BCC] * len(pos), dx, dy, dz)
    V = O.seeded_potential(seed, nx * ny * nz)
    psi = O.seeded_psi(seed, nb, nx * ny * nz, cplx)
    H = qsb.Hamiltonian(nx, ny, nz, dx, dy, dz)
    H.set_potential(V)
    H.set_projectors(*tab)
    H.set_kinetic(1)
    return H, tab, V, psi


@pytest.mark.parametrize("grid,nb,cplx,g", [
    ((32, 32, 32, 0.1875, 0.1875, 0.1875), 16, False, (0.0, 0.0, 0.0)),   # config 0 shape
    ((32, 32, 32, 0.1875, 0.1875, 0.1875), 40, False, (0.0, 0.0, 0.0)),   # two band chunks, ragged
    ((33, 17, 9, 0.2, 0.3, 0.25), 3, False, (0.0, 0.0, 0.0)),             # odd extents, a half pair
    ((20, 18, 16, 0.3, 0.3, 0.3), 1, False, (0.0, 0.0, 0.0)),             # one real band: R2C / C2R
    ((20, 18, 16, 0.3, 0.3, 0.3), 35, False, (0.0, 0.0, 0.0)),            # pairs over two chunks, odd tail
    ((24, 20, 16, 0.25, 0.3, 0.375), 3, True, (0.3, -0.2, 0.7)),          # Bloch vector
    ((24, 20, 16, 0.25, 0.3, 0.375), 35, True, (0.26, 0.52, 0.0)),        # two chunks, complex
    ((15, 12, 10, 0.3, 0.3, 0.3), 2, True, (0.0, 0.0, 0.0))])
def test_fft_hamiltonian_vs_oracle(qsb, grid, nb, cplx, g):
    import torch
    H, tab, V, psi = _setup(qsb, grid, nb, cplx, 31)
    ref = O.hamiltonian_fft(grid, V, tab, psi, nb, cplx, g)
    p = torch.from_numpy(np.ascontiguousarray(psi)).cuda()
    p0 = p.clone()
    hp = torch.full_like(p, float("nan"))
    H.apply(p, hp, cplx, g)
    torch.cuda.synchronize()
    assert torch.equal(p, p0)                      # psi is not touched by the transforms
    assert rel(hp.cpu().numpy(), ref) < TOL64
    # FD8 again on the same context: the switch goes both ways
    H.set_kinetic(0)
    H.apply(p, hp, cplx, g)
    assert rel(hp.cpu().numpy(), O.hamiltonian(grid, V, tab, psi, nb, cplx, g)) < TOL64


@pytest.mark.parametrize("cplx", [False, True])
def test_fft_hamiltonian_fp32(qsb, cplx):
    import torch
    grid = (24, 20, 16, 0.25, 0.3, 0.375)
    g = (0.3, -0.2, 0.7) if cplx else (0.0, 0.0, 0.0)
    H, tab, V, psi = _setup(qsb, grid, 5, cplx, 32)
    ref = O.hamiltonian_fft(grid, V, tab, psi, 5, cplx, g)
    p = torch.from_numpy(np.ascontiguousarray(psi)).float().cuda()
    hp = torch.empty_like(p)
    H.apply(p, hp, cplx, g)
    assert rel(hp.double().cpu().numpy(), ref) < TOL32


def test_lobpcg_on_the_fft_operator_reaches_dense_eigenvalues(qsb):
    import torch
    n, a = 10, 6.0
    h = a / n
    grid = (n, n, n, h, h, h)
    N = n ** 3
    H, tab, V, _ = _setup(qsb, grid, 1, False, 33)
    exact = O.dense_eigenvalues(grid, V, tab, 6, fft=True)
    nb = 10
    es = qsb.EigenSolver(N, nb, False)
    es.set_hamiltonian(H)
    X = torch.from_numpy(O.orthonormal_psi(3, nb, N, h ** 3)).cuda()
    keep = torch.zeros_like(X)
    ev = np.zeros(nb)
    for step in range(40):
        es.lobpcg_d(h ** 3, nb, 4, ev, X, keep, step == 0)
    np.testing.assert_allclose(np.sort(ev)[:6], exact, rtol=0, atol=1e-8)
    assert qsb.device_status() == 0


@pytest.mark.parametrize("name", ["ham_fft_real_c0", "ham_fft_kpt_even", "ham_fft_kpt_odd"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_fft_hamiltonian_vs_reference_fixture(qsb, name, prec):
    """-1/2 (grad + ik)^2 psi + V psi of the FFT-kinetic context against the
    output of the reference's own mHamiltonianMatrix_ddm_bundle (algorithm 1),
    stored in tests/golden/<name>.npz (tests/golden/make_golden.py): even and
    odd extents, Gamma and k-points on the reference's k index grid."""
    import torch
    from cases import CASES, FFT_KPT
    case = CASES[name]
    inp = case["inputs"]()
    gold = np.load(os.path.join(GOLD, name + ".npz"))
    np.testing.assert_array_equal(gold["checksum"], np.array([float(np.sum(v)) for v in inp["checked"]]))
    grid, nb = inp["grid"], inp["nb"]
    cplx = name != "ham_fft_real_c0"
    g = O.kpoint_vector(grid, *FFT_KPT[name])
    H = qsb.Hamiltonian(*grid)
    H.set_potential(inp["V"])
    H.set_kinetic(1)
    p = torch.from_numpy(np.ascontiguousarray(inp["psi"])).cuda()
    if prec == "f32":
        p = p.float()
    hp = torch.full_like(p, float("nan"))
    H.apply(p, hp, cplx, g)
    torch.cuda.synchronize()
    assert rel(hp.double().cpu().numpy(), gold["out"]) < (TOL64 if prec == "f64" else TOL32)
