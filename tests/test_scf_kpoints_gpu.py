"""GPU checks of the k-point SCF (qsb_scf_set_kpoints / qsb_scf_run_kpoints)
through the C ABI against the oracle k-point loop (oracle/scf_oracle.py
scf_kpoints: the reference's own Eigen_z_multi_mpi per k-point, fixture
tests/golden/scf_kpt.npz made by tests/golden/make_golden.py).

The config-0 cell on a 20^3 grid with the 2 x 2 x 2 Gamma-centred k mesh (8
k-points, 10 complex bands each), LDA, Fermi 0.01 Ha, Kerker-DIIS.  Bars: the
FP64 run follows the oracle's energies within 1e-6 Ha per step over the first
8 steps and ends within 1e-6 Ha / atom of it; two contexts that each own half
of the k-points, joined by a sum over host buffers (the form qsb_dist gives the
ranks of a multi-GPU run), reproduce the single-context run to 1e-10 Ha; the
mixed-precision run converged to 1e-8 Ha / atom ends within 1e-6 Ha / atom of
the FP64 one."""
import os
import threading

import numpy as np
import pytest

import oracle as O
from cases import SCF_KPT, scf_kpt_inputs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _run(qsb, precision="fp64", owned=None, reduce=None, tol=None, max_steps=None):
    import torch
    inp = scf_kpt_inputs()
    nx, ny, nz, dx, dy, dz = inp["grid"]
    N = nx * ny * nz
    sp = inp["sp"][0]
    H = qsb.Hamiltonian(nx, ny, nz, dx, dy, dz)
    H.set_gth_projectors(inp["pos"], [0, 0], [sp["nl"]], [sp["r"]], [sp["h"]], O.RCUT_FACTOR)
    H.set_potential(np.zeros(N))
    es = qsb.EigenSolver(N, SCF_KPT["nb"], True, precision)
    scf = qsb.SCF(H, es, SCF_KPT["nb"], SCF_KPT["n_el"])
    scf.set_gth_local(inp["pos"], [0, 0], [sp["zion"]], [sp["rloc"]], [sp["c1"]], [sp["c2"]])
    p = SCF_KPT["params"]
    scf.set_mixing(p["amplitude"], p["q0"], p["depth"])
    scf.set_smearing(p["kbt"])
    scf.set_kpoints(inp["kvecs"], inp["weights"], owned)
    if reduce is not None:
        scf.set_reduce(reduce)
    own = [True] * len(inp["weights"]) if owned is None else [bool(o) for o in owned]
    Xs = [torch.from_numpy(x.copy()).cuda() if o else None for x, o in zip(inp["Xs"], own)]
    keeps = [torch.zeros_like(x) if x is not None else None for x in Xs]
    e, ev, occ = scf.run_kpoints(Xs, keeps, p["lobpcg_iters"], max_steps or p["max_steps"], tol or p["tol_per_atom"])
    return dict(e=e, ev=ev, occ=occ, scf=scf, H=H, es=es, Xs=Xs)


def test_fp64_kpoint_scf_follows_the_oracle(qsb):
    r = _run(qsb)
    gold = np.load(os.path.join(GOLD, "scf_kpt.npz"))
    ge = gold["energies"]
    k = min(8, len(ge), len(r["e"]))
    np.testing.assert_allclose(r["e"][:k], ge[:k], rtol=0, atol=1e-6)
    assert abs(r["e"][-1] - ge[-1]) / 2 < 1e-6, (r["e"][-1], ge[-1])
    assert abs(len(r["e"]) - len(ge)) <= 4
    w = scf_kpt_inputs()["weights"]
    assert abs(float(np.sum(w[:, None] * r["occ"])) - SCF_KPT["n_el"]) < 1e-9
    assert qsb.device_status() == 0


class _ThreadSum:
    """Sum over the contexts of the threads of one process, in context order."""

    def __init__(self, n):
        self.n = n
        self.bar = threading.Barrier(n, timeout=120)
        self.bufs = [None] * n

    def fn(self, i):
        def f(buf):
            self.bufs[i] = buf.copy()
            self.bar.wait()
            total = self.bufs[0].copy()
            for j in range(1, self.n):
                total += self.bufs[j]
            self.bar.wait()
            buf[:] = total
        return f


def test_two_contexts_sharing_the_kpoints_equal_one(qsb):
    import qsb_dist
    one = _run(qsb)
    nk = len(scf_kpt_inputs()["weights"])
    owned = [qsb_dist.partition_kpoints(nk, 2, r) for r in range(2)]
    ts = _ThreadSum(2)
    res = [None, None]
    errs = []

    def worker(r):
        try:
            res[r] = _run(qsb, owned=owned[r], reduce=ts.fn(r))
        except Exception as e:              # reported below
            errs.append(e)
            ts.bar.abort()

    th = [threading.Thread(target=worker, args=(r,)) for r in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
    for r in range(2):
        assert len(res[r]["e"]) == len(one["e"])
        np.testing.assert_allclose(res[r]["e"], one["e"], rtol=0, atol=1e-10)
        np.testing.assert_allclose(res[r]["ev"], one["ev"], rtol=0, atol=1e-10)
    assert qsb.device_status() == 0


def test_mixed_kpoint_scf_reaches_the_fp64_energy(qsb):
    r64 = _run(qsb, "fp64", tol=1e-8, max_steps=100)
    r32 = _run(qsb, "mixed", tol=1e-8, max_steps=100)
    assert abs(r32["e"][-1] - r64["e"][-1]) / 2 < 1e-6, (r32["e"][-1], r64["e"][-1])
    assert qsb.device_status() == 0
