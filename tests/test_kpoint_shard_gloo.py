"""World-size-2 check, on the CPU (gloo), of the host side of the sharded
k-point SCF step: the k-point partition (qsb_dist.partition_kpoints), the sum
over ranks (qsb_dist.allreduce_sum, the callback qsb_scf_set_reduce takes) of
the levels, which every rank needs for the one Fermi level
(qsb_fermi_occupations), and of the partial output densities.  Each rank
forms its own k-points' part exactly as qsb_scf_run_kpoints does (levels of
k-points owned elsewhere are zero, the density is sum_k w_k sum_n f_nk |psi_nk|^2
over its own k-points); the joined step equals the single-process step to 1e-12."""
import os
import socket

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NK, NB, N, N_EL = 8, 6, 2000, 7.0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _inputs():
    rng = np.random.default_rng(11)
    levels = np.sort(rng.uniform(-0.5, 0.4, (NK, NB)), axis=1)
    states = rng.uniform(-0.5, 0.5, (NK, 2 * NB, N))          # complex SoA bundles per k-point
    w = rng.uniform(0.5, 1.5, NK)
    return levels, states, w / w.sum()


def _step(qsb, owned, reduce):
    levels, states, w = _inputs()
    rq = np.where(np.asarray(owned)[:, None] != 0, levels, 0.0).ravel().copy()
    reduce(rq)
    occ, mu = qsb.fermi_occupations(rq, N_EL, 0.01, np.repeat(w, NB))
    occ = occ.reshape(NK, NB)
    rho = np.zeros(N)
    for k in range(NK):
        if owned[k]:
            re, im = states[k][0::2], states[k][1::2]
            rho += np.einsum("n,ni->i", w[k] * occ[k], re * re + im * im)
    reduce(rho)
    return occ, mu, rho


def _rank_main(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "qumasun-workshop-template_b200"))
    import qsb
    import qsb_dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        owned = qsb_dist.partition_kpoints(NK, world, rank)
        occ, mu, rho = _step(qsb, owned, qsb_dist.allreduce_sum())
        out[rank] = (owned.tolist(), occ.tolist(), mu, rho.tolist())
    finally:
        dist.destroy_process_group()


def test_sharded_kpoint_step_equals_the_single_process_step(qsb_host):
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    occ1, mu1, rho1 = _step(qsb_host, [1] * NK, lambda a: None)
    owned = np.array([out[r][0] for r in range(world)])
    assert np.array_equal(owned.sum(axis=0), np.ones(NK)) and owned.sum(axis=1).min() > 0
    for r in range(world):
        _, occ, mu, rho = out[r]
        np.testing.assert_allclose(np.array(occ), occ1, rtol=0, atol=1e-12)
        assert abs(mu - mu1) < 1e-12
        np.testing.assert_allclose(np.array(rho), rho1, rtol=1e-12, atol=0)
