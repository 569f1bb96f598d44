"""k-point sharding of the device SCF over ranks (one process per GPU), the
split the reference makes over its (spin, k) groups
(source/qumasun_base1.constructor.h:66,136-160; the density gathered by
mReduceFieldInSamePlace, source/qumasun_base1.density.h:43, and the Fermi level
over all groups, source/qumasun_base1.occupancy.h:76-170).

Each rank owns a part of the k list and runs qsb_scf_run_kpoints on it; per SCF
step the library calls back twice for a sum over the ranks (the levels, n_k x nb
doubles, which the Fermi level needs on every rank; the output density, N
doubles) and once before the first step (the starting density).  Nothing else
crosses ranks: the solver, H.psi and the pencil solves stay on each GPU.  The
sums here go through torch.distributed (NCCL between GPUs, gloo on the CPU),
staged in host buffers by the library."""
import numpy as np


def partition_kpoints(n_k, world, rank, cost=None):
    """Owned flags of `rank`: the k-points dealt to ranks largest cost first,
    each to the rank with the least total so far (ties: lowest rank), so the
    split does not depend on which rank computes it."""
    cost = np.ones(n_k) if cost is None else np.asarray(cost, np.float64)
    load = np.zeros(world)
    owner = np.empty(n_k, np.int64)
    for k in sorted(range(n_k), key=lambda i: (-cost[i], i)):
        r = int(np.argmin(load))
        owner[k] = r
        load[r] += cost[k]
    return (owner == rank).astype(np.int32)


def allreduce_sum(group=None):
    """A reduction for qsb.SCF.set_reduce: replaces the host array by its sum
    over the process group (torch.distributed, any backend; with NCCL the
    buffer goes through the rank's current CUDA device)."""
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)

    def fn(buf):
        t = torch.from_numpy(buf)
        if backend == "nccl":
            d = t.to("cuda")
            dist.all_reduce(d, op=dist.ReduceOp.SUM, group=group)
            t.copy_(d.cpu())
        else:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return fn
