"""Host pieces of the k-point SCF on the CPU: the weighted Fermi occupations
(qsb_fermi_occupations) against the oracle's k-group restatement of
mSetOccupancyTemperature, whose per-level formula is the reference's own
SetOccupancy; and the k-point partition of the sharded form."""
import numpy as np
import pytest

import scf_oracle as S


def test_weighted_fermi_occupations_match_the_oracle(qsb_host):
    rng = np.random.default_rng(7)
    nk, nb = 6, 9
    eig = np.sort(rng.uniform(-0.8, 0.6, (nk, nb)), axis=1)
    w = rng.uniform(0.5, 1.5, nk)
    w /= w.sum()
    for n_el in (3.0, 7.5, 12.0):
        want, mu_w = S.fermi_occupancy_kpoints(eig, w, n_el, 0.01)
        occ, mu = qsb_host.fermi_occupations(eig, n_el, 0.01, np.repeat(w, nb))
        f_want = want / w[:, None]
        np.testing.assert_allclose(occ.reshape(nk, nb), f_want, rtol=0, atol=1e-13)
        assert abs(mu - mu_w) < 1e-12
        assert abs(float(np.sum(np.repeat(w, nb) * occ)) - n_el) < 1e-12


def test_fermi_occupations_reject_bad_input(qsb_host):
    with pytest.raises(qsb_host.QsbError, match="more electrons"):
        qsb_host.fermi_occupations(np.zeros(3), 7.0, 0.01)
    with pytest.raises(qsb_host.QsbError):
        qsb_host.fermi_occupations(np.array([0.0, np.nan]), 1.0, 0.01)


def test_partition_balances_and_covers(qsb_host):
    import qsb_dist
    for n_k, world in ((64, 2), (64, 8), (7, 3), (3, 4)):
        cost = np.random.default_rng(n_k + world).uniform(1, 3, n_k)
        owned = np.array([qsb_dist.partition_kpoints(n_k, world, r, cost) for r in range(world)])
        assert np.array_equal(owned.sum(axis=0), np.ones(n_k))          # every k-point exactly once
        loads = owned @ cost
        assert loads.max() - loads.min() <= cost.max() + 1e-12         # greedy bound
