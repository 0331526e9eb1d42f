"""The oracle's t-V bond field on the finite-temperature path (CPU).

The restatement of dqmc_update.f90 and of the bond field's steps in
dqmc_ft_sweep_0b.f90 / dqmc_ft_sweep_b0.f90 / dqmc_ft_core.f90 is pinned two
ways: the propagated G agrees with the one recomputed from the UDV stack at
every stabilisation (the sweeps' order of props and the B products' order
agree), and a spinless t-V ring samples the exact Trotterised density and
kinetic energy (tests/_ed.py, trotter_tv_ring).
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(__file__))
from _cases import TEST_SEED0  # noqa: E402
from _ed import binned_mean, trotter_tv_ring  # noqa: E402

CASES = {
    "hc3_tv": dict(lattice=2, l1=3, l2=3, beta=1.0, dtau=0.1, rv=1.0, nflr=1, kinetic=0, update=1, nwrap=5,
                   nublock=4),
    "sq4_tuv_fft": dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.05, rhub=2.0, rv=1.0, mu=0.1, nflr=2, kinetic=1,
                        update=0, hs=0, nwrap=10),
    "ch6_tv_dense": dict(lattice=3, l1=6, l2=1, beta=1.0, dtau=0.1, rv=2.0, nflr=1, kinetic=2, update=2, nwrap=5,
                         nublock=8),
    "sq4_plq_tuv": dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.1, rhub=2.0, rv=0.6, rhub_plq=0.8, alpha=0.3,
                        theta=0.2, nflr=2, mu=0.1, kinetic=0, update=1, hs=1, nwrap=5, nublock=4),
}


@pytest.mark.parametrize("case", list(CASES))
def test_oracle_tv_sweeps_wrap_consistently(oracle, case):
    m = oracle.Model(**CASES[case])
    c = oracle.Chain(m, TEST_SEED0)
    c.sweep_start()
    v0 = c.vconf().copy()
    for _ in range(2):
        c.sweep_b0(); c.sweep_0b()
    d = c.diag()
    assert d["max_wrap_error"] < 1e-10
    assert 0 < d["accepted_v"] < d["proposed_v"]
    assert d["proposed_v"] == 4 * m.ltrot * m.nn_nf * m.nn_lf
    assert not np.array_equal(c.vconf(), v0)
    assert set(np.unique(c.vconf()[:, :, :m.nn_lf])) <= {1, 2}


def test_oracle_spinless_tv_ring_matches_exact_trotterised_values(oracle):
    """128 chains x 500 measured sweeps of the 6-site ring (V = 2, beta = 1,
    dtau = 0.1): the kinetic energy per site within four standard errors; the
    density is 1/2 by particle-hole symmetry."""
    L, V, beta, dtau, C = 6, 2.0, 1.0, 0.1, 128
    nx, kx = trotter_tv_ring(L, 1.0, V, beta, dtau)
    m = oracle.Model(lattice=3, l1=L, l2=1, beta=beta, dtau=dtau, rv=V, nflr=1, kinetic=0, update=1, nwrap=5,
                     nublock=4)
    ch = [oracle.Chain(m, TEST_SEED0 + 7 * c) for c in range(C)]
    for c in ch:
        c.sweep_start()
        for _ in range(20):
            c.sweep_b0(lmeasure=False); c.sweep_0b(lmeasure=False)
    ns, ks = [], []
    for _ in range(500):
        e = []
        for c in ch:
            c.obser_init(); c.sweep_b0(); c.sweep_0b()
            e.append(c.bins()["energy"])
        e = np.array(e)
        ns.append((e[:, 1].sum() / e[:, 0].sum()).real)
        ks.append((e[:, 2].sum() / e[:, 0].sum()).real / L)
    nm, _ = binned_mean(ns)
    km, ke = binned_mean(ks)
    assert abs(nx - 0.5) < 1e-12 and abs(nm - 0.5) < 1e-10
    assert abs(km - kx) < 4 * ke, (km, ke, kx)
