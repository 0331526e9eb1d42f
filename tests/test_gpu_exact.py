"""GPU against exact Trotterised values: an independent pin of the library.

DQMC samples the Trotterised partition function Tr B^Lt exactly (the discrete
HS decoupling is an identity), so its equal-time averages must match
Tr[B^Lt O] / Tr[B^Lt] computed in Fock space (tests/_ed.py) within statistical
error alone.  Checked here for a 6-site SU(2) Hubbard ring (chain lattice,
U = 4, beta = 2, dtau = 0.1, exact HS field) with the checkerboard and the dense
kinetic term: double occupancy and kinetic energy per site, from 512 chains x
300 measured sweeps, within four standard errors (about 0.5% of the value).

The repulsive U is decoupled in the charge channel with an imaginary coupling,
so a configuration's G_ii = 1/2 + i y has an unbounded imaginary part near a
zero of det(1 + B), and the per-configuration estimators (1 - G_ii)^2 are heavy
tailed (one sample of the double occupancy in 150000 is -852).  The binned
error bars include those samples; the last test checks that the GPU reproduces
such a sample of the oracle's to ten digits.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(__file__))
from _ed import binned_mean, trotter_ring  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kinetic,update", [(0, 0), (2, 1), (0, 2)])
def test_hubbard_ring_matches_exact_trotterised_values(sb, kinetic, update):
    L, U, beta, dtau, C = 6, 4.0, 2.0, 0.1, 512
    Dx, Kx = trotter_ring(L, 1.0, U, beta, dtau, dense=kinetic == 2)
    p = sb.DqmcParams.make(lattice=3, l1=L, l2=1, beta=beta, dtau=dtau, rhub=U, nflr=2, kinetic=kinetic,
                           update=update, hs=0, nwrap=10, nublock=4)
    g = sb.Dqmc(p, n_chains=C, seeds=[sb.test_seed(c) for c in range(C)])
    g.sweep_start()
    g.sweeps(100, False)
    ds, ks = [], []
    for _ in range(300):
        g.obser_init()
        g.sweeps(1, True)
        e = g.energy_all()
        ds.append(float(np.mean((e[:, 3] / e[:, 0]).real)) / L)
        ks.append(float(np.mean((e[:, 2] / e[:, 0]).real)) / L)
    g.close()
    dm, de = binned_mean(ds)
    km, ke = binned_mean(ks)
    print(f"kinetic {kinetic} update {update}: D {dm:.5f} +- {de:.5f} (exact {Dx:.5f}), "
          f"Ekin {km:.5f} +- {ke:.5f} (exact {Kx:.5f})")
    assert abs(dm - Dx) < 4 * de, (dm, de, Dx)
    assert abs(km - Kx) < 4 * ke, (km, ke, Kx)


def test_heavy_tailed_sample_matches_oracle(sb, oracle):
    """Chain 76 (seed test_seed(76)) of the dense-kinetic ring: its measured
    sweeps 100..155, the last holding a double-occupancy sample of about -852,
    agree with the oracle's chain of the same seed to 1e-9 relative."""
    L, kw = 6, dict(lattice=3, l1=6, l2=1, beta=2.0, dtau=0.1, rhub=4.0, nflr=2, kinetic=2, update=0, hs=0,
                    nwrap=10, nublock=4)
    C, ch = 80, 76
    g = sb.Dqmc(sb.DqmcParams.make(**kw), n_chains=C, seeds=[sb.test_seed(c) for c in range(C)])
    c = oracle.Chain(oracle.Model(**kw), sb.test_seed(ch))
    g.sweep_start(); c.sweep_start()
    g.sweeps(100, False)
    for _ in range(100):
        c.sweep_b0(lmeasure=False); c.sweep_0b(lmeasure=False)
    for s in range(56):
        g.obser_init(); g.sweeps(1, True)
        c.obser_init(); c.sweep_b0(lmeasure=True); c.sweep_0b(lmeasure=True)
        eg, eo = g.energy_all()[ch], c.bins()["energy"]
        for k in (0, 2, 3):
            assert abs(eg[k] - eo[k]) <= 1e-9 * max(1.0, abs(eo[k])), (s, k, eg[k], eo[k])
    assert (eo[3] / eo[0]).real / L < -800.0
    g.close()
