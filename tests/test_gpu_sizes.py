"""Edge sizes on the GPU against the oracle: the largest supported lattice
(honeycomb 16 x 16, N = 512, the shared-memory limit of the per-chain
kernels), a stabilisation interval that does not divide ltrot (ragged last
interval), a single time slice per interval (nwrap = 1), and long
intervals whose B(tau2, tau1) products hold more propagation ops than one
launch takes (nwrap = 40: 9 ops per checkerboard slice on the square lattice,
7 on the honeycomb one), so the product runs as several launches."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = {
    "hc16_n512": dict(lattice=2, l1=16, l2=16, beta=0.4, dtau=0.1, rhub=4.0, nflr=2, kinetic=0, update=1, hs=0,
                      nwrap=2, nublock=32),
    "sq4_ragged_wrap": dict(lattice=1, l1=4, l2=4, beta=1.3, dtau=0.1, rhub=4.0, nflr=2, kinetic=0, update=1, hs=1,
                            nwrap=5, nublock=8),
    "sq4_nwrap1": dict(lattice=1, l1=4, l2=4, beta=0.5, dtau=0.1, rhub=4.0, nflr=2, kinetic=1, update=1, hs=0,
                       nwrap=1, nublock=4),
    "sq4_cb_nwrap40": dict(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.05, rhub=2.0, nflr=2, kinetic=0, update=1,
                           hs=1, nwrap=40, nublock=8),
    "hc3_cb_nwrap40": dict(lattice=2, l1=3, l2=3, beta=2.0, dtau=0.05, rhub=2.0, nflr=2, kinetic=0, update=2,
                           hs=0, nwrap=40, nublock=8),
}


@pytest.mark.parametrize("case", list(SIZES))
def test_sweeps_at_edge_sizes(sb, oracle, case):
    kw = SIZES[case]
    p = sb.DqmcParams.make(**kw)
    g = sb.Dqmc(p, n_chains=1, seeds=[sb.test_seed(0)])
    m = oracle.Model(**kw)
    c = oracle.Chain(m, sb.test_seed(0))
    g.sweep_start(); c.sweep_start()
    assert np.max(np.abs(g.green() - c.green())) < 1e-9
    g.obser_init(); c.obser_init()
    g.sweep_b0(); g.sweep_0b()
    c.sweep_b0(); c.sweep_0b()
    assert np.array_equal(g.conf(0), c.conf())
    assert np.max(np.abs(g.green() - c.green())) < 1e-9
    assert g.diag()["max_wrap_error"] < 1e-9
    bg, bc = g.bins(0), c.bins()
    assert np.max(np.abs(bg["energy"] - bc["energy"])) < 1e-8 * max(1.0, np.max(np.abs(bc["energy"])))
