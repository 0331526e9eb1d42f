"""The t-V bond field on the finite-temperature path, GPU against the oracle.

The field of dqmc_config_v (one Ising variable per bond and slice) enters the
finite-temperature sweeps as in dqmc_ft_sweep_0b.f90:96-106 and
dqmc_ft_sweep_b0.f90:79-90: per bond family the nflag = 2 step, the family's
bond-by-bond updates (dqmc_update.f90), then nflag = 1.  The cases here carry
the bond field alone (rhub = 0); the t-U-V cases of the shared parity table
run it beside the U field.  Checked: the bond field, G, the phase and the
acceptance counts after full sweeps, the bins, and the spinless ring's density
and kinetic energy against exact Trotterised values.
"""
import os
import sys

import numpy as np
import pytest

from tests._cases import rel_err

sys.path.insert(0, os.path.dirname(__file__))
from _ed import binned_mean, trotter_tv_ring  # noqa: E402

pytestmark = pytest.mark.gpu

TCASES = {
    "hc3_tv_cb_delay": dict(lattice=2, l1=3, l2=3, beta=1.0, dtau=0.1, rv=1.0, nflr=1, kinetic=0, update=1,
                            nwrap=5, nublock=4),
    "sq4_tv_fft_fast": dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.05, rv=1.5, nflr=1, mu=0.1, kinetic=1,
                            update=0, nwrap=10),
    "ch6_tv_dense_sub": dict(lattice=3, l1=6, l2=1, beta=1.0, dtau=0.1, rv=2.0, nflr=1, kinetic=2, update=2,
                             nwrap=5, nublock=8),
    "cu422_tv_cb_delay": dict(lattice=4, l1=4, l2=2, l3=2, beta=0.8, dtau=0.1, rv=1.0, nflr=1, kinetic=0,
                              update=1, nwrap=4, nublock=4),
    # a ragged last stabilisation interval (ltrot = 13, nwrap = 5) on a larger honeycomb, with the U field
    "hc6_tuv_ragged": dict(lattice=2, l1=6, l2=6, beta=1.3, dtau=0.1, rhub=2.0, rv=0.8, nflr=2, kinetic=0,
                           update=1, hs=1, nwrap=5, nublock=16),
    # a stabilisation after every slice
    "sq4_tv_nwrap1": dict(lattice=1, l1=4, l2=4, beta=0.4, dtau=0.1, rv=1.0, nflr=1, kinetic=1, update=2,
                          nwrap=1, nublock=8),
}


@pytest.fixture(scope="module")
def sb():
    import sunhubbardmy_b200 as sb
    return sb


@pytest.mark.parametrize("case", list(TCASES))
def test_tv_sweeps_match_oracle(sb, oracle, case):
    kw = TCASES[case]
    nch = 2
    g = sb.Dqmc(sb.DqmcParams.make(**kw), n_chains=nch, seeds=[sb.test_seed(c) for c in range(nch)])
    m = oracle.Model(**kw)
    ch = [oracle.Chain(m, sb.test_seed(c)) for c in range(nch)]
    for k in range(nch):
        assert np.array_equal(g.vconf(k), ch[k].vconf()), k
    g.sweep_start(); g.obser_init()
    for c in ch:
        c.sweep_start(); c.obser_init()
    for _ in range(2):
        g.sweep_b0(); g.sweep_0b()
        for c in ch:
            c.sweep_b0(); c.sweep_0b()
    for k in range(nch):
        assert np.array_equal(g.vconf(k), ch[k].vconf()), k
        assert np.max(np.abs(g.green(k) - ch[k].green())) < 1e-10
        dg, dc = g.diag(k), ch[k].diag()
        assert dg["accepted_v"] == dc["accepted_v"] and dg["proposed_v"] == dc["proposed_v"]
        assert 0 < dg["accepted_v"] < dg["proposed_v"]
        assert dg["max_wrap_error"] < 1e-10
        assert abs(dg["phase"] - dc["phase"]) < 1e-9
        bg, bc = g.bins(k), ch[k].bins()
        assert bg["nobs"] == bc["nobs"]
        for key in ("energy", "cpcm", "nn", "jj", "bb"):
            assert rel_err(bg[key], bc[key]) < 1e-8, key
    g.close()


def test_tv_vconf_roundtrip_and_sweep_from_set_field(sb, oracle):
    """A bond field written through set_vconf is the one the next sweep
    starts from (the same field in the oracle gives the same sweep)."""
    kw = TCASES["hc3_tv_cb_delay"]
    g = sb.Dqmc(sb.DqmcParams.make(**kw), n_chains=1, seeds=[sb.test_seed(5)])
    m = oracle.Model(**kw)
    c = oracle.Chain(m, sb.test_seed(5))
    rng = np.random.default_rng(3)
    v = g.vconf(0)
    v[...] = rng.integers(1, 3, v.shape, dtype=np.int32)
    g.set_vconf(v, 0)
    c.set_vconf(v)
    assert np.array_equal(g.vconf(0), v)
    g.sweep_start(); c.sweep_start()
    assert np.max(np.abs(g.green() - c.green())) < 1e-10
    g.sweep_b0(); c.sweep_b0()
    assert np.array_equal(g.vconf(0), c.vconf())
    assert np.max(np.abs(g.green() - c.green())) < 1e-10
    g.close()


def test_spinless_tv_ring_matches_exact_trotterised_values(sb):
    """6-site spinless t-V ring (V = 2, beta = 1, dtau = 0.1), 512 chains x 300
    measured sweeps: density and kinetic energy per site within four standard
    errors of Tr[B^Lt O] / Tr[B^Lt] (tests/_ed.py, trotter_tv_ring)."""
    L, V, beta, dtau, C = 6, 2.0, 1.0, 0.1, 512
    nx, kx = trotter_tv_ring(L, 1.0, V, beta, dtau)
    p = sb.DqmcParams.make(lattice=3, l1=L, l2=1, beta=beta, dtau=dtau, rv=V, nflr=1, kinetic=0, update=1,
                           nwrap=5, nublock=4)
    g = sb.Dqmc(p, n_chains=C, seeds=[sb.test_seed(c) for c in range(C)])
    g.sweep_start()
    g.sweeps(50, False)
    ns, ks, sg = [], [], []
    for _ in range(300):
        g.obser_init()
        g.sweeps(1, True)
        e = g.energy_all()
        ns.append(float((e[:, 1].sum() / e[:, 0].sum()).real))
        ks.append(float((e[:, 2].sum() / e[:, 0].sum()).real) / L)
        sg.append(float(e[:, 0].real.sum() / np.abs(e[:, 0]).sum()))
    g.close()
    nm, ne = binned_mean(ns)
    km, ke = binned_mean(ks)
    print(f"sign {np.mean(sg):.4f}: n {nm:.6f} +- {ne:.6f} (exact {nx:.6f}), "
          f"Ekin {km:.5f} +- {ke:.5f} (exact {kx:.5f})")
    assert abs(nm - nx) < max(4 * ne, 1e-10), (nm, ne, nx)
    assert abs(km - kx) < 4 * ke, (km, ke, kx)
