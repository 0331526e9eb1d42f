"""Unequal-time (dynamic) measurement on the GPU against the CPU oracle.

The pass of dqmc_sweep with ltau = 1 (src/dqmc_ft_ctrl.f90:97-101): push_stage,
a 0b sweep without updates that propagates G(tau,0) and G(0,tau) and
recomputes them with green_tau at every stabilisation, dyn_measure at every
time index, then pop_stage.  Checked: the znn_tau bins (relative 1e-9), the
final G(0,0), G(beta,0), G(0,beta) (1e-9 absolute, |G| = O(1)), and that the
chain state (G, HS field, the following 0b sweep) is restored exactly as the
oracle restores it.
"""
import numpy as np
import pytest

from tests._cases import rel_err

pytestmark = pytest.mark.gpu

DCASES = {
    "sq4_cb_exact": dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.1, rhub=4.0, nflr=2, kinetic=0, update=1, hs=0,
                         nwrap=5, nublock=4, ltau=1, dyntau=1.0),
    "sq4_fft_gen4": dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.05, rhub=4.0, nflr=2, kinetic=1, update=1, hs=1,
                         nwrap=10, nublock=4, ltau=1, dyntau=1.0),
    "hc3_su4": dict(lattice=2, l1=3, l2=3, beta=1.0, dtau=0.1, rhub=6.0, nflr=4, kinetic=0, update=2, hs=0,
                    nwrap=5, nublock=8, ltau=1, dyntau=1.0),
    "sq4_dense_gen4": dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.1, rhub=4.0, nflr=2, kinetic=2, update=1, hs=1,
                           nwrap=5, nublock=4, ltau=1, dyntau=1.0),
    # cubic lattice: znn_tau, zspsm_tau and gtau0 (dyn_measure3d.f90)
    "cu422_cb_gen4": dict(lattice=4, l1=4, l2=2, l3=2, beta=1.0, dtau=0.1, rhub=4.0, nflr=2, kinetic=0, update=1,
                          hs=1, nwrap=5, nublock=4, ltau=1, dyntau=0.6),
    # r_cubic: the same three observables summed over the orbital pairs
    "rc222_cb_gen4": dict(lattice=5, l1=2, l2=2, l3=2, beta=1.0, dtau=0.1, rhub=4.0, nflr=2, kinetic=0, update=1,
                          hs=1, nwrap=5, nublock=4, rtd=0.7, ltau=1, dyntau=0.6),
    # the plaquette field's blocks in the propagation of G(tau, 0) and G(0, tau)
    "sq4_plq_gen4": dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.1, rhub=4.0, nflr=2, kinetic=0, update=1, hs=1,
                         nwrap=5, nublock=4, rhub_plq=0.8, alpha=0.3, theta=0.2, ltau=1, dyntau=0.8),
    # the bond field's mix and scale steps in the same propagation
    "hc3_tuv_cb": dict(lattice=2, l1=3, l2=3, beta=1.0, dtau=0.1, rhub=2.0, rv=0.8, nflr=2, kinetic=0, update=1,
                       hs=1, nwrap=5, nublock=4, ltau=1, dyntau=1.0),
    "sq4_tv_fft": dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.05, rhub=0.0, rv=1.0, nflr=1, kinetic=1, update=1,
                       hs=1, nwrap=10, nublock=4, ltau=1, dyntau=0.5),
}


@pytest.fixture(scope="module")
def sb():
    import sunhubbardmy_b200 as sb
    return sb


@pytest.mark.parametrize("case", list(DCASES))
def test_dyn_pass_matches_oracle(sb, oracle, case):
    kw = DCASES[case]
    p = sb.DqmcParams.make(**kw)
    g = sb.Dqmc(p, n_chains=2, seeds=[sb.test_seed(c) for c in range(2)])
    m = oracle.Model(**kw)
    ch = [oracle.Chain(m, sb.test_seed(c)) for c in range(2)]
    g.sweep_start(); g.obser_init()
    for c in ch:
        c.sweep_start(); c.obser_init()
    g.sweep_b0(); [c.sweep_b0() for c in ch]
    g.sweep_dyn(); [c.sweep_dyn() for c in ch]
    for k in range(2):
        bg, bc = g.dyn_bins(k), ch[k].dyn_bins()
        assert bg.shape == bc.shape == (m.ntdm + 1, 2, 2, m.lq)
        assert rel_err(bg, bc) < 1e-9
        for a, b in zip(g.dyn_mats(k), ch[k].dyn_mats()):
            assert np.max(np.abs(a - b)) < 1e-9
        assert np.max(np.abs(g.green(k) - ch[k].green())) < 1e-10
        assert abs(g.diag(k)["phase"] - ch[k].diag()["phase"]) < 1e-9
    # the following 0b sweep with updates continues from the restored state
    g.sweep_0b(); [c.sweep_0b() for c in ch]
    for k in range(2):
        assert np.array_equal(g.conf(k), ch[k].conf())
        if kw.get("rv", 0.0):
            assert np.array_equal(g.vconf(k), ch[k].vconf())
        assert np.max(np.abs(g.green(k) - ch[k].green())) < 1e-10


def test_dyn_free_fermions_known_answer(sb):
    """U = 0: G(0,0) = (1 + B)^-1 and at tau = beta G(beta,0) = B G(0,0),
    G(0,beta) = -(1 - G(0,0)) B^-1, with B = exp(-beta K) from the library's own
    kinetic propagator applied to the identity."""
    kw = dict(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.1, rhub=0.0, nflr=2, kinetic=1, nwrap=5, ltau=1, dyntau=2.0)
    p = sb.DqmcParams.make(**kw)
    g = sb.Dqmc(p, n_chains=1)
    N = p.ndim
    g.set_green(np.eye(N, dtype=complex))
    for _ in range(p.ltrot):
        g.h0_prop(0, 1); g.h0_prop(0, 1)       # left_forward half steps: B = prod exp(-dtau K)
    B = g.green()
    g.sweep_start(); g.obser_init()
    g.sweep_b0()                            # the pass follows a b0 sweep (left factors in the stack)
    g.sweep_dyn()
    g00, gt0, g0t = g.dyn_mats()
    G0 = np.linalg.inv(np.eye(N) + B)
    assert np.max(np.abs(g00 - G0)) < 1e-11
    assert np.max(np.abs(gt0 - B @ G0)) < 1e-11
    assert np.max(np.abs(g0t + (np.eye(N) - G0) @ np.linalg.inv(B))) < 1e-9


def test_graph_sweeps_run_the_dyn_pass(sb, oracle):
    kw = DCASES["sq4_fft_gen4"]
    p = sb.DqmcParams.make(**kw)
    g1 = sb.Dqmc(p, n_chains=1, seeds=[sb.test_seed(0)])
    g2 = sb.Dqmc(p, n_chains=1, seeds=[sb.test_seed(0)])
    for g in (g1, g2):
        g.sweep_start(); g.obser_init()
    g1.sweeps(2, True)
    for _ in range(2):
        g2.sweep_b0(); g2.sweep_dyn(); g2.sweep_0b()
    assert np.array_equal(g1.conf(0), g2.conf(0))
    assert rel_err(g1.dyn_bins(0), g2.dyn_bins(0)) < 1e-12
    assert np.max(np.abs(g1.green() - g2.green())) < 1e-12
