"""GPU parity of the projective (ground-state) path against the CPU oracle,
through the C ABI: dqmc_proj_sweep_start_0b, the submatrix-LR bond and site
updates, dqmc_proj_sweep_b0 / _0b with the mid-slice measurement.

The walker's trial state is taken from the oracle (zheev via scipy) and set
on the GPU handle, so both sides start from identical eigenvectors; the
library's own eigensolver is checked separately (CPU test of
dqmc_trial_state).  Tolerances: UR, UL, (UL UR)^-1 and G to 1e-9 relative to
their scale after whole sweeps (1e-11 after a single operator), HS fields and
accept counts exactly, bins to 1e-8.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# small t-V / Hubbard projective cases (configs 4 shape: honeycomb t-V,
# nflr = 1, ne = ndim/2, trial perturbed by rndness)
PCASES = {
    "hc3_tv": dict(lattice=2, l1=3, l2=3, beta=2.0, dtau=0.1, rv=1.0, rhub=0.0, nflr=1, kinetic=0,
                   nwrap=5, proj=1, rndness=1e-3, update=2),
    "hc3_tv_win8": dict(lattice=2, l1=3, l2=3, beta=2.0, dtau=0.1, rv=1.5, rhub=0.0, nflr=1, kinetic=0,
                        nwrap=4, proj=1, rndness=1e-3, update=2, nublock=8, obs_mid_len=3),
    "sq4_hub": dict(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.1, rv=0.0, rhub=4.0, nflr=2, kinetic=0,
                    nwrap=5, proj=1, rndness=0.05, update=2, hs=0, nublock=8, mu=0.0),
    "hc2_tuv": dict(lattice=2, l1=2, l2=2, beta=1.6, dtau=0.1, rv=0.8, rhub=2.0, nflr=2, kinetic=0,
                    nwrap=4, proj=1, rndness=0.05, update=2, hs=0, nublock=4),
    "sq4_tv_fft": dict(lattice=1, l1=4, l2=4, beta=1.5, dtau=0.05, rv=1.0, rhub=0.0, nflr=1, kinetic=1,
                       nwrap=10, proj=1, rndness=0.02, update=2),
    "hc3_tv_dense": dict(lattice=2, l1=3, l2=3, beta=2.0, dtau=0.1, rv=1.0, rhub=0.0, nflr=1, kinetic=2,
                         nwrap=5, proj=1, rndness=1e-3, update=2),
    # the plaquette field (dqmc_proj_update_plqu.f90) beside the U field, and beside both U and bond fields
    "sq4_hub_plq": dict(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.1, rv=0.0, rhub=3.0, nflr=2, kinetic=0,
                        nwrap=5, proj=1, rndness=0.05, update=2, hs=0, nublock=8, rhub_plq=0.8, alpha=0.3, theta=0.2),
    "hc2_tuv_plq": dict(lattice=2, l1=2, l2=2, beta=1.6, dtau=0.1, rv=0.8, rhub=2.0, nflr=2, kinetic=0,
                        nwrap=4, proj=1, rndness=0.05, update=2, hs=0, nublock=4, rhub_plq=0.6, alpha=0.25),
}


@pytest.fixture(scope="module")
def sb():
    import sunhubbardmy_b200 as sb
    return sb


def make_pair(sb, oracle, case, n_chains=1):
    kw = PCASES[case]
    p = sb.DqmcParams.make(**kw)
    g = sb.Dqmc(p, n_chains=n_chains, seeds=[sb.test_seed(c) for c in range(n_chains)])
    m = oracle.Model(**kw)
    ch = [oracle.Chain(m, sb.test_seed(c)) for c in range(n_chains)]
    for c in range(n_chains):
        P, _ = ch[c].trial()
        g.set_trial(P, c)
    return g, m, ch


def rel(a, b):
    return np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b)))


@pytest.mark.parametrize("case", list(PCASES))
def test_fields_and_trial_draws(sb, oracle, case):
    """The fresh-start draws (U field, bond field, trial hopping) follow the
    reference's order: both sides hold identical fields and equivalent trial
    subspaces."""
    kw = PCASES[case]
    p = sb.DqmcParams.make(**kw)
    g = sb.Dqmc(p, n_chains=2, seeds=[sb.test_seed(c) for c in range(2)])
    m = oracle.Model(**kw)
    for c in range(2):
        ch = oracle.Chain(m, sb.test_seed(c))
        if kw["rv"] != 0:
            assert np.array_equal(g.vconf(c), ch.vconf())
        if kw["rhub"] != 0:
            assert np.array_equal(g.conf(c), ch.conf())
        if kw.get("rhub_plq", 0.0):
            assert np.array_equal(g.conf_plq(c), ch.conf_plq())
        Pg, wg = g.trial(c)
        Po, wo = ch.trial()
        ne = p.ne
        assert np.max(np.abs(wg - wo)) < 1e-12
        prg = Pg[:, :ne] @ Pg[:, :ne].conj().T
        pro = Po[:, :ne] @ Po[:, :ne].conj().T
        assert np.max(np.abs(prg - pro)) < 1e-10


@pytest.mark.parametrize("case", list(PCASES))
def test_proj_sweep_start(sb, oracle, case):
    g, m, ch = make_pair(sb, oracle, case)
    g.sweep_start()
    ch[0].proj_sweep_start()
    ur, ul, li = g.proj_state(0)
    uro, ulo, lio = ch[0].proj_state()
    assert rel(ur, uro) < 1e-11
    assert rel(ul, ulo) < 1e-12
    assert rel(li, lio) < 1e-10
    dg, dc = g.diag(0), ch[0].diag()
    assert abs(dg["logweight"].real - dc["logweight"].real) < 1e-9 * max(1.0, abs(dc["logweight"].real))
    assert abs(dg["phase"] - dc["phase"]) < 1e-10
    # G = I - UR (UL UR)^-1 UL
    g.proj_green()
    assert np.max(np.abs(g.green(0) - ch[0].proj_green())) < 1e-10


@pytest.mark.parametrize("case", ["hc3_tv", "hc3_tv_win8", "sq4_hub", "hc2_tuv"])
def test_proj_update_operator(sb, oracle, case):
    """One proj_update (a whole bond family or all sites of a slice) from the
    sweep_start state: identical accept decisions, UR and (UL UR)^-1 close."""
    g, m, ch = make_pair(sb, oracle, case)
    g.sweep_start()
    ch[0].proj_sweep_start()
    kw = PCASES[case]
    nf_list = ([1, 2] if kw["rv"] != 0 else []) + ([0] if kw["rhub"] != 0 else [])
    nt = m.ltrot
    for nf in nf_list:
        g.proj_update(nt, nf)
        ch[0].proj_update(nt, nf)
        if kw["rv"] != 0:
            assert np.array_equal(g.vconf(0), ch[0].vconf())
        if kw["rhub"] != 0:
            assert np.array_equal(g.conf(0), ch[0].conf())
        ur, ul, li = g.proj_state(0)
        uro, ulo, lio = ch[0].proj_state()
        assert rel(ur, uro) < 1e-11
        assert rel(li, lio) < 1e-9
    dg, dc = g.diag(0), ch[0].diag()
    assert dg["accepted_v"] == dc["accepted_v"] and dg["proposed_v"] == dc["proposed_v"]
    assert dg["accepted"] == dc["accepted"] and dg["proposed"] == dc["proposed"]
    assert abs(dg["phase"] - dc["phase"]) < 1e-10


@pytest.mark.parametrize("update,flavour", [(0, "FAST"), (1, "DELAY"), (2, "SUBMATRIX_G_EXACT"), (2, "SUBMATRIX")])
@pytest.mark.parametrize("case", ["hc3_tv_win8", "sq4_hub", "hc2_tuv"])
def test_proj_update_flavours(sb, oracle, case, update, flavour):
    """A GPU handle built with update = fast (0), delay (1) or submatrix (2)
    against the oracle's restatement of the matching projective update
    (dqmc_proj_update.f90, dqmc_proj_update_delay.f90, the submatrix-G and
    submatrix-LR flavours) over every family of two slices: identical fields
    and accept counts, UR and (UL UR)^-1 to 1e-9.  (The submatrix-G bond
    update is taken with the exact inverse of the bond's 2 x 2 block; the
    reference's expressions differ in one entry, see test_oracle.)"""
    kw = dict(PCASES[case], update=update)
    p = sb.DqmcParams.make(**kw)
    g = sb.Dqmc(p, n_chains=1, seeds=[sb.test_seed(0)])
    m = oracle.Model(**kw)
    ch = oracle.Chain(m, sb.test_seed(0))
    g.set_trial(ch.trial()[0], 0)
    g.sweep_start(); ch.proj_sweep_start()
    nf_list = (list(range(1, m.nn_nf + 1)) if kw["rv"] != 0 else []) + ([0] if kw["rhub"] != 0 else [])
    f = getattr(oracle, flavour)
    for nt in (m.ltrot, m.ltrot - 1):
        for nf in nf_list:
            g.proj_update(nt, nf)
            ch.proj_update(nt, nf, flavour=f)
    if kw["rv"] != 0:
        assert np.array_equal(g.vconf(0), ch.vconf())
    if kw["rhub"] != 0:
        assert np.array_equal(g.conf(0), ch.conf())
    for x, y in zip(g.proj_state(0), ch.proj_state()):
        assert rel(x, y) < 1e-9
    dg, dc = g.diag(0), ch.diag()
    assert dg["accepted_v"] == dc["accepted_v"] and dg["accepted"] == dc["accepted"]
    g.close()


@pytest.mark.parametrize("case", list(PCASES))
def test_proj_sweeps_match_oracle(sb, oracle, case):
    """Two full sweeps (b0 + 0b) with updates and the mid-slice measurement."""
    g, m, ch = make_pair(sb, oracle, case, n_chains=2)
    kw = PCASES[case]
    g.sweep_start(); g.obser_init()
    for c in ch:
        c.proj_sweep_start(); c.obser_init()
    for _ in range(2):
        g.sweep_b0(); g.sweep_0b()
        for c in ch:
            c.proj_sweep_b0(); c.proj_sweep_0b()
    for k, c in enumerate(ch):
        if kw["rv"] != 0:
            assert np.array_equal(g.vconf(k), c.vconf()), k
        if kw["rhub"] != 0:
            assert np.array_equal(g.conf(k), c.conf()), k
        dg, dc = g.diag(k), c.diag()
        assert dg["accepted_v"] == dc["accepted_v"] and dg["accepted"] == dc["accepted"]
        if kw.get("rhub_plq", 0.0):
            assert np.array_equal(g.conf_plq(k), c.conf_plq()), k
            assert dg["accepted_plq"] == dc["accepted_plq"] and dg["proposed_plq"] == dc["proposed_plq"]
        assert dg["logcount"] == dc["logcount"]
        assert dg["max_wrap_error"] < 1e-8
        assert abs(dg["phase"] - dc["phase"]) < 1e-9
        ur, ul, li = g.proj_state(k)
        uro, ulo, lio = c.proj_state()
        assert rel(ur, uro) < 1e-9 and rel(ul, ulo) < 1e-9 and rel(li, lio) < 1e-8
        assert np.max(np.abs(g.green(k) - c.green())) < 1e-9
        eg, ec = g.bins(k)["energy"], c.bins()["energy"]
        assert np.max(np.abs(eg - ec)) < 1e-8 * max(1.0, np.max(np.abs(ec)))
        bg, bc = g.bins(k), c.bins()
        for name in ("cpcm", "spsm", "nn", "jj", "bb"):
            assert np.max(np.abs(bg[name] - bc[name])) < 1e-8 * max(1.0, np.max(np.abs(bc[name]))), name


def test_proj_graph_matches_stepwise(sb, oracle):
    """The captured-graph sweep replays the same launches as b0 + 0b."""
    kw = PCASES["hc3_tv"]
    p = sb.DqmcParams.make(**kw)
    a = sb.Dqmc(p, n_chains=2)
    b = sb.Dqmc(p, n_chains=2)
    for h in (a, b):
        h.sweep_start(); h.obser_init()
    a.sweeps(2, True)
    for _ in range(2):
        b.sweep_b0(); b.sweep_0b()
    for c in range(2):
        assert np.array_equal(a.vconf(c), b.vconf(c))
        assert np.max(np.abs(a.green(c) - b.green(c))) < 1e-12
        assert np.allclose(a.bins_raw(c), b.bins_raw(c), rtol=0, atol=1e-12)


# unequal-time window [ntauin, ntauin + ntdm] inside the projection (ltau): the
# measured 0b sweep runs dqmc_proj_dyn at nt = ntauin.  sq4_tv_fft starts the
# window between stabilisation points (ntauin = 5, nwrap = 10).
DYN = {"hc3_tv": 1.0, "sq4_hub": 1.0, "hc2_tuv": 0.8, "sq4_tv_fft": 1.0, "hc3_tv_dense": 1.0, "sq4_hub_plq": 1.0}


@pytest.mark.parametrize("case", list(DYN))
def test_proj_dyn_matches_oracle(sb, oracle, case):
    """znn_tau bins of the projective unequal-time pass against the oracle's
    restatement of dqmc_proj_dyn after two measured sweeps; the pass leaves the
    sweep itself (fields, G, equal-time bins) unchanged; the propagated
    G(t,t) agrees with the fresh one at the stabilisation points."""
    kw = dict(PCASES[case], ltau=1, dyntau=DYN[case])
    p = sb.DqmcParams.make(**kw)
    g = sb.Dqmc(p, n_chains=2, seeds=[sb.test_seed(c) for c in range(2)])
    m = oracle.Model(**kw)
    ch = [oracle.Chain(m, sb.test_seed(c)) for c in range(2)]
    for c in range(2):
        P, _ = ch[c].trial()
        g.set_trial(P, c)
    g.sweep_start(); g.obser_init()
    for c in ch:
        c.proj_sweep_start(); c.obser_init()
    for _ in range(2):
        g.sweep_b0(); g.sweep_0b()
        for c in ch:
            c.proj_sweep_b0(); c.proj_sweep_0b()
    for k, c in enumerate(ch):
        dg_, dc_ = g.dyn_bins(k), c.dyn_bins()
        assert np.max(np.abs(dc_)) > 0.0
        assert rel(dg_, dc_) < 1e-8
        dgk = g.diag(k)
        assert dgk["max_dyn_error"] < 1e-8 and c.max_dyn_error() < 1e-8
        assert dgk["dyn_count"] >= 2 and dgk["dyn_log10_sum"] / dgk["dyn_count"] < -8
        if kw["rv"] != 0:
            assert np.array_equal(g.vconf(k), c.vconf()), k
        if kw["rhub"] != 0:
            assert np.array_equal(g.conf(k), c.conf()), k
        ur, ul, li = g.proj_state(k)
        uro, ulo, lio = c.proj_state()
        assert rel(ur, uro) < 1e-9 and rel(ul, ulo) < 1e-9
        bg, bc = g.bins(k), c.bins()
        for name in ("energy", "cpcm", "nn", "jj"):
            assert np.max(np.abs(bg[name] - bc[name])) < 1e-8 * max(1.0, np.max(np.abs(bc[name]))), name


def test_proj_dyn_graph_matches_stepwise(sb):
    kw = dict(PCASES["hc3_tv"], ltau=1, dyntau=1.0)
    p = sb.DqmcParams.make(**kw)
    a = sb.Dqmc(p, n_chains=2)
    b = sb.Dqmc(p, n_chains=2)
    for h in (a, b):
        h.sweep_start(); h.obser_init()
    a.sweeps(2, True)
    for _ in range(2):
        b.sweep_b0(); b.sweep_0b()
    for c in range(2):
        assert np.allclose(a.dyn_bins(c), b.dyn_bins(c), rtol=0, atol=1e-12)


def test_proj_dyn_rejects_dyntau_beta(sb):
    kw = dict(PCASES["hc3_tv"], ltau=1, dyntau=PCASES["hc3_tv"]["beta"])
    with pytest.raises(Exception):
        sb.DqmcParams.make(**kw)
