"""Batched chains of uneven lattice sizes in one handle (one CTA per chain),
each chain checked against its own oracle chain: identical HS fields and
accept counts, Green's functions within 1e-10, energy bins within 1e-8."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GROUPS = {
    "honeycomb_su4_L2_L3": [
        (dict(lattice=2, l1=2, l2=2, beta=1.6, dtau=0.1, rhub=6.0, nflr=4, kinetic=0, update=2, hs=0, nwrap=8, nublock=16), 3),
        (dict(lattice=2, l1=3, l2=3, beta=1.6, dtau=0.1, rhub=6.0, nflr=4, kinetic=0, update=2, hs=0, nwrap=8, nublock=32), 2),
    ],
    "square_fft_L4_L6": [
        (dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.05, rhub=4.0, nflr=2, kinetic=1, update=1, hs=1, nwrap=10, nublock=8), 2),
        (dict(lattice=1, l1=6, l2=6, beta=1.0, dtau=0.05, rhub=4.0, nflr=2, kinetic=1, update=1, hs=1, nwrap=10, nublock=16), 2),
    ],
}


@pytest.mark.parametrize("name", list(GROUPS))
def test_mixed_sizes_match_oracle(oracle, name):
    import sunhubbardmy_b200 as sb
    plist, kws = [], []
    for kw, n in GROUPS[name]:
        plist += [sb.DqmcParams.make(**kw)] * n
        kws += [kw] * n
    nch = len(plist)
    g = sb.Dqmc(plist, n_chains=nch, seeds=[sb.test_seed(c) for c in range(nch)])
    models = {}
    chains = []
    for c, kw in enumerate(kws):
        key = tuple(sorted(kw.items()))
        if key not in models:
            models[key] = oracle.Model(**kw)
        chains.append(oracle.Chain(models[key], sb.test_seed(c)))
    g.sweep_start(); g.obser_init()
    for ch in chains:
        ch.sweep_start(); ch.obser_init()
    g.sweeps(1, True)
    for ch in chains:
        ch.sweep_b0(); ch.sweep_0b()
    for c, ch in enumerate(chains):
        assert g.ndim(c) == ch.model.ndim
        assert np.array_equal(g.conf(c), ch.conf()), c
        assert np.max(np.abs(g.green(c) - ch.green())) < 1e-10
        dg, dc = g.diag(c), ch.diag()
        assert dg["accepted"] == dc["accepted"]
        eg, ec = g.bins(c)["energy"], ch.bins()["energy"]
        assert np.max(np.abs(eg - ec)) < 1e-8 * max(1.0, np.max(np.abs(ec)))


def test_autotuner_keeps_results(oracle):
    """The tuned flush depth changes only the speed: the tuned handle's chains
    still reproduce the oracle."""
    import sunhubbardmy_b200 as sb
    from sunhubbardmy_b200.autotune import batched
    kw = dict(lattice=2, l1=3, l2=3, beta=1.6, dtau=0.1, rhub=6.0, nflr=4, kinetic=0, update=2, hs=0, nwrap=8, nublock=32)
    g, report = batched([(sb.DqmcParams.make(**kw), 2)], candidates=(8, 16), tune_chains=2)
    assert report[18]["nublock"] in (8, 16)
    m = oracle.Model(**kw)
    ch = oracle.Chain(m, sb.test_seed(0))
    g.sweep_start(); ch.sweep_start()
    g.sweep_b0(); g.sweep_0b(); ch.sweep_b0(); ch.sweep_0b()
    assert np.array_equal(g.conf(0), ch.conf())
    assert np.max(np.abs(g.green(0) - ch.green())) < 1e-10


def test_concurrent_handles_equal_separate_sweeps(sb):
    """dqmc_gpu_sweeps_multi runs each handle's captured sweep on its own
    stream; the chains evolve exactly as with dqmc_gpu_sweeps one handle at a
    time."""
    kw = dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.05, rhub=4.0, nflr=2, kinetic=1, update=1, hs=1,
              nwrap=10, nublock=8)
    p = sb.DqmcParams.make(**kw)
    a = [sb.Dqmc(p, n_chains=2, seeds=[sb.test_seed(2 * k + c) for c in range(2)]) for k in range(2)]
    b = [sb.Dqmc(p, n_chains=2, seeds=[sb.test_seed(2 * k + c) for c in range(2)]) for k in range(2)]
    for g in a + b:
        g.sweep_start(); g.obser_init()
    ms = sb.sweeps_concurrent(a, 2, True)
    assert ms > 0
    for g in b:
        g.sweeps(2, True)
    for ga, gb in zip(a, b):
        for c in range(2):
            assert np.array_equal(ga.conf(c), gb.conf(c))
            assert np.max(np.abs(ga.green(c) - gb.green(c))) == 0.0
            assert np.array_equal(ga.bins_raw(c), gb.bins_raw(c))


@pytest.mark.parametrize("name", list(GROUPS))
@pytest.mark.parametrize("split", [1, 2])
def test_size_classes_on_streams_equal_one_handle(name, split):
    """The size classes as concurrent handles (autotune.size_classes) give the
    chains of one handle of all of them (autotune.batched), same seeds: the same
    HS fields and accept counts, Green's functions and bins equal to rounding
    (one handle of mixed square sizes propagates with the generic pass, a
    handle of one size with its size's register FFT pass); the whole-field
    accessors keep the chain order."""
    import sunhubbardmy_b200 as sb
    from sunhubbardmy_b200.autotune import batched, size_classes
    groups = [(sb.DqmcParams.make(**kw), n) for kw, n in GROUPS[name]]
    one, _ = batched(groups, tune=False, seed0=5)
    grp, _ = size_classes(groups, tune=False, seed0=5, split=split)
    assert grp.n_chains == one.n_chains
    assert len(grp.handles) == sum(min(split, n) for _, n in groups)
    for g in (one, grp):
        g.sweep_start(); g.obser_init()
        g.sweeps(2, True)
    for c in range(one.n_chains):
        assert grp.ndim(c) == one.ndim(c)
        assert np.array_equal(grp.conf(c), one.conf(c)), c
        assert np.max(np.abs(grp.green(c) - one.green(c))) < 1e-12, c
        bg, bo = grp.bins_raw(c), one.bins_raw(c)
        assert np.max(np.abs(bg - bo)) <= 1e-10 * max(1.0, np.max(np.abs(bo))), c
        dg, do = grp.diag(c), one.diag(c)
        assert dg["accepted"] == do["accepted"] and abs(dg["phase"] - do["phase"]) < 1e-12, c
    ca = grp.conf_all()
    assert np.array_equal(ca, one.conf_all())
    ca2 = ca.copy()
    ca2[::7] = 1
    grp.set_conf_all(ca2)
    assert np.array_equal(grp.conf_all(), ca2)
    assert grp.sweep_kernels() > 0
    grp.close()
    one.close()
