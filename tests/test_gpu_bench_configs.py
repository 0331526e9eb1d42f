"""GPU parity at the benchmarked configurations, against the oracle.

The other parity tests use miniature lattices.  These run the oracle and the
GPU from the same seed at the shapes the benchmarks time:

* square 16 x 16, U = 4, beta = 10, dtau = 0.05, FFT kinetic term, general
  4-component HS field, delay depth 32: one full b0 + 0b sweep;
* honeycomb SU(4), U = 6, beta = 8, dtau = 0.1, exact HS field, submatrix
  depth 32, at L = 6, 9 and 12 (one chain of each size of the batched
  workload): one sweep;
* projective spinless t-V, honeycomb L = 12 (N = 288, ne = 144), theta = 20,
  dtau = 0.1, submatrix-LR depth 32: one walker, one sweep;
* square 4 x 4, U = 4, beta = 4, fast update, exact HS field: the full run
  of 200 warm-up and 1000 measured sweeps.

Bars: identical HS fields and accept counts; after every wrap check the
freshly computed G agrees with the oracle's to 1e-10 relative (the wrap trace
of both sides, the reference's -DTEST_LEVEL3 print of gf_tmp), except at the
projective shape, where the bar is the oracle's own spread between two LAPACK
implementations (see its test); the GPU's largest wrap error is within 2x of
the oracle's on the same field (each is printed); accept tests decided
within 1e-12 of their random number are counted on both sides and printed,
not altered.  For the full config-1 run,
the per-bin energies and double occupancy agree within one standard error
of the bin series (and, since the chains are identical, to rounding).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CONFIG2 = dict(lattice=1, l1=16, l2=16, beta=10.0, dtau=0.05, rhub=4.0, nflr=2, kinetic=1, update=1, hs=1,
               nwrap=10, nublock=32)
CONFIG1 = dict(lattice=1, l1=4, l2=4, beta=4.0, dtau=0.1, rhub=4.0, nflr=2, kinetic=0, update=0, hs=0, nwrap=10)
CONFIG4 = dict(lattice=2, l1=12, l2=12, beta=20.0, dtau=0.1, rv=1.0, rhub=0.0, nflr=1, kinetic=0, nwrap=10, proj=1,
               rndness=1e-3, update=2, nublock=32)


def config3(L):
    return dict(lattice=2, l1=L, l2=L, beta=8.0, dtau=0.1, rhub=6.0, nflr=4, kinetic=0, update=2, hs=0, nwrap=10,
                nublock=32)


def _compare_traces(tg, to, label):
    """Per wrap check: relative difference of the fresh G's, and the two wrap errors."""
    assert len(tg) == len(to) > 0, (len(tg), len(to))
    rel = [float(np.max(np.abs(a - b)) / np.max(np.abs(b))) for (a, _), (b, _) in zip(tg, to)]
    wg = max(e for _, e in tg)
    wo = max(e for _, e in to)
    print(f"{label}: {len(rel)} wrap checks, max rel |G_gpu - G_oracle| = {max(rel):.2e}, "
          f"max wrap error gpu {wg:.2e} oracle {wo:.2e}")
    return rel, wg, wo


def _run_ft(sb, oracle, kw, sweeps=1):
    p = sb.DqmcParams.make(**kw)
    g = sb.Dqmc(p, n_chains=1, seeds=[sb.test_seed(0)])
    m = oracle.Model(**kw)
    c = oracle.Chain(m, sb.test_seed(0))
    g.sweep_start(); c.sweep_start()
    g.obser_init(); c.obser_init()
    g.trace_wraps(2 * p.nst * sweeps)
    c.trace(2 * p.nst * sweeps)
    for _ in range(sweeps):
        g.sweep_b0(); g.sweep_0b()
        c.sweep_b0(); c.sweep_0b()
    return p, g, c


def _check_ft(g, c, label):
    dg, dc = g.diag(0), c.diag()
    print(f"{label}: accepted {dg['accepted']:.0f}/{dg['proposed']:.0f}, near ties gpu {dg['near_ties']} "
          f"oracle {dc['near_ties']}")
    assert np.array_equal(g.conf(0), c.conf()), f"{label}: HS fields differ (near ties: {dg['near_ties']})"
    assert dg["accepted"] == dc["accepted"] and dg["proposed"] == dc["proposed"]
    rel, wg, wo = _compare_traces(g.trace_get(0), c.trace_get(), label)
    assert max(rel) <= 1e-10
    assert wg <= 2.0 * wo + 1e-14
    assert abs(dg["phase"] - dc["phase"]) < 1e-9
    eg, ec = g.bins(0)["energy"], c.bins()["energy"]
    assert np.max(np.abs(eg - ec)) <= 1e-8 * np.max(np.abs(ec))


def test_config2_full_shape_one_sweep(sb, oracle):
    oracle.use_scipy_lapack(True)
    try:
        p, g, c = _run_ft(sb, oracle, CONFIG2)
    finally:
        oracle.use_scipy_lapack(False)
    _check_ft(g, c, "config2 square 16x16 beta=10 FFT delay 32")


@pytest.mark.parametrize("L", [6, 9, 12])
def test_config3_sizes_one_sweep(sb, oracle, L):
    oracle.use_scipy_lapack(True)
    try:
        p, g, c = _run_ft(sb, oracle, config3(L))
    finally:
        oracle.use_scipy_lapack(False)
    _check_ft(g, c, f"config3 honeycomb L={L} SU(4) beta=8 submatrix 32")


def _oracle_walker(oracle, lapack_scipy, nst):
    oracle.use_scipy_lapack(lapack_scipy)
    try:
        m = oracle.Model(**CONFIG4)
        c = oracle.Chain(m, 1909706392)
        c.proj_sweep_start()
        c.obser_init()
        c.trace(2 * nst)
        c.proj_sweep_b0(); c.proj_sweep_0b()
    finally:
        oracle.use_scipy_lapack(False)
    return m, c


def test_config4_walker_one_sweep(sb, oracle):
    """The projective walker at theta = 20: G = 1 - UR (UL UR)^-1 UL with a
    144 x 144 UL UR whose conditioning sets the floor of any two
    implementations' agreement.  The oracle run twice, once with scipy's
    LAPACK and once with its own restated LAPACK, already differs by ~2e-9 in
    G at some wrap checks and its wrap error moves between ~7e-10 and
    ~2e-9, so the 1e-10 bar of the square and honeycomb Hubbard shapes does not
    apply here.  The bars are therefore relative to that measured spread: the
    GPU's G is within max(1e-10, the oracle's largest two-LAPACK difference)
    of the oracle at every wrap check, and the GPU's largest wrap error is within 2x
    of the larger oracle wrap error.  Fields and accept counts stay exact."""
    p = sb.DqmcParams.make(**CONFIG4)
    assert sb.test_seed(0) == 1909706392
    m, c = _oracle_walker(oracle, True, p.nst)
    _, c2 = _oracle_walker(oracle, False, p.nst)
    g = sb.Dqmc(p, n_chains=1, seeds=[sb.test_seed(0)])
    g.set_trial(c.trial()[0])
    g.sweep_start()
    g.obser_init()
    g.trace_wraps(2 * p.nst)
    g.sweep_b0(); g.sweep_0b()
    dg, dc = g.diag(0), c.diag()
    label = "config4 t-V honeycomb L=12 ne=144 theta=20"
    print(f"{label}: accepted {dg['accepted_v']:.0f}/{dg['proposed_v']:.0f}, near ties gpu {dg['near_ties']} "
          f"oracle {dc['near_ties']}")
    assert np.array_equal(g.vconf(0), c.vconf()), f"{label}: bond fields differ (near ties: {dg['near_ties']})"
    assert np.array_equal(c2.vconf(), c.vconf())
    assert dg["accepted_v"] == dc["accepted_v"] and dg["proposed_v"] == dc["proposed_v"]
    to, to2 = c.trace_get(), c2.trace_get()
    spread = [float(np.max(np.abs(a - b)) / np.max(np.abs(b))) for (a, _), (b, _) in zip(to2, to)]
    rel, wg, wo = _compare_traces(g.trace_get(0), to, label)
    wo2 = max(e for _, e in to2)
    print(f"{label}: oracle two-LAPACK spread of G max {max(spread):.2e}, oracle wrap errors {wo:.2e} / {wo2:.2e}")
    assert max(rel) <= max(1e-10, max(spread))
    assert wg <= 2.0 * max(wo, wo2) + 1e-14
    assert abs(dg["phase"] - dc["phase"]) < 1e-9


def test_config1_full_run(sb, oracle):
    """200 warm-up and 1000 measured sweeps, 20 bins of 50 sweeps."""
    p = sb.DqmcParams.make(**CONFIG1)
    g = sb.Dqmc(p, n_chains=1, seeds=[sb.test_seed(0)])
    m = oracle.Model(**CONFIG1)
    c = oracle.Chain(m, sb.test_seed(0))
    g.sweep_start(); c.sweep_start()
    g.sweeps(200, False)
    for _ in range(200):
        c.sweep_b0(True, False); c.sweep_0b(True, False)
    eg, ec = [], []
    for _ in range(20):
        g.obser_init(); c.obser_init()
        g.sweeps(50, True)
        for _ in range(50):
            c.sweep_b0(); c.sweep_0b()
        eg.append(g.bins(0)["energy"]); ec.append(c.bins()["energy"])
    eg, ec = np.array(eg), np.array(ec)
    dg, dc = g.diag(0), c.diag()
    print(f"config1: near ties gpu {dg['near_ties']} oracle {dc['near_ties']}, "
          f"max wrap error gpu {dg['max_wrap_error']:.2e} oracle {dc['max_wrap_error']:.2e}")
    assert np.array_equal(g.conf(0), c.conf())
    assert dg["accepted"] == dc["accepted"]
    # per-bin estimates: kinetic energy (energy_bin(3)) and double occupancy
    # Re(energy_bin(4)) / Re(energy_bin(1)) / N (zint_u = sum_i Gc_ii^2)
    N = p.ndim
    for name, k in (("kinetic energy", 2), ("double occupancy", 3)):
        xg = (eg[:, k].real / eg[:, 0].real) / (N if k == 3 else 1.0)
        xo = (ec[:, k].real / ec[:, 0].real) / (N if k == 3 else 1.0)
        se = np.std(xo, ddof=1) / np.sqrt(len(xo))
        print(f"config1 {name}: gpu {xg.mean():.6f} oracle {xo.mean():.6f} +- {se:.6f}")
        assert abs(xg.mean() - xo.mean()) <= se
        assert np.max(np.abs(xg - xo)) <= 1e-8 * np.max(np.abs(xo))
    assert dg["max_wrap_error"] <= 2.0 * dc["max_wrap_error"] + 1e-14
