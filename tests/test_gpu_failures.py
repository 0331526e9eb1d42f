"""Numerical-failure status of the sweep entry points, on the GPU.

The reference stops the run when a LAPACK call reports info /= 0
(lib/s_matrix.f90:1260-1267) or the Green's function inversion fails
(src/dqmc_ft_core/dqmc_ft_sweep_b0.f90:188-194).  The library reports those
points instead: DQMC_ENUMERIC for a singular or non-finite Green's function,
DQMC_EWRAP for a wrap error above the caller's tolerance, or, with
re-stabilisation on, a rebuild of the stack and G from the HS field.

The failures are made on the host, with ordinary data: a zeroed UDV stack
entry (a singular middle matrix M, whose QR has zero pivots), NaN entries in
G, or a tolerance no wrap check can meet.  NaN arithmetic does not fault the
GPU, and every kernel runs over its usual index ranges.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# beta = 2, dtau = 0.1, nwrap = 5: ltrot = 20, nst = 4 stabilisations per half sweep
SQ = dict(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.1, rhub=4.0, nflr=2, kinetic=0, update=1, hs=1, nwrap=5,
          nublock=8)


def _handle(sb, n_chains=2):
    p = sb.DqmcParams.make(**SQ)
    g = sb.Dqmc(p, n_chains=n_chains, seeds=[sb.test_seed(c) for c in range(n_chains)])
    g.sweep_start()
    return g, p


def _zero_entry(g, p, n, c):
    z = np.zeros((p.ndim, p.ndim), complex)
    g.set_stack(n, u=z, v=z, c=c)


def test_stack_accessors_round_trip(sb):
    g, p = _handle(sb)
    u, d, v, ld = g.stack(2, c=1)
    assert np.max(np.abs(u.conj().T @ u - np.eye(p.ndim))) < 1e-12    # U is unitary
    g.set_stack(2, u=u, d=d, v=v, logdetq=ld, c=1)
    u2, d2, v2, ld2 = g.stack(2, c=1)
    assert np.array_equal(u, u2) and np.array_equal(d, d2) and np.array_equal(v, v2) and ld == ld2


def test_singular_green_returns_enumeric(sb):
    """A zeroed right factor makes M = 0 in green_equaltime at that
    stabilisation of the b0 sweep: the call returns DQMC_ENUMERIC, only the
    broken chain carries the code, and its G stays the propagated one."""
    g, p = _handle(sb)
    _zero_entry(g, p, 2, c=1)
    with pytest.raises(sb.DqmcError) as e:
        g.sweep_b0(True, False)
    assert e.value.code == sb.ENUMERIC
    assert g.diag(1)["info"] & sb.FAIL_SINGULAR
    assert g.diag(0)["info"] == 0
    assert np.all(np.isfinite(g.green(1)))
    assert np.isfinite(g.diag(1)["logweight"].real)
    # the zeroed entry was replaced by the b0 sweep's new left factor, so the
    # next half sweep runs clean
    g.reset_diag()
    g.sweep_0b(True, False)
    assert g.diag(1)["info"] == 0 and g.diag(1)["max_wrap_error"] < 1e-8


def test_restabilisation_rebuilds_from_the_field(sb):
    """With re-stabilisation on, the same failure in a 0b sweep is repaired:
    the call succeeds and G equals a fresh sweep_start of the current field."""
    g, p = _handle(sb)
    g.set_checks(0.0, True)
    g.sweep_b0(True, False)
    _zero_entry(g, p, 2, c=0)            # a left factor used by the 0b sweep
    g.sweep_0b(True, False)
    d = g.diag(0)
    assert d["restabilized"] == 1 and d["info"] & sb.FAIL_SINGULAR
    ref = sb.Dqmc(p, n_chains=1, seeds=[sb.test_seed(0)])
    ref.set_conf(g.conf(0))
    ref.sweep_start()
    assert np.max(np.abs(g.green(0) - ref.green(0))) < 1e-10
    assert abs(g.diag(0)["phase"] - ref.diag(0)["phase"]) < 1e-10


def test_wrap_tolerance_returns_ewrap(sb):
    g, p = _handle(sb)
    g.set_checks(1e-30)                  # no wrap check can meet this
    with pytest.raises(sb.DqmcError) as e:
        g.sweeps(1, False)
    assert e.value.code == sb.EWRAP
    assert g.diag(0)["info"] == sb.FAIL_WRAP and g.diag(1)["info"] == sb.FAIL_WRAP
    g.set_checks(1e-6)
    g.reset_diag()
    g.sweeps(2, False)
    assert g.diag(0)["info"] == 0 and g.diag(0)["max_wrap_error"] < 1e-6


def test_nan_green_is_replaced_at_the_next_stabilisation(sb):
    """NaN in the propagated G: the updates reject every proposal until the
    next stabilisation replaces G by the fresh one.  Without a tolerance the
    call succeeds; with one, the non-finite wrap error is reported."""
    g, p = _handle(sb)
    bad = np.full((p.ndim, p.ndim), np.nan + 0j)
    g.set_green(bad, c=0)
    g.sweep_b0(True, False)
    assert np.all(np.isfinite(g.green(0)))
    g.set_checks(1e-6)
    g.set_green(bad, c=1)
    with pytest.raises(sb.DqmcError) as e:
        g.sweep_0b(True, False)
    assert e.value.code == sb.EWRAP and g.diag(1)["info"] & sb.FAIL_WRAP
    assert np.all(np.isfinite(g.green(1)))


def test_projective_singular_ulr_returns_enumeric(sb):
    kw = dict(lattice=2, l1=3, l2=3, beta=2.0, dtau=0.1, rv=1.0, rhub=0.0, nflr=1, kinetic=0, nwrap=5, proj=1,
              rndness=1e-3, update=2, nublock=8)
    p = sb.DqmcParams.make(**kw)
    g = sb.Dqmc(p, n_chains=1)
    g.sweep_start()
    ur, ul, inv = g.proj_state(0)
    g.set_proj_state(np.zeros_like(ur), ul, inv, c=0)
    with pytest.raises(sb.DqmcError) as e:
        g.proj_green()
    assert e.value.code == sb.ENUMERIC and g.diag(0)["info"] & sb.FAIL_SINGULAR
