"""The plaquette Hubbard-Stratonovich field (hconf, src/dqmc_config_plqu/),
checked on the CPU: the oracle's free-fermion Green's function with the
plaquette blocks against (1 + B^Lt)^-1 built here from the reference's
plaquette matrix, the order of the fresh-start draws (plaquette field before
the U field, dqmc_ft_ctrl.f90:19-29), the consistency of its sweeps (the wrap
error of an update-modified G against the recomputed one) and the library's
parameter checks.
"""
import numpy as np
import pytest
from scipy.linalg import expm

ETA = [-np.sqrt(2 * (3 + np.sqrt(6))), -np.sqrt(2 * (3 - np.sqrt(6))), np.sqrt(2 * (3 - np.sqrt(6))),
       np.sqrt(2 * (3 + np.sqrt(6)))]


def vstmat(z, nnf, alpha, theta):
    """dqmc_set_plqconf.f90:50-67: the Fortran reshape of the listed values."""
    z0, z1, z1h = 1.0 / nnf, alpha * np.exp(-1j * theta), alpha * np.exp(1j * theta)
    if z == 4:
        cols = [[z0, z1, 0, -z1], [z1h, z0, -z1h, 0], [0, -z1, z0, z1], [-z1h, 0, z1h, z0]]
    else:
        cols = [[z0, z1, 0, 0, 0, -z1], [z1h, z0, -z1h, 0, 0, 0], [0, -z1, z0, z1, 0, 0],
                [0, 0, z1h, z0, -z1h, 0], [0, 0, 0, -z1, z0, z1], [-z1h, 0, 0, 0, z1h, z0]]
    return np.array(cols, complex).T


CASES = [dict(lattice=1, l1=4, l2=4, nnf=4), dict(lattice=2, l1=3, l2=3, nnf=3)]


@pytest.mark.parametrize("case", CASES, ids=["square", "honeycomb"])
def test_plaquette_free_fermion_green(oracle, case):
    """U = 0: G = (1 + B^Lt)^-1 with the slice B = K1..Knnf P_lq..P_1 Knnf..K1,
    P_i the block exp(i alpha_p eta(s) vstmat) on plaquette i's sites."""
    dtau, beta, mu, rp, alpha, theta = 0.1, 0.6, 0.2, 0.7, 0.3, 0.25
    kw = dict(lattice=case["lattice"], l1=case["l1"], l2=case["l2"], beta=beta, dtau=dtau, rhub=0.0, mu=mu,
              rhub_plq=rp, alpha=alpha, theta=theta, nflr=2, kinetic=2, nwrap=3)
    m = oracle.Model(**kw)
    c = oracle.Chain(m, 9)
    c.sweep_start()
    N, lq, lt = m.ndim, m.lq, m.ltrot
    t = m.tables()
    H = m.h0mat()
    K = expm(-0.5 * dtau * H)
    v = vstmat(t["plq_cord"].shape[1], case["nnf"], alpha, theta * np.pi)
    ap = np.sqrt(dtau * rp)
    cp = c.conf_plq()
    B = np.eye(N, dtype=complex)
    for nt in range(lt):
        P = np.eye(N, dtype=complex)
        for i in range(lq):
            E = np.eye(N, dtype=complex)
            idx = t["plq_cord"][i] - 1
            E[np.ix_(idx, idx)] = expm(1j * ap * ETA[cp[nt, i] - 1] * v)
            P = E @ P
        B = (K @ P @ K) @ B
    G = np.linalg.inv(np.eye(N) + B)
    assert np.max(np.abs(c.green() - G)) < 1e-12


def test_plaquette_field_is_drawn_before_the_u_field(oracle):
    kw = dict(lattice=1, l1=4, l2=4, beta=0.5, dtau=0.1, rhub=4.0, rhub_plq=1.0, nflr=2, hs=1, nwrap=5)
    m = oracle.Model(**kw)
    c = oracle.Chain(m, 21)
    bare = oracle.Chain(oracle.Model(**dict(kw, rhub=0.0, rhub_plq=0.0)), 21)   # draws nothing at start
    lt, lq, N = m.ltrot, m.lq, m.ndim
    r = np.array([bare.uniform() for _ in range(lt * lq + lt * N)])
    assert np.array_equal(c.conf_plq().ravel(), np.ceil(r[:lt * lq] * 4).astype(int))
    assert np.array_equal(c.conf().ravel(), np.ceil(r[lt * lq:] * m.lcomp).astype(int))


@pytest.mark.parametrize("case", CASES, ids=["square", "honeycomb"])
def test_plaquette_sweeps_keep_the_wrap_error_small(oracle, case):
    """The rank-z plaquette updates and props of the sweeps against the B
    products of the stabilisation: the wrap error stays at rounding level."""
    kw = dict(lattice=case["lattice"], l1=case["l1"], l2=case["l2"], beta=1.0, dtau=0.1, rhub=3.0, rhub_plq=1.0,
              alpha=0.3, theta=0.2, nflr=2, hs=1, kinetic=0, update=0, nwrap=5)
    c = oracle.Chain(oracle.Model(**kw), 4)
    c.sweep_start()
    for _ in range(2):
        c.sweep_b0(); c.sweep_0b()
    d = c.diag()
    assert d["proposed_plq"] == 4 * c.model.lq * c.model.ltrot
    assert 0 < d["accepted_plq"] < d["proposed_plq"]
    assert d["max_wrap_error"] < 1e-10


def test_plaquette_parameter_checks():
    import sunhubbardmy_b200 as sb
    base = dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.1, rhub=4.0, rhub_plq=1.0, nwrap=5)
    assert sb.DqmcParams.make(**base).rhub_plq == 1.0
    assert sb.DqmcParams.make(**dict(base, proj=1)).proj == 1       # the projective path takes it too
    assert sb.DqmcParams.make(**dict(base, ltau=1, dyntau=0.5)).ltau == 1   # and the unequal-time pass
    for bad in (dict(lattice=3, l2=1), dict(lattice=4, l3=2), dict(rhub_plq=-1.0)):
        with pytest.raises(sb.DqmcError):
            sb.DqmcParams.make(**dict(base, **bad))
    g = sb.read_dqmc_in("&model_para\nla = 4,\nlb = 4,\nrhub_plq = 0.5,\nlprojplqu = .true.,\n/\n&ctrl_para\n/\n")
    assert g["rhub_plq"] == 0.5 and g["lprojplqu"] == 1


def test_projective_plaquette_sweeps_keep_the_wrap_error_small(oracle):
    """dqmc_proj_update_plqu.f90: the rank-z changes of UR and (UL UR)^-1 agree
    with their recomputation at the stabilisations."""
    kw = dict(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.1, rhub=2.0, rhub_plq=0.8, alpha=0.3, theta=0.2, nflr=2,
              hs=1, kinetic=0, update=2, nwrap=5, proj=1, rndness=0.1)
    c = oracle.Chain(oracle.Model(**kw), 13)
    c.proj_sweep_start()
    for _ in range(2):
        c.proj_sweep_b0(); c.proj_sweep_0b()
    d = c.diag()
    assert 0 < d["accepted_plq"] < d["proposed_plq"] == 4 * 16 * 20
    assert d["max_wrap_error"] < 1e-10
