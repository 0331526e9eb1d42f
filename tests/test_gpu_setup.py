"""Device-side set-up: the batched Jacobi eigensolver (kern_eig.cu).

dqmc_gpu_create diagonalises every walker's trial Hamiltonian (set_trial_h0 /
dqmc_set_proj, s_eig_he = zheev in the reference) and, for the dense kinetic
term, the seth0 hopping matrix (dqmc_set_h0conf.f90:484-509) on the GPU.  The
checks are against the library's host eigensolver (dqmc_trial_state, itself
checked against LAPACK zheev in tests/test_host.py) and against the oracle's
dense kinetic operators (expm of the hopping matrix):

* eigenvalues to 1e-12 (relative to the spectrum's scale);
* the eigenvectors unitary to 1e-13 and the projector onto the ne lowest
  states equal to 1e-10 (the basis inside a degenerate level is free);
* urt = exp(-dtau H0 / 2) to 1e-12 through a dense-kinetic sweep's G.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TRIAL_CASES = [
    dict(lattice=2, l1=3, l2=3, beta=2.0, dtau=0.1, rv=1.0, nflr=1, nwrap=5, proj=1, rndness=1e-3),
    dict(lattice=2, l1=3, l2=3, beta=2.0, dtau=0.1, rv=1.0, nflr=1, nwrap=5, proj=1, rndness=0.3, flux_x=0.3, mu=0.1),
    dict(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.1, rhub=4.0, nflr=2, nwrap=5, proj=1, rndness=0.2, xmag=1.0),
    dict(lattice=1, l1=5, l2=4, beta=2.0, dtau=0.1, rhub=4.0, nflr=2, nwrap=5, proj=1, rndness=0.2, kinetic=2),
]


@pytest.mark.parametrize("kw", TRIAL_CASES)
def test_device_trial_states_match_host_eigensolver(sb, kw):
    p = sb.DqmcParams.make(**kw)
    seeds = [sb.test_seed(c) for c in range(3)]
    g = sb.Dqmc(p, n_chains=3, seeds=seeds)
    ne, N = p.ne, p.ndim
    for c, seed in enumerate(seeds):
        P, w = g.trial(c)
        Ph, wh = sb.trial_state(p, seed)
        scale = max(1.0, float(np.max(np.abs(wh))))
        assert np.max(np.abs(w - wh)) < 1e-12 * scale
        assert np.all(np.diff(w) >= 0)
        assert np.max(np.abs(P.conj().T @ P - np.eye(N))) < 1e-13
        d = np.max(np.abs(P[:, :ne] @ P[:, :ne].conj().T - Ph[:, :ne] @ Ph[:, :ne].conj().T))
        assert d < 1e-10, d
    g.close()


def test_device_trial_state_at_the_benchmarked_walker(sb):
    """Honeycomb L = 12 (N = 288, ne = 144), rndness 1e-3: the projector of the
    device eigensolver against the host one, with the level gap at ne printed."""
    kw = dict(lattice=2, l1=12, l2=12, beta=20.0, dtau=0.1, rv=1.0, rhub=0.0, nflr=1, kinetic=0, nwrap=10,
              proj=1, rndness=1e-3, update=2, nublock=32)
    p = sb.DqmcParams.make(**kw)
    g = sb.Dqmc(p, n_chains=2, seeds=[sb.test_seed(0), sb.test_seed(1)])
    ne = p.ne
    for c in range(2):
        P, w = g.trial(c)
        Ph, wh = sb.trial_state(p, sb.test_seed(c))
        gap = wh[ne] - wh[ne - 1]
        d = float(np.max(np.abs(P[:, :ne] @ P[:, :ne].conj().T - Ph[:, :ne] @ Ph[:, :ne].conj().T)))
        print(f"walker {c}: gap at ne {gap:.2e}, max |w - w_host| {np.max(np.abs(w - wh)):.2e}, projector {d:.2e}")
        assert np.max(np.abs(w - wh)) < 1e-12 * max(1.0, np.max(np.abs(wh)))
        # the projector is determined to about eps / gap
        assert d < max(1e-10, 1e-14 / gap), d
    g.close()


@pytest.mark.parametrize("kw", [
    dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.1, rhub=4.0, nflr=2, kinetic=2, nwrap=5),
    dict(lattice=2, l1=3, l2=3, beta=1.0, dtau=0.1, rhub=4.0, nflr=2, kinetic=2, nwrap=5, flux_x=0.3, mu=0.2),
    dict(lattice=1, l1=3, l2=3, beta=1.0, dtau=0.1, rhub=4.0, nflr=2, kinetic=2, nwrap=5, mu=0.1),   # odd N
])
def test_device_dense_kinetic_operator(sb, oracle, kw):
    """urt from the device eigensolver: G after sweep_start (B products with the
    dense kinetic term over all slices) agrees with the oracle's, whose urt is
    built from LAPACK-style host eigenpairs of the same hopping matrix."""
    p = sb.DqmcParams.make(**kw)
    g = sb.Dqmc(p, n_chains=1, seeds=[sb.test_seed(0)])
    m = oracle.Model(**kw)
    c = oracle.Chain(m, sb.test_seed(0))
    g.sweep_start(); c.sweep_start()
    err = float(np.max(np.abs(g.green(0) - c.green())))
    assert err < 1e-10, err
    g.close()
