"""Shared parameter sets and helpers for the parity tests.

The cases are small versions of the benchmark configurations (square Hubbard
with checkerboard, FFT or dense kinetic term, exact or general HS field;
honeycomb SU(4); the 1D chain; the cubic and r_cubic lattices; the plaquette field; the t-V bond
field) sized so the
oracle finishes each in well under a second.
"""
import numpy as np

# keyword sets accepted by both sunhubbardmy_b200.DqmcParams.make and
# oracle.pyoracle.Model (same names as dqmc.in)
CASES = {
    "sq4_cb_exact_fast": dict(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.1, rhub=4.0, nflr=2,
                              kinetic=0, update=0, hs=0, nwrap=10),
    "sq4_fft_gen4_delay": dict(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.05, rhub=4.0, nflr=2,
                               kinetic=1, update=1, hs=1, nwrap=10, nublock=4),
    "hc3_cb_su4_sub": dict(lattice=2, l1=3, l2=3, beta=2.0, dtau=0.1, rhub=6.0, nflr=4,
                           kinetic=0, update=2, hs=0, nwrap=10, nublock=8),
    "sq6_cb_gen4_delay_mu": dict(lattice=1, l1=6, l2=6, beta=1.5, dtau=0.1, rhub=3.0, nflr=2, mu=0.3,
                                 kinetic=0, update=1, hs=1, nwrap=5, nublock=8),
    # FFT kinetic term on 8 x 8 and 16 x 16 (the register-resident FFT pass)
    "sq8_fft_exact_delay": dict(lattice=1, l1=8, l2=8, beta=1.0, dtau=0.05, rhub=4.0, nflr=2, mu=0.2,
                                kinetic=1, update=1, hs=0, nwrap=10, nublock=16),
    # (U = 2 with mu = 0.3 keeps I + B(beta, 0) of the random start well conditioned
    # at this size, so G itself is accurate to ~1e-12)
    "sq16_fft_gen4_delay": dict(lattice=1, l1=16, l2=16, beta=1.0, dtau=0.05, rhub=2.0, nflr=2, mu=0.3,
                                kinetic=1, update=1, hs=1, nwrap=10, nublock=32),
    # dense kinetic term (the zgemm branch of the h0conf props)
    "sq4_dense_gen4_delay": dict(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.1, rhub=4.0, nflr=2, mu=0.2,
                                 kinetic=2, update=1, hs=1, nwrap=10, nublock=8),
    "hc3_dense_su4_sub": dict(lattice=2, l1=3, l2=3, beta=1.6, dtau=0.1, rhub=6.0, nflr=4,
                              kinetic=2, update=2, hs=0, nwrap=8, nublock=8),
    # the 1D chain (its own build of the reference, equaltime_measure1d.f90)
    "ch8_cb_gen4_delay": dict(lattice=3, l1=8, l2=1, beta=2.0, dtau=0.1, rhub=4.0, nflr=2, mu=0.2, t2=0.3,
                              flux_x=0.1, kinetic=0, update=1, hs=1, nwrap=5, nublock=4),
    "ch10_dense_exact_sub": dict(lattice=3, l1=10, l2=1, beta=2.0, dtau=0.1, rhub=3.0, nflr=2,
                                 kinetic=2, update=2, hs=0, nwrap=10, nublock=8),
    # the cubic lattice (-DCUBIC build, equaltime_measure3d.f90): six bond families
    "cu4_cb_gen4_delay": dict(lattice=4, l1=4, l2=4, l3=4, beta=1.0, dtau=0.1, rhub=4.0, nflr=2, mu=0.2,
                              kinetic=0, update=1, hs=1, nwrap=5, nublock=8),
    "cu422_cb_exact_fast": dict(lattice=4, l1=4, l2=2, l3=2, beta=1.0, dtau=0.1, rhub=4.0, nflr=2,
                                kinetic=0, update=0, hs=0, nwrap=10),
    "cu224_dense_exact_sub": dict(lattice=4, l1=2, l2=2, l3=4, beta=1.5, dtau=0.1, rhub=4.0, nflr=2, mu=0.1,
                                  kinetic=2, update=2, hs=0, nwrap=5, nublock=8),
    # the r_cubic lattice (-DR_CUBIC): six orbitals per cell, family 4 with
    # shared sites and the interlayer hopping rtd
    "rc222_cb_gen4_delay": dict(lattice=5, l1=2, l2=2, l3=2, beta=1.0, dtau=0.1, rhub=4.0, nflr=2, mu=0.1, rtd=0.7,
                                kinetic=0, update=1, hs=1, nwrap=5, nublock=8),
    "rc322_dense_exact_sub": dict(lattice=5, l1=3, l2=2, l3=2, beta=1.0, dtau=0.1, rhub=3.0, nflr=2,
                                  kinetic=2, update=2, hs=0, nwrap=5, nublock=8),
    # the plaquette field (hconf) beside the U field
    "sq4_plq_gen4_delay": dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.1, rhub=3.0, rhub_plq=1.0, alpha=0.3,
                               theta=0.2, nflr=2, mu=0.1, kinetic=0, update=1, hs=1, nwrap=5, nublock=4),
    "hc3_plq_dense_exact_fast": dict(lattice=2, l1=3, l2=3, beta=1.0, dtau=0.1, rhub=3.0, rhub_plq=0.8, alpha=0.25,
                                     theta=0.1, nflr=2, kinetic=2, update=0, hs=0, nwrap=5),
    # the t-V bond field (vconf) beside the U field on the finite-temperature path
    "hc3_tuv_cb_gen4_delay": dict(lattice=2, l1=3, l2=3, beta=1.0, dtau=0.1, rhub=2.0, rv=0.8, nflr=2,
                                  kinetic=0, update=1, hs=1, nwrap=5, nublock=4),
    "sq4_tuv_fft_exact_fast": dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.05, rhub=2.0, rv=1.0, mu=0.1, nflr=2,
                                   kinetic=1, update=0, hs=0, nwrap=10),
    "ch8_tuv_dense_exact_sub": dict(lattice=3, l1=8, l2=1, beta=1.0, dtau=0.1, rhub=2.0, rv=1.2, nflr=2,
                                    kinetic=2, update=2, hs=0, nwrap=5, nublock=8),
    "cu422_tuv_cb_gen4_delay": dict(lattice=4, l1=4, l2=2, l3=2, beta=1.0, dtau=0.1, rhub=3.0, rv=0.7, nflr=2,
                                    kinetic=0, update=1, hs=1, nwrap=5, nublock=8),
    # all three fields: plaquettes, bonds and sites in one slice
    "sq4_plq_tuv_cb_gen4_delay": dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.1, rhub=2.0, rv=0.6, rhub_plq=0.8,
                                      alpha=0.3, theta=0.2, nflr=2, mu=0.1, kinetic=0, update=1, hs=1, nwrap=5,
                                      nublock=4),
}

TEST_SEED0 = 1909706392   # abs((0*1981+2008)*951049)


def rand_green(n: int, seed: int = 0) -> np.ndarray:
    """A well-conditioned complex matrix shaped like an equal-time G."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return np.asfortranarray(0.5 * np.eye(n) + 0.05 * a)


def rel_err(a, b) -> float:
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b))))
