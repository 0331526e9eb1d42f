"""The C-ABI boundary on the GPU: the replay driver (the reference's
dqmc_main / dqmc_ft_ctrl call order in C) against the Python driver on the
same seed, and the SFMT state hand-over (get_rng / set_rng)."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KW = dict(lattice=1, l1=4, l2=4, beta=1.0, dtau=0.1, rhub=4.0, nflr=2, kinetic=0, update=1, hs=1, nwrap=5,
          nublock=8, nsweep=2, nbin=2)


def test_replay_driver_matches_the_python_driver(sb, tmp_path):
    exe = os.path.join(ROOT, "sunhubbardmy_b200", "_lib", "replay_ft")
    assert os.path.exists(exe), "build with make -C sunhubbardmy_b200/csrc"
    (tmp_path / "dqmc.in").write_text(
        "&model_para\nla = 4, lb = 4, beta = 1.d0, dtau = 0.1d0, rhub = 4.d0, nflr = 2\n/\n"
        "&ctrl_para\nnwrap = 5, nsweep = 2, nbin = 2, nublock = 8\n/\n")
    subprocess.run([exe, "dqmc.in", "lattice=1", "update=1", "kinetic=0", "hs=1", "nwarmup=1"], cwd=tmp_path,
                   check=True, timeout=300)
    rows = [l.split() for l in (tmp_path / "replay.out").read_text().splitlines() if l.startswith("bin")]
    got = np.array([[float(x) for x in r[3:]] for r in rows]).reshape(2, 10, 2)

    p = sb.DqmcParams.make(**KW)
    g = sb.Dqmc(p, n_chains=1, seeds=[sb.test_seed(0)])
    g.sweep_start()
    g.sweep_b0(True, False); g.sweep_0b(True, False)
    ref = []
    for _ in range(2):
        g.obser_init()
        for _ in range(2):
            g.sweep_b0(True, True); g.sweep_0b(True, True)
        e = g.bins(0)["energy"]
        ref.append(np.stack([e.real, e.imag], axis=1))
    assert np.max(np.abs(got - np.array(ref))) <= 1e-12 * max(1.0, np.max(np.abs(ref)))
    conf = np.array((tmp_path / "conf_u.out").read_text().split()[1:], np.int32)
    assert np.array_equal(conf, g.conf(0).ravel())


def test_rng_state_hand_over(sb):
    """A chain given another chain's field and SFMT state continues its
    stream: identical draws and identical sweeps."""
    p = sb.DqmcParams.make(**KW)
    g = sb.Dqmc(p, n_chains=2, seeds=[sb.test_seed(0), sb.test_seed(7)])
    st = g.rng_state(0)
    assert st.shape == (625,) and 0 <= st[624] <= 624
    g.set_conf(g.conf(0), c=1)
    g.set_rng_state(st, c=1)
    assert np.array_equal(g.rng_state(1), st)
    g.sweep_start()
    g.sweeps(2, False)
    assert np.array_equal(g.conf(0), g.conf(1))
    assert np.max(np.abs(g.green(0) - g.green(1))) == 0.0
    assert np.array_equal(g.draw_u32(50, c=0), g.draw_u32(50, c=1))
    bad = st.copy(); bad[624] = 700
    with pytest.raises(sb.DqmcError):
        g.set_rng_state(bad, c=1)
