"""GPU parity: every kernel of the sweep against the CPU oracle, through the C ABI.

Tolerances: matrices built by the same operator sequence agree to 1e-12
relative; Green's functions recomputed from the UDV stack to 1e-10 absolute
(|G| = O(1)), the reference's own wrap-error scale; HS fields and accept
counts exactly.
"""
import numpy as np
import pytest

from tests._cases import CASES, TEST_SEED0, rand_green, rel_err

pytestmark = pytest.mark.gpu

OPS = [0, 1, 2, 3, 4]


@pytest.fixture(scope="module")
def sb():
    import sunhubbardmy_b200 as sb
    return sb


def make_pair(sb, oracle, case, n_chains=1):
    kw = CASES[case]
    p = sb.DqmcParams.make(**kw)
    g = sb.Dqmc(p, n_chains=n_chains, seeds=[sb.test_seed(c) for c in range(n_chains)])
    m = oracle.Model(**kw)
    ch = [oracle.Chain(m, sb.test_seed(c)) for c in range(n_chains)]
    return g, m, ch


def test_sfmt_draws_match(sb, oracle):
    g, m, ch = make_pair(sb, oracle, "sq4_cb_exact_fast")
    # the conf draw consumed ltrot*N draws on both sides; compare the next draws
    assert np.array_equal(g.conf(0), ch[0].conf())
    gpu = g.draw_u32(600)
    cpu = np.array([int(round(ch[0].uniform() * 4294967296.0 - 0.5)) for _ in range(600)], np.uint32)
    assert np.array_equal(gpu, cpu)


@pytest.mark.parametrize("opa,opb", [(0, 0), (2, 0), (0, 1), (0, 2), (2, 2)])
@pytest.mark.parametrize("mnk", [(16, 16, 16), (37, 29, 13), (72, 72, 72), (130, 65, 97)])
def test_zgemm_dmma(sb, opa, opb, mnk):
    m_, n_, k_ = mnk
    N = 256
    p = sb.DqmcParams.make(lattice=1, l1=16, l2=16, beta=1.0, dtau=0.1, rhub=4.0, nwrap=10)
    with sb.Dqmc(p, 1) as g:
        rng = np.random.default_rng(1)
        A = np.asfortranarray(rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N)))
        B = np.asfortranarray(rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N)))
        Cm = np.asfortranarray(rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N)))
        g.set_work(0, A); g.set_work(1, B); g.set_work(2, Cm)
        g.test_zgemm(m_, n_, k_, opa, opb, 0, 1, 2, beta=1.0)
        out = g.work(2)
    def op(X, o, r, c):
        if o == 0:
            return X[:r, :c]
        Y = X[:c, :r].T
        return Y.conj() if o == 2 else Y
    ref = Cm.copy()
    ref[:m_, :n_] = op(A, opa, m_, k_) @ op(B, opb, k_, n_) + Cm[:m_, :n_]
    assert rel_err(out, ref) < 1e-13


@pytest.mark.parametrize("N_L", [(16, 4), (72, 6), (256, 16)])
def test_qr_householder(sb, N_L):
    N, L = N_L
    p = sb.DqmcParams.make(lattice=1, l1=L, l2=N // L, beta=1.0, dtau=0.1, rhub=4.0, nwrap=10)
    with sb.Dqmc(p, 1) as g:
        rng = np.random.default_rng(2)
        # graded columns, like B U D in the stabilisation
        A = (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))) * np.logspace(8, -8, N)[None, :]
        A = np.asfortranarray(A)
        g.set_work(0, A)
        ld = g.test_qr(0, 1)[0]
        F = g.work(0)
        Q = g.work(1)
    R = np.triu(F)
    assert np.allclose(np.diag(R).imag, 0.0)
    assert np.max(np.abs(Q.conj().T @ Q - np.eye(N))) < 1e-12
    col = np.max(np.abs(A), axis=0)
    assert np.max(np.abs(Q @ R - A) / col[None, :]) < 1e-12
    sign, logabs = np.linalg.slogdet(Q)
    assert abs(np.exp(1j * ld.imag) - sign) < 1e-10 and abs(ld.real) < 1e-10


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("op", OPS)
def test_h0_prop(sb, oracle, case, op):
    g, m, ch = make_pair(sb, oracle, case)
    N = m.ndim
    G0 = rand_green(N, 3)
    nfs = range(1, m.nn_nf + 1) if CASES[case]["kinetic"] == 0 else [1]
    for nf in nfs:
        g.set_green(G0)
        g.h0_prop(op, nf)
        ref = G0.copy(order="F")
        m.h0_prop(op, nf, ref)
        assert rel_err(g.green(), ref) < 1e-12, (op, nf)


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("op", OPS)
def test_u_prop(sb, oracle, case, op):
    g, m, ch = make_pair(sb, oracle, case)
    N = m.ndim
    G0 = rand_green(N, 4)
    conf = ch[0].conf()
    for nt in (1, m.ltrot):
        g.set_green(G0)
        g.u_prop(op, nt)
        ref = G0.copy(order="F")
        m.u_prop(conf, op, nt, ref)
        assert rel_err(g.green(), ref) < 1e-13


@pytest.mark.parametrize("case", list(CASES))
def test_update_accept_sequence(sb, oracle, case):
    g, m, ch = make_pair(sb, oracle, case)
    ch[0].sweep_start()
    G0 = ch[0].green()
    ph = ch[0].diag()["phase"]
    g.set_green(G0)
    g.set_phase(ph)
    for nt in (1, 2, m.ltrot):
        g.update(nt)
        ch[0].update(nt)
        assert np.array_equal(g.conf(0), ch[0].conf()), nt
        assert np.max(np.abs(g.green() - ch[0].green())) < 1e-10
        dg, dc = g.diag(), ch[0].diag()
        assert dg["accepted"] == dc["accepted"]
        assert abs(dg["phase"] - dc["phase"]) < 1e-10


@pytest.mark.parametrize("case", list(CASES))
def test_measure(sb, oracle, case):
    g, m, ch = make_pair(sb, oracle, case)
    ch[0].sweep_start()
    G0 = ch[0].green()
    g.set_green(G0)
    g.set_phase(ch[0].diag()["phase"])
    g.obser_init(); ch[0].obser_init()
    g.measure(); ch[0].measure()
    bg, bc = g.bins(0), ch[0].bins()
    for key in ("energy", "cpcm", "spsm", "nn", "pair_onsite", "jj", "bb", "pair_nn", "pair_sn", "zn"):
        assert rel_err(bg[key], bc[key]) < 1e-11, key
    assert abs(bg["zj"] - bc["zj"]) < 1e-10 and abs(bg["zb"] - bc["zb"]) < 1e-10


@pytest.mark.parametrize("case", list(CASES))
def test_sweep_start(sb, oracle, case):
    g, m, ch = make_pair(sb, oracle, case)
    g.sweep_start(); ch[0].sweep_start()
    assert np.max(np.abs(g.green() - ch[0].green())) < 1e-10
    dg, dc = g.diag(), ch[0].diag()
    assert abs(dg["logweight"].real - dc["logweight"].real) < 1e-8 * max(1.0, abs(dc["logweight"].real))
    assert abs(dg["phase"] - dc["phase"]) < 1e-10


@pytest.mark.parametrize("case", list(CASES))
def test_full_sweeps(sb, oracle, case):
    nch = 2
    g, m, ch = make_pair(sb, oracle, case, n_chains=nch)
    g.sweep_start()
    g.obser_init()
    for c in ch:
        c.sweep_start(); c.obser_init()
    for s in range(2):
        g.sweep_b0(); g.sweep_0b()
        for c in ch:
            c.sweep_b0(); c.sweep_0b()
    for k in range(nch):
        assert np.array_equal(g.conf(k), ch[k].conf()), k
        assert np.max(np.abs(g.green(k) - ch[k].green())) < 1e-10
        dg, dc = g.diag(k), ch[k].diag()
        assert dg["accepted"] == dc["accepted"] and dg["proposed"] == dc["proposed"]
        if CASES[case]["lattice"] == 5 and CASES[case]["kinetic"] == 0:
            # r_cubic checkerboard: two bonds of family 4 share a site, so the
            # family's operator is not symmetric and the sweep's wrap, G K^-1 ..
            # K^T, is not the B product of the stack (dqmc_ft_sweep_b0.f90:58-61
            # against dqmc_ft_core.f90:80-117); the reference's wrap error is
            # O(dtau^2) there, and the GPU's must equal the oracle's
            assert abs(dg["max_wrap_error"] - dc["max_wrap_error"]) < 1e-9 * dc["max_wrap_error"]
        else:
            assert dg["max_wrap_error"] < 1e-10
        assert abs(dg["phase"] - dc["phase"]) < 1e-9
        if CASES[case].get("rhub_plq", 0.0):
            assert np.array_equal(g.conf_plq(k), ch[k].conf_plq()), k
            assert dg["accepted_plq"] == dc["accepted_plq"] and dg["proposed_plq"] == dc["proposed_plq"]
        if CASES[case].get("rv", 0.0):
            assert np.array_equal(g.vconf(k), ch[k].vconf()), k
            assert dg["accepted_v"] == dc["accepted_v"] and dg["proposed_v"] == dc["proposed_v"]
            assert 0 < dg["accepted_v"] < dg["proposed_v"]
        bg, bc = g.bins(k), ch[k].bins()
        assert bg["nobs"] == bc["nobs"]
        for key in ("energy", "cpcm", "nn", "jj", "bb"):
            assert rel_err(bg[key], bc[key]) < 1e-8, key


def test_graph_sweeps_equal_stepwise(sb, oracle):
    case = "sq4_fft_gen4_delay"
    g1, m, _ = make_pair(sb, oracle, case)
    g2, _, _ = make_pair(sb, oracle, case)
    g1.sweep_start(); g2.sweep_start()
    g1.obser_init(); g2.obser_init()
    g1.sweeps(2, True)
    for _ in range(2):
        g2.sweep_b0(); g2.sweep_0b()
    assert np.array_equal(g1.conf(0), g2.conf(0))
    assert np.max(np.abs(g1.green() - g2.green())) < 1e-12
    assert rel_err(g1.bins(0)["energy"], g2.bins(0)["energy"]) < 1e-12
