"""CPU checks of the oracle (the parity checker) against independent references.

The oracle restates the Fortran reference; the reference itself cannot run
here (no Fortran compiler, MPI or MKL), so these tests pin the restatement by
  * an independent numpy restatement of the reference's SFMT, written in the
    reference's own 64-bit formulation (lib/m_spring.f90:256-379);
  * scipy's LAPACK for the restated zgeqr2 / zlaqp2 / zung2r / zgetf2;
  * known answers: the free-fermion Green's function and the Hubbard atom;
  * internal consistency of the three local-update flavours.
"""
import numpy as np
import pytest
import scipy.linalg as sl
from scipy.linalg import lapack

from tests._cases import CASES


# ---------------------------------------------------------------- SFMT
def sfmt_numpy(seed: int, count: int) -> np.ndarray:
    """spring_sfmt_init + spring_sfmt_source in the reference's 64-bit form."""
    M64 = (1 << 64) - 1
    pt32 = [0] * 624
    pt32[0] = seed & 0xFFFFFFFF
    for i in range(1, 624):
        pt32[i] = (1812433253 * (pt32[i - 1] ^ (pt32[i - 1] >> 30)) + i) & 0xFFFFFFFF
    parity = (1, 0, 0, 331998852)
    inner = 0
    for i in range(4):
        work = pt32[i] & parity[i]
        for _ in range(32):
            inner ^= work & 1
            work >>= 1
    if inner != 1:
        done = False
        for i in range(4):
            work = 1
            for _ in range(32):
                if work & parity[i]:
                    pt32[i] ^= work
                    done = True
                    break
                work <<= 1
            if done:
                break
    pt64 = [(pt32[2 * i + 1] << 32) | pt32[2 * i] for i in range(312)]

    def core(a_t, a_b, b_t, b_b, c_t, c_b, d_t, d_b):
        x_t = ((a_t << 8) | (a_b >> 56)) & M64
        x_b = (a_b << 8) & M64
        y_t = c_t >> 8
        y_b = ((c_t << 56) & M64) | (c_b >> 8)
        r_b = a_b ^ x_b ^ ((b_b >> 11) & 8667995624701935) ^ y_b ^ (((d_b & 70364449226751) << 18) & M64)
        r_t = a_t ^ x_t ^ ((b_t >> 11) & 9007156306837503) ^ y_t ^ (((d_t & 70364449226751) << 18) & M64)
        return r_t, r_b

    def kernel():
        r1_b, r1_t, r2_b, r2_t = pt64[308], pt64[309], pt64[310], pt64[311]
        for i in range(156):
            j = i + 122 if i < 34 else i + 122 - 156
            t, b = core(pt64[2 * i + 1], pt64[2 * i], pt64[2 * j + 1], pt64[2 * j], r1_t, r1_b, r2_t, r2_b)
            pt64[2 * i + 1], pt64[2 * i] = t, b
            r1_b, r1_t = r2_b, r2_t
            r2_b, r2_t = pt64[2 * i], pt64[2 * i + 1]

    out = []
    idx = 624
    for _ in range(count):
        if idx >= 624:
            kernel()
            idx = 0
        w = pt64[idx // 2]
        out.append((w >> 32) & 0xFFFFFFFF if idx & 1 else w & 0xFFFFFFFF)
        idx += 1
    return np.array(out, dtype=np.uint32)


def test_sfmt_matches_independent_restatement(oracle):
    seed = oracle.lib().orc_test_seed(0)
    assert seed == 1909706392
    ref = sfmt_numpy(seed, 2000)
    m = oracle.Model(**CASES["sq4_cb_exact_fast"])
    c = oracle.Chain(m, seed, draw_conf=False)
    got = np.array([int(round(c.uniform() * 4294967296.0 - 0.5)) for _ in range(2000)], np.uint32)
    assert np.array_equal(got, ref)


def test_test_seed_wraps_like_int32(oracle):
    import sunhubbardmy_b200 as sb
    for r in range(8):
        assert oracle.lib().orc_test_seed(r) == sb.test_seed(r)
    assert sb.test_seed(1) == 501232835      # |(3989 * 951049) mod 2^32 as int32|


# ---------------------------------------------------------------- LAPACK restatements
def _cmat(m, n, seed):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n)))


def test_zgeqr2_matches_lapack(oracle):
    a = _cmat(40, 40, 1)
    ours, tau = a.copy(order="F"), np.zeros(40, complex)
    oracle.lib().orc_zgeqr2(40, 40, oracle._ptr(ours), 40, oracle._ptr(tau))
    qr, tau_ref, _, info = lapack.zgeqrf(a)
    assert info == 0
    assert np.max(np.abs(np.triu(ours) - np.triu(qr))) < 1e-12
    assert np.max(np.abs(tau - tau_ref)) < 1e-12
    q = ours.copy(order="F")
    oracle.lib().orc_zung2r(40, 40, 40, oracle._ptr(q), 40, oracle._ptr(tau))
    q_ref, _, info = lapack.zungqr(qr, tau_ref)
    assert np.max(np.abs(q - q_ref)) < 1e-12


def test_zgeqp2_matches_zgeqp3(oracle):
    a = _cmat(30, 30, 2) * np.logspace(3, -3, 30)[None, :][:, np.random.default_rng(5).permutation(30)]
    ours, tau = np.asfortranarray(a), np.zeros(30, complex)
    ours = ours.copy(order="F")
    jp = np.zeros(30, np.int32)
    oracle.lib().orc_zgeqp2(30, 30, oracle._ptr(ours), 30, oracle._ptr(jp), oracle._ptr(tau))
    qr, jpvt, tau_ref, _, info = lapack.zgeqp3(np.asfortranarray(a))
    assert np.array_equal(jp, jpvt)          # scipy returns 1-based pivots too
    assert np.max(np.abs(np.triu(ours) - np.triu(qr))) < 1e-10 * np.max(np.abs(qr))


def test_zgetf2_matches_zgetrf(oracle):
    a = _cmat(25, 25, 3)
    ours, ipiv = a.copy(order="F"), np.zeros(25, np.int32)
    oracle.lib().orc_zgetf2(25, 25, oracle._ptr(ours), 25, oracle._ptr(ipiv))
    lu, piv, info = lapack.zgetrf(a)
    assert np.array_equal(ipiv - 1, piv)
    assert np.max(np.abs(ours - lu)) < 1e-12


def test_inv_logdet(oracle):
    a = _cmat(20, 20, 4) + 3 * np.eye(20)
    inv = a.copy(order="F")
    ld = np.zeros(2)
    oracle.lib().orc_inv_logdet_lu(20, oracle._ptr(inv), oracle._ptr(ld))
    sign, logabs = np.linalg.slogdet(a)
    assert np.max(np.abs(inv - np.linalg.inv(a))) < 1e-12
    assert abs(ld[0] - logabs) < 1e-12
    assert abs(np.exp(1j * ld[1]) - sign) < 1e-12


# ---------------------------------------------------------------- known answers
def test_free_fermion_green_fft(oracle):
    m = oracle.Model(lattice=1, l1=4, l2=4, beta=4.0, dtau=0.1, rhub=0.0, kinetic=1, nwrap=10)
    c = oracle.Chain(m, 1)
    c.sweep_start()
    H = m.h0mat()
    w, v = np.linalg.eigh(H)
    g_ex = (v * (1.0 / (1.0 + np.exp(-m.params.beta * w)))[None, :]) @ v.conj().T
    assert np.max(np.abs(c.green() - g_ex)) < 1e-12


def test_free_fermion_green_checkerboard(oracle):
    kw = dict(lattice=2, l1=3, l2=3, beta=3.0, dtau=0.1, rhub=0.0, kinetic=0, nwrap=10, mu=0.2)
    m = oracle.Model(**kw)
    c = oracle.Chain(m, 1)
    c.sweep_start()
    # B(beta, 0) from the 2x2 bond exponentials, applied in the reference's order
    N = m.ndim
    B = np.eye(N, dtype=complex, order="F")
    for _ in range(m.ltrot):
        for nf in list(range(1, m.nn_nf + 1)) + list(range(m.nn_nf, 0, -1)):
            m.h0_prop(oracle.LEFT_FORWARD, nf, B)
    g_ex = np.linalg.inv(np.eye(N) + B)
    assert np.max(np.abs(c.green() - g_ex)) < 1e-11
    # and the bond exponential really is exp(-dtau/2 h_bond)
    kin = m.kinetic()
    t = m.tables()
    i0 = t["nnlf_list"][0] - 1
    i1 = t["nnlist"][i0, 0] - 1
    H = m.h0mat()
    h = np.array([[-kw["mu"] / m.nn_nf, H[i0, i1]], [H[i1, i0], -kw["mu"] / m.nn_nf]])
    assert np.max(np.abs(kin["urt"][0] - sl.expm(-0.5 * kw["dtau"] * h))) < 1e-14


@pytest.mark.parametrize("lattice", [1, 2])
def test_free_fermion_green_dense(oracle, lattice):
    """Dense kinetic term: every h0 op is exp(-+dtau/2 H0) from the left or the
    right, and the U = 0 Green's function is (1 + exp(-beta H0))^-1."""
    kw = dict(lattice=lattice, l1=4 if lattice == 1 else 3, l2=4 if lattice == 1 else 3, beta=2.0, dtau=0.1,
              rhub=0.0, kinetic=2, nwrap=5, mu=0.3, xmag=0.2)
    m = oracle.Model(**kw)
    H = m.h0mat()
    N = m.ndim
    km, kp = sl.expm(-0.5 * kw["dtau"] * H), sl.expm(0.5 * kw["dtau"] * H)
    X = np.asfortranarray(np.random.default_rng(5).standard_normal((N, N)) + 0j)
    for op, ref in ((oracle.LEFT_FORWARD, km @ X), (oracle.LEFT_BACKWARD, kp @ X), (oracle.RIGHT_FORWARD, X @ km),
                    (oracle.RIGHT_BACKWARD, X @ kp), (oracle.LEFT_FORWARD_HC, km.conj().T @ X)):
        g = X.copy(order="F")
        m.h0_prop(op, 1, g)
        assert np.max(np.abs(g - ref)) < 1e-12, op
    c = oracle.Chain(m, 1)
    c.sweep_start()
    w, v = np.linalg.eigh(H)
    g_ex = (v * (1.0 / (1.0 + np.exp(-kw["beta"] * w)))[None, :]) @ v.conj().T
    assert np.max(np.abs(c.green() - g_ex)) < 1e-11


def test_projective_dyn_self_consistency(oracle):
    """dqmc_proj_dyn: the G(t,t) propagated through the window agrees with the
    one recomputed from (UL, UR) at the stabilisation points (xmax_dyn), and
    the first time index of znn_tau holds the equal-time density correlation
    (1/2 - n_i)(1/2 - n_j) - G(0,0)_ji (G(0,0) - 1)_ij / nflr summed over cells."""
    kw = dict(lattice=2, l1=3, l2=3, beta=2.0, dtau=0.1, rv=1.0, rhub=0.0, nflr=1, kinetic=0,
              nwrap=5, proj=1, rndness=1e-3, update=2, ltau=1, dyntau=1.0)
    m = oracle.Model(**kw)
    c = oracle.Chain(m, 7)
    c.proj_sweep_start()
    c.obser_init()
    c.proj_sweep_b0(lupdate=True, lmeasure=False)
    c.proj_sweep_0b(lupdate=True, lmeasure=True)
    b = c.dyn_bins()
    assert np.all(np.isfinite(b)) and np.max(np.abs(b)) > 0
    assert 0.0 < c.max_dyn_error() < 1e-10


def test_chain_energy_terms(oracle):
    """The chain's energy_bin of one measurement against the formulas of
    equaltime_measure1d.f90 evaluated from G directly: density, kinetic energy
    -2 nflr rt Re(Gc expar) over the bonds plus -2 t2 Re Gc over the two second
    neighbours, double occupancy and the bond term; plaquette bins stay zero."""
    kw = dict(lattice=3, l1=8, l2=1, beta=1.0, dtau=0.1, rhub=3.0, nflr=2, mu=0.2, t2=0.3, flux_x=0.1,
              kinetic=2, update=1, hs=1, nwrap=5, nublock=4)
    m = oracle.Model(**kw)
    c = oracle.Chain(m, 3)
    c.sweep_start()
    c.obser_init()
    c.measure()
    g = c.green()
    N = m.ndim
    gc = np.eye(N) - g.T
    ph = c.diag()["phase"]
    zphi = (np.sign(ph.real) / ph.real) * ph
    t = m.tables()
    kin = 0.0
    for i0 in t["nnlf_list"] - 1:
        for nf, d in ((0, 1), (1, -1)):
            i_n = t["nnlist"][i0, nf] - 1
            e = np.exp(2j * np.pi * kw["flux_x"] * d / kw["l1"])
            kin += -2 * kw["nflr"] * 1.0 * (gc[i0, i_n] * e).real
    for i in range(N):
        for nf in range(2):
            kin += -2 * kw["t2"] * gc[i, t["snlist"][i, nf] - 1].real
    zv = sum(gc[i0, t["nnlist"][i0, nf] - 1].real for i0 in t["nnlf_list"] - 1 for nf in range(2))
    e = c.bins()["energy"]
    assert abs(e[1] - np.trace(gc) / N * zphi) < 1e-12
    assert abs(e[2] - kin * zphi) < 1e-12
    assert abs(e[3] - np.sum(np.diag(gc) ** 2) * zphi) < 1e-12
    assert abs(e[4] - zv * zphi) < 1e-12
    assert np.all(e[5:8] == 0)


def test_hubbard_atom_double_occupancy(oracle):
    """rt = 0: independent sites, H = U/2 (n - 1)^2 per site at half filling;
    D = e^{-beta U / 2} / (2 (1 + e^{-beta U/2})).  EXACTHS is exact here, so the
    Monte Carlo mean must agree within its statistical error."""
    U, beta = 2.0, 1.0
    kw = dict(lattice=1, l1=2, l2=2, beta=beta, dtau=0.1, rt=0.0, rhub=U, nflr=2, kinetic=0,
              update=1, hs=0, nwrap=10, nublock=4)
    m = oracle.Model(**kw)
    c = oracle.Chain(m, 7)
    c.sweep_start()
    for _ in range(20):
        c.sweep_b0(True, False); c.sweep_0b(True, False)
    series = []
    for _ in range(300):
        c.obser_init()
        c.sweep_b0(True, True); c.sweep_0b(True, True)
        b = c.bins()
        series.append((b["energy"][3] / b["energy"][0]).real / m.ndim)
    s = np.asarray(series)
    d_exact = np.exp(-beta * U / 2) / (2 * (1 + np.exp(-beta * U / 2)))
    err = s.std(ddof=1) / np.sqrt(len(s)) * 3.0      # generous: autocorrelation
    assert abs(s.mean() - d_exact) < max(err, 2e-3), (s.mean(), d_exact)


# ---------------------------------------------------------------- consistency
@pytest.mark.parametrize("case", ["sq4_cb_exact_fast", "hc3_cb_su4_sub"])
def test_update_flavours_agree(oracle, case):
    kw = dict(CASES[case])
    out = []
    for upd in (0, 1, 2):
        kw["update"] = upd
        kw["nublock"] = 8 if upd else 0
        m = oracle.Model(**kw)
        c = oracle.Chain(m, 1909706392)
        c.sweep_start()
        c.sweep_b0(); c.sweep_0b()
        out.append((c.conf(), c.green(), c.diag()))
    for conf, g, d in out[1:]:
        assert np.array_equal(conf, out[0][0])
        assert np.max(np.abs(g - out[0][1])) < 1e-10
        assert d["accepted"] == out[0][2]["accepted"]
        assert d["max_wrap_error"] < 1e-10


def test_lattice_tables(oracle):
    for kw in (dict(lattice=1, l1=4, l2=6), dict(lattice=2, l1=3, l2=4), dict(lattice=3, l1=8, l2=1)):
        m = oracle.Model(beta=1.0, dtau=0.1, **kw)
        t = m.tables()
        N, lq = m.ndim, m.lq
        # every family pairs each A site with a distinct B site
        for f in range(m.nn_nf):
            b = t["nnlist"][t["nnlf_list"] - 1, f]
            assert len(set(b.tolist())) == m.nn_lf
            assert not set(b.tolist()) & set(t["nnlf_list"].tolist())
        # imj: zero distance is the last bin, and each row is a permutation
        assert np.all(np.diag(t["imj"]) == lq)
        for i in range(lq):
            assert sorted(t["imj"][i].tolist()) == list(range(1, lq + 1))
        assert t["list"][:, 0].max() == lq and t["list"][:, 1].max() == m.nsub


# ---------------------------------------------------------------- projective path
PROJ_TV = dict(lattice=2, l1=3, l2=3, beta=2.0, dtau=0.1, rv=1.2, rhub=0.0, nflr=1, kinetic=0,
               nwrap=5, proj=1, rndness=1e-3, update=2, nublock=8)


def test_qr_pqmc_tall_and_wide(oracle):
    """s_zgeQR_pqmc: orthonormal Q spanning the columns (rows) of A with
    det R > 0 and log|det R| returned."""
    rng = np.random.default_rng(3)
    for shape in ((18, 9), (9, 18)):
        a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        q, lw = oracle.qr_pqmc(a)
        if shape[0] >= shape[1]:
            assert np.allclose(q.conj().T @ q, np.eye(shape[1]), atol=1e-13)
            r = q.conj().T @ a
            assert np.allclose(q @ r, a, atol=1e-12)
            assert np.allclose(np.tril(r, -1), 0, atol=1e-12)
        else:
            # wide: factored through the plain transpose, Q returned transposed
            qt = q.T
            assert np.allclose(qt.conj().T @ qt, np.eye(shape[0]), atol=1e-13)
            r = qt.conj().T @ a.T
            assert np.allclose(np.tril(r, -1), 0, atol=1e-12)
        d = np.diag(r)
        assert np.allclose(d.imag, 0, atol=1e-12)
        assert np.prod(np.sign(d.real)) > 0
        assert abs(lw - np.sum(np.log(np.abs(d.real)))) < 1e-10


def test_bond_field_hs_identity(oracle):
    """vconf: per bond B_s = U diag(e^{a s}, e^{-a s}) U^T = exp(a s sigma_x) with
    cosh a = exp(dtau V / 2), and lambda sum_s det(1 + B_s) equals the Fock-space
    trace of exp(-dtau V (n1 - 1/2)(n2 - 1/2)) (two sites, one flavour):
    2 e^{-dtau V/4} + 2 e^{dtau V/4}, with lambda = exp(-dtau V / 4) / 2
    (src/dqmc_config_v/dqmc_set_conf.f90:20-22)."""
    m = oracle.Model(**PROJ_TV)
    dtau, V = PROJ_TV["dtau"], PROJ_TV["rv"]
    a = np.arccosh(np.exp(dtau * V / 2))
    t = m.tables()
    nnf = m.nn_nf
    b0 = 0
    i1 = t["nnlf_list"][b0] - 1
    i2 = t["nnlist"][i1, 0] - 1
    lam = 0.5 * np.exp(-dtau * V / 4)
    total = 0.0
    for s, val in ((-1, 1), (1, 2)):
        vconf = np.ones((m.ltrot, nnf, m.ndim), np.int32)
        vconf[0, 0, b0] = val
        g = np.asfortranarray(np.eye(m.ndim, dtype=complex))
        oracle.vconf_prop(m, vconf, oracle.LEFT_FORWARD, 1, 1, 2, g)
        oracle.vconf_prop(m, vconf, oracle.LEFT_FORWARD, 1, 1, 1, g)
        blk = g[np.ix_([i1, i2], [i1, i2])]
        assert np.allclose(blk, sl.expm(a * s * np.array([[0, 1], [1, 0]])), atol=1e-14)
        total += lam * np.linalg.det(np.eye(2) + blk).real
    assert abs(total - (2 * np.exp(-dtau * V / 4) + 2 * np.exp(dtau * V / 4))) < 1e-13
    # inverse props undo the forward ones (left and right)
    g = np.asfortranarray(np.eye(m.ndim, dtype=complex) + 0.1)
    g0 = g.copy()
    vconf = np.random.default_rng(1).integers(1, 3, size=(m.ltrot, nnf, m.ndim)).astype(np.int32)
    for op_f, op_b in ((oracle.LEFT_FORWARD, oracle.LEFT_BACKWARD), (oracle.RIGHT_FORWARD, oracle.RIGHT_BACKWARD)):
        for nflag in (2, 1):
            oracle.vconf_prop(m, vconf, op_f, 3, 2, nflag, g)
        for nflag in (2, 1):
            oracle.vconf_prop(m, vconf, op_b, 3, 2, nflag, g)
        assert np.allclose(g, g0, atol=1e-13)


def _dense_bmat(oracle, m, nt_from, nt_to):
    """B(nt_to, nt_from-1) of the free (field-free) projective model from the
    oracle's kinetic props: prod over slices of e^{-dtau K/2}(nf..1) e^{-dtau K/2}(1..nf)."""
    B = np.asfortranarray(np.eye(m.ndim, dtype=complex))
    for _ in range(nt_from, nt_to + 1):
        for nf in range(1, m.nn_nf + 1):
            m.h0_prop(oracle.LEFT_FORWARD, nf, B)
        for nf in range(m.nn_nf, 0, -1):
            m.h0_prop(oracle.LEFT_FORWARD, nf, B)
    return B


def test_projective_free_fermion_green(oracle):
    """Without interactions, the stabilised projective stack reproduces the
    dense G(tau) = I - B(tau,0) P [P^H B(beta,0) P]^-1 P^H B(beta,tau) at
    tau = beta (sweep_start) and at the measured middle slice of both sweeps."""
    kw = dict(lattice=2, l1=3, l2=3, beta=3.0, dtau=0.1, rv=0.0, rhub=0.0, nflr=1, kinetic=0,
              nwrap=7, proj=1, rndness=0.05, mu=0.1)
    m = oracle.Model(**kw)
    c = oracle.Chain(m, 12345)
    P, _ = c.trial()
    P = P[:, :m.ne]
    lt = m.ltrot

    def g_at(nt):
        Bl = _dense_bmat(oracle, m, 1, nt)
        Br = _dense_bmat(oracle, m, nt + 1, lt)
        UR = Bl @ P
        UL = P.conj().T @ Br
        return np.eye(m.ndim) - UR @ np.linalg.solve(UL @ UR, UL)

    c.proj_sweep_start()
    assert np.max(np.abs(c.proj_green() - g_at(lt))) < 1e-11
    c.obser_init()
    c.proj_sweep_b0(lupdate=False, lmeasure=True)
    d = c.diag()
    assert d["max_wrap_error"] < 1e-11
    # the measurement sits at nt = ltrot/2 (obs_eqt_mid_len = 1); its G is the
    # chain's last G only until the next stabilisation, so recompute the density
    gmid = g_at(lt // 2)
    dens = np.real(np.trace(np.eye(m.ndim) - gmid)) / m.lq
    e = c.bins()["energy"]
    # energy_bin(2) accumulates sum_i Gc_ii / lq, weighted by the sign
    assert abs(e[1].real / e[0].real - dens) < 1e-10
    c.proj_sweep_0b(lupdate=False, lmeasure=False)
    assert c.diag()["max_wrap_error"] < 1e-11


def test_projective_update_flavours_agree(oracle):
    """Fast rank-2 bond update (dqmc_proj_update.f90) and submatrix-LR
    (dqmc_proj_update_submatrix_LR.f90): same fields, same UR and (UL UR)^-1."""
    for nub in (2, 4, 8, 32):
        kw = dict(PROJ_TV, nublock=nub)
        m = oracle.Model(**kw)
        a = oracle.Chain(m, 7)
        b = oracle.Chain(m, 7)
        a.proj_sweep_start(); b.proj_sweep_start()
        for nt in (m.ltrot, m.ltrot - 1):
            for nf in (1, 2, 3):
                a.proj_update(nt, nf, flavour=oracle.FAST)
                b.proj_update(nt, nf, flavour=oracle.SUBMATRIX)
        assert np.array_equal(a.vconf(), b.vconf())
        for x, y in zip(a.proj_state(), b.proj_state()):
            assert np.max(np.abs(x - y)) < 1e-12 * max(1.0, np.max(np.abs(y)))
        assert a.diag()["accepted_v"] == b.diag()["accepted_v"] > 0


PROJ_U = dict(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.1, rv=0.0, rhub=4.0, nflr=2, kinetic=0, nwrap=5, proj=1,
              rndness=0.05, hs=0, mu=0.0)


@pytest.mark.parametrize("field,flavour", [("bond", "DELAY"), ("bond", "SUBMATRIX_G_EXACT"), ("site", "DELAY"),
                                           ("site", "SUBMATRIX_G")])
def test_projective_delay_flavours(oracle, field, flavour):
    """The delayed (dqmc_proj_update_delay.f90) and submatrix-G
    (dqmc_proj_update_submatrix_G.f90, -DDELAYG) projective updates of both
    fields against the fast flavour over three slices: same fields and accept
    counts, UR and (UL UR)^-1 to rounding.  For the bond field the
    submatrix-G flavour is taken with the exact inverse of the bond's 2 x 2
    block; the reference's own expressions for that inverse give different
    ratios (test_reference_delayg_block_inverse)."""
    f = getattr(oracle, flavour)
    kw0 = PROJ_TV if field == "bond" else PROJ_U
    nfs = (1, 2, 3) if field == "bond" else (0,)
    for nub in (2, 4, 8, 16):
        m = oracle.Model(**dict(kw0, nublock=nub))
        a = oracle.Chain(m, 11)
        b = oracle.Chain(m, 11)
        a.proj_sweep_start(); b.proj_sweep_start()
        for nt in (m.ltrot, m.ltrot - 1, m.ltrot - 2):
            for nf in nfs:
                a.proj_update(nt, nf, flavour=oracle.FAST)
                b.proj_update(nt, nf, flavour=f)
        key = "accepted_v" if field == "bond" else "accepted"
        assert np.array_equal(a.vconf(), b.vconf()) and np.array_equal(a.conf(), b.conf())
        for x, y in zip(a.proj_state(), b.proj_state()):
            assert np.max(np.abs(x - y)) < 1e-11 * max(1.0, np.max(np.abs(y)))
        assert a.diag()[key] == b.diag()[key] > 0


def test_reference_delayg_block_inverse():
    """The bond-field submatrix-G update inverts the accepted bond's 2 x 2 block
    v5 = [[a, b], [c, d]] with v3(1,1) = 1/a + (1/a) b (1/(d - b c / a)) (1/a) c,
    v3(1,2) = -(1/a) b / (d - b c / a), v3(2,1) = -(1/a) c / (a - c b / d),
    v3(2,2) = 1 / (d - b c / a) (src/dqmc_config_v/dqmc_proj_update_submatrix_G.f90).
    Three entries are those of the inverse; the (2,1) entry is the inverse's
    -c / (ad - bc) times d / a, so the flavour's later ratios in a block
    differ from the other flavours' unless a = d (they are 1/dp + ... and
    1/dm + ..., which differ for the t-V field)."""
    rng = np.random.default_rng(0)
    a, b, c, d = rng.normal(size=4) + 1j * rng.normal(size=4)
    v3 = np.array([[1 / a + (1 / a) * b * (1 / (d - (1 / a) * b * c)) * (1 / a) * c, -(1 / a) * b / (d - (1 / a) * b * c)],
                   [-(1 / a) * c / (a - (1 / d) * c * b), 1 / (d - (1 / a) * b * c)]])
    inv = np.linalg.inv(np.array([[a, b], [c, d]]))
    assert abs(v3[0, 0] - inv[0, 0]) < 1e-12 and abs(v3[0, 1] - inv[0, 1]) < 1e-12 and abs(v3[1, 1] - inv[1, 1]) < 1e-12
    assert abs(v3[1, 0] - inv[1, 0] * d / a) < 1e-12 and abs(v3[1, 0] - inv[1, 0]) > 1e-3
    # a = d: the expressions agree with the inverse
    v3s = np.array([[0, 0], [-(1 / a) * c / (a - (1 / a) * c * b), 0]])
    assert abs(v3s[1, 0] - np.linalg.inv(np.array([[a, b], [c, a]]))[1, 0]) < 1e-12


def test_projective_sweeps_wrap_error(oracle):
    """Two sweeps of the t-V projector with updates keep the wrap error and the
    phase difference at the rounding level."""
    m = oracle.Model(**PROJ_TV)
    c = oracle.Chain(m, 99)
    c.proj_sweep_start(); c.obser_init()
    for _ in range(2):
        c.proj_sweep_b0(); c.proj_sweep_0b()
    d = c.diag()
    assert d["max_wrap_error"] < 1e-9 and d["max_phasediff"] < 1e-9
    assert d["logcount"] == 4 * m.nst
    assert d["proposed_v"] == 4 * m.ltrot * m.nn_nf * m.nn_lf


def test_effective_action_gradient_by_finite_differences():
    """The numpy restatement of the learned effective action (the checker of
    the tensor-core network kernels): backpropagated gradient against central
    differences of its own forward value."""
    from oracle import nn_oracle as no
    rng = np.random.default_rng(0)
    th = rng.standard_normal(no.NP) * 0.2
    fields = [rng.choice([-1, 1], size=(4, 4, 4)) for _ in range(2)]
    r = np.array([0.7, -0.3])
    _, g = no.gradient(th, fields, r, emulate_bf16=False)
    eps = 1e-6
    for idx in (0, 5, 27 * 32 + 3, 27 * 32 + 32 + 100, no.NP - 40, no.NP - 2, no.NP - 1):
        tp = th.copy(); tp[idx] += eps
        tm = th.copy(); tm[idx] -= eps
        fd = sum(rr * (no.forward(tp, f, False) - no.forward(tm, f, False)) / (2 * eps) for f, rr in zip(fields, r))
        assert abs(g[idx] - fd) < 1e-7 * max(1.0, abs(fd))


@pytest.mark.parametrize("lattice,kinetic", [(1, 1), (2, 0)])
def test_dyn_pass_free_fermions(oracle, lattice, kinetic):
    """U = 0: the unequal-time pass gives G(tau,0) = B(tau) G0, G(0,tau) =
    -(1 - G0) B(tau)^-1, G(tau,tau) = B(tau) G0 B(tau)^-1 with G0 = (1 + B(beta))^-1,
    so znn_tau follows in closed form; phase 1.  Also: the pass restores the
    stack and G (pop_stage)."""
    kw = dict(lattice=lattice, l1=3 if lattice == 2 else 4, l2=3 if lattice == 2 else 4, beta=1.2, dtau=0.1,
              rhub=0.0, nflr=2, kinetic=kinetic, nwrap=4, ltau=1, dyntau=1.2)
    m = oracle.Model(**kw)
    c = oracle.Chain(m, 11)
    c.sweep_start()
    c.sweep_b0(lupdate=False, lmeasure=False)
    g_before = c.green()
    c.obser_init()
    c.sweep_dyn()
    assert np.max(np.abs(c.green() - g_before)) == 0.0
    N, lq, lt = m.ndim, m.lq, m.ltrot
    Bb = np.asfortranarray(np.eye(N, dtype=complex))
    c.bmat_left_forward(lt, 1, Bb)
    G0 = np.linalg.inv(np.eye(N) + Bb)
    t = m.tables()                                      # 1-based list, imj
    cell, orb, imj = t["list"][:, 0] - 1, t["list"][:, 1] - 1, t["imj"] - 1
    expect = np.zeros((m.ntdm + 1, 2, 2, lq), complex)
    for nt in range(1, lt + 2):
        B = np.asfortranarray(np.eye(N, dtype=complex))
        if nt > 1:
            c.bmat_left_forward(nt - 1, 1, B)
        Bi = np.linalg.inv(B)
        gt0, g0t, gtt = B @ G0, -(np.eye(N) - G0) @ Bi, B @ G0 @ Bi
        for j in range(N):
            for i in range(N):
                d = imj[cell[i], cell[j]]
                expect[nt - 1, orb[j], orb[i], d] += ((0.5 - gtt[i, i].real) * (0.5 - G0[j, j].real)
                                                      - 0.5 * g0t[j, i] * gt0[i, j])
    got = c.dyn_bins()
    assert np.max(np.abs(got - expect)) < 1e-9 * max(1.0, np.max(np.abs(expect)))


@pytest.mark.parametrize("kinetic", [0, 2])
def test_hubbard_ring_against_exact_trotterised_values(oracle, kinetic):
    """An independent pin of the whole finite-temperature algorithm (HS draws,
    fast updates, B products, UDV stabilisation, measurement): a 6-site SU(2)
    Hubbard ring (chain lattice, U = 4, beta = 2, dtau = 0.1, exact HS field,
    checkerboard or dense kinetic term) against Tr[B^Lt O] / Tr[B^Lt] in Fock
    space (tests/_ed.py), which DQMC samples exactly.  Double occupancy and
    kinetic energy per site agree within four standard errors of 16000 sweeps."""
    import sys, os
    sys.path.insert(0, os.path.dirname(__file__))
    from _ed import binned_mean, trotter_ring
    L, U, beta, dtau = 6, 4.0, 2.0, 0.1
    Dx, Kx = trotter_ring(L, 1.0, U, beta, dtau, dense=kinetic == 2)
    m = oracle.Model(lattice=3, l1=L, l2=1, beta=beta, dtau=dtau, rhub=U, nflr=2, kinetic=kinetic, update=0, hs=0,
                     nwrap=10)
    c = oracle.Chain(m, 21)
    c.sweep_start()
    for _ in range(200):
        c.sweep_b0(lmeasure=False); c.sweep_0b(lmeasure=False)
    ds, ks = [], []
    for _ in range(16000):
        c.obser_init(); c.sweep_b0(lmeasure=False); c.sweep_0b(lmeasure=True)
        e = c.bins()["energy"]
        ds.append((e[3] / e[0]).real / L)
        ks.append((e[2] / e[0]).real / L)
    dm, de = binned_mean(ds)
    km, ke = binned_mean(ks)
    assert abs(dm - Dx) < 4 * de, (dm, de, Dx)
    assert abs(km - Kx) < 4 * ke, (km, ke, Kx)
