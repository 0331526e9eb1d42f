"""The cubic and r_cubic lattices (the reference's -DCUBIC and -DR_CUBIC
builds), checked on the CPU.

The tables are rebuilt here from the definitions of setup_latt3d_sub and
setup_cubic_sub (src/lattice.f90:1033-1157, 1280-1472) and compared with the
library's (dqmc_model_tables, host only) and the oracle's.  The oracle's
free-fermion Green's function (U = 0) is compared with (1 + B^Lt)^-1 built
here from the six bond families, and its 3D measurement with the formulas of
equaltime_measure3d.f90 evaluated here on a random G.  The writers of
dqmc.out's lattice block (print_latt3d_sub), of equaltime_output3d.f90 and of
dyn_output3d.f90 are checked for their layout.  The r_cubic lattice
(setup_r_cubic_sub, src/lattice.f90:1486-1605) gets the same table, free
fermion and measurement checks; its family 4 has bonds with a common site, so
(1 + B^Lt)^-1 is built here with the bonds of a family applied one after the
other, as the reference's loops do.
"""
import io
import os

import numpy as np
import pytest
from scipy.linalg import expm

SIZES = [(4, 2, 2), (2, 4, 4), (4, 4, 2), (2, 2, 2)]


def npbc(nr, l):
    return nr - l if nr > l else (nr + l if nr < 1 else nr)


def reference_tables(l1, l2, l3):
    """1-based tables written from the reference's loops."""
    nc = l1 * l2 * l3

    def site(a, b, c):
        return (npbc(c, l3) - 1) * l1 * l2 + (npbc(a, l1) - 1) * l2 + npbc(b, l2)
    ulist = np.zeros((nc, 3), int)
    nnlf = []
    for i1 in range(1, l1 + 1):
        for i2 in range(1, l2 + 1):
            for i3 in range(1, l3 + 1):
                s = (i3 - 1) * l1 * l2 + (i1 - 1) * l2 + i2
                ulist[s - 1] = (i1, i2, i3)
                if (i1 + i2 + i3) % 2 == 0:
                    nnlf.append(s)
    nn = np.zeros((nc, 6), int)
    sn = np.zeros((nc, 12), int)
    for i in range(nc):
        u1, u2, u3 = ulist[i]
        nn[i] = [site(u1, u2, u3 + 1), site(u1 + 1, u2, u3), site(u1, u2 + 1, u3),
                 site(u1, u2, u3 - 1), site(u1 - 1, u2, u3), site(u1, u2 - 1, u3)]
        sn[i] = [site(u1 + 1, u2 + 1, u3), site(u1 - 1, u2 + 1, u3), site(u1 - 1, u2 - 1, u3), site(u1 + 1, u2 - 1, u3),
                 site(u1, u2 + 1, u3 + 1), site(u1, u2 + 1, u3 - 1), site(u1, u2 - 1, u3 - 1), site(u1, u2 - 1, u3 + 1),
                 site(u1 + 1, u2, u3 + 1), site(u1 + 1, u2, u3 - 1), site(u1 - 1, u2, u3 - 1), site(u1 - 1, u2, u3 + 1)]
    imj = np.zeros((nc, nc), int)
    for j in range(nc):
        for i in range(nc):
            nx = npbc(ulist[i, 0] - ulist[j, 0], l1)
            ny = npbc(ulist[i, 1] - ulist[j, 1], l2)
            nz = npbc(ulist[i, 2] - ulist[j, 2], l3)
            imj[i, j] = (nz - 1) * l1 * l2 + ny + (nx - 1) * l2
    order = [(1, 1, 1), (1, 1, 0), (1, 0, 1), (1, 0, 0), (0, 1, 1), (0, 1, 0), (0, 0, 1), (0, 0, 0)]
    cubes = {t: [] for t in order}
    for i1 in range(1, l1 + 1):
        for i2 in range(1, l2 + 1):
            for i3 in range(1, l3 + 1):
                cubes[(i1 % 2, i2 % 2, i3 % 2)].append(
                    [site(i1, i2, i3), site(i1 + 1, i2, i3), site(i1 + 1, i2 + 1, i3), site(i1, i2 + 1, i3),
                     site(i1, i2, i3 + 1), site(i1 + 1, i2, i3 + 1), site(i1 + 1, i2 + 1, i3 + 1),
                     site(i1, i2 + 1, i3 + 1)])
    plq = np.array([c for t in order for c in cubes[t]], int)
    lst = np.stack([np.arange(1, nc + 1), np.ones(nc, int)], axis=1)
    return dict(nnlist=nn, nnlf_list=np.array(nnlf), list=lst, imj=imj, plq_cord=plq, snlist=sn)


def kw_of(l1, l2, l3, **extra):
    kw = dict(lattice=4, l1=l1, l2=l2, l3=l3, beta=1.0, dtau=0.1, rhub=4.0, nflr=2, nwrap=5)
    kw.update(extra)
    return kw


@pytest.mark.parametrize("size", SIZES)
def test_cubic_tables_follow_reference_definitions(oracle, size):
    import sunhubbardmy_b200 as sb
    ref = reference_tables(*size)
    kw = kw_of(*size)
    t = sb.DqmcParams.make(**kw).tables()
    to = oracle.Model(**kw).tables()
    for k, v in ref.items():
        assert np.array_equal(t[k], v), k
        assert np.array_equal(to[k], v), k


def test_cubic_params():
    import sunhubbardmy_b200 as sb
    p = sb.DqmcParams.make(**kw_of(4, 2, 2, nu=0.0))
    assert (p.ndim, p.lq, p.ne, p.l3) == (16, 16, 8, 2)
    assert sb.DqmcParams.make(lattice=1, l1=4, l2=4, l3=7).l3 == 1     # 2D lattices keep l3 = 1
    for bad in (dict(l1=3), dict(l3=1), dict(l3=3)):
        with pytest.raises(sb.DqmcError):
            sb.DqmcParams.make(**dict(kw_of(4, 2, 2), **bad))
    with pytest.raises(sb.DqmcError):
        sb.DqmcParams.make(**kw_of(4, 4, 4, kinetic=1)).tables()        # the FFT pass is square-only
    g = sb.read_dqmc_in("&model_para\nla = 4,\nlb = 2,\nlc = 6,\nrhub = 4.0,\n/\n&ctrl_para\nnwrap = 10\n/\n")
    assert (g["l1"], g["l2"], g["l3"]) == (4, 2, 6)


def bond_hamiltonians(l1, l2, l3, rt, mu):
    """The six bond families' hopping matrices h_f (with -mu/6 on both ends of
    every bond, dqmc_set_h0conf.f90:76-123) and the full seth0 matrix."""
    ref = reference_tables(l1, l2, l3)
    N = l1 * l2 * l3
    hf = []
    for f in range(6):
        h = np.zeros((N, N))
        for a in ref["nnlf_list"]:
            b = ref["nnlist"][a - 1, f]
            h[a - 1, b - 1] += -rt
            h[b - 1, a - 1] += -rt
            h[a - 1, a - 1] += -mu / 6.0
            h[b - 1, b - 1] += -mu / 6.0
        hf.append(h)
    return hf


@pytest.mark.parametrize("kinetic", [0, 2])
@pytest.mark.parametrize("size", [(4, 2, 2), (2, 2, 4)])
def test_cubic_free_fermion_green(oracle, size, kinetic):
    """U = 0: G(beta, beta) = (1 + B^Lt)^-1 with the slice B = K1 ... K6 K6 ... K1,
    K_f = exp(-dtau h_f / 2) (checkerboard), or B = exp(-dtau H0) (dense)."""
    dtau, beta, mu = 0.1, 1.0, 0.3
    kw = kw_of(*size, rhub=0.0, mu=mu, kinetic=kinetic, beta=beta, dtau=dtau)
    c = oracle.Chain(oracle.Model(**kw), 5)
    c.sweep_start()
    hf = bond_hamiltonians(*size, 1.0, mu)
    N = hf[0].shape[0]
    if kinetic == 0:
        K = [expm(-0.5 * dtau * h) for h in hf]
        half = np.eye(N)
        for k in K:
            half = half @ k
        B = half @ half.T
    else:
        H = sum(hf)
        B = expm(-dtau * H)
    G = np.linalg.inv(np.eye(N) + np.linalg.matrix_power(B, int(round(beta / dtau))))
    assert np.max(np.abs(c.green() - G)) < 1e-12


def test_cubic_measurement_formulas(oracle):
    """equaltime_measure3d.f90 on a random G: energy_bin(1:4), cpcm, spsm, nn,
    bondcorr, zn and zb; nothing else is filled."""
    l1, l2, l3, nflr = 4, 2, 2, 4
    kw = kw_of(l1, l2, l3, nflr=nflr)
    m = oracle.Model(**kw)
    c = oracle.Chain(m, 3)
    N = m.ndim
    rng = np.random.default_rng(11)
    G = np.asfortranarray(0.5 * np.eye(N) + 0.1 * (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))))
    c.set_green(G)
    c.set_phase(1.0 + 0.0j)
    c.obser_init()
    c.measure()
    b = c.bins()
    ref = reference_tables(l1, l2, l3)
    Gc = np.eye(N) - G.T
    imj = ref["imj"] - 1
    nn1 = ref["nnlist"][:, 0] - 1
    zk = sum(-2.0 * Gc[a - 1, ref["nnlist"][a - 1, f] - 1].real for a in ref["nnlf_list"] for f in range(6))
    e = b["energy"]
    assert abs(e[0] - 1.0) < 1e-14
    assert abs(e[1] - np.trace(Gc) / N) < 1e-12
    assert abs(e[2] - zk) < 1e-11
    assert abs(e[3] - np.sum(np.diag(Gc) ** 2)) < 1e-11
    assert np.all(e[4:] == 0)
    cp = np.zeros(N, complex); sp = np.zeros(N, complex); nn = np.zeros(N, complex); bb = np.zeros(N, complex)
    fsp, fn = 1.0 - 1.0 / nflr ** 2, 1.0 / nflr
    for j in range(N):
        for i in range(N):
            k = imj[i, j]
            cp[k] += Gc[i, j]
            sp[k] += Gc[i, j] * G[i, j] * fsp
            nn[k] += Gc[i, i] * Gc[j, j] + fn * Gc[i, j] * G[i, j]
    for j0 in range(N):
        jn = nn1[j0]
        for i0 in range(N):
            i_n = nn1[i0]
            bb[imj[i0, j0]] += ((Gc[j0, jn] + Gc[jn, j0]) * (Gc[i0, i_n] + Gc[i_n, i0]) +
                                (Gc[i0, jn] * G[i_n, j0] + Gc[i_n, j0] * G[i0, jn] + Gc[i0, j0] * G[i_n, jn] +
                                 Gc[i_n, jn] * G[i0, j0]) * fn)
    for key, ref_v in (("cpcm", cp), ("spsm", sp), ("nn", nn)):
        assert np.max(np.abs(b[key][0, 0] - ref_v)) < 1e-11, key
        assert np.all(b[key][1:] == 0) and np.all(b[key][0, 1:] == 0), key
    assert np.max(np.abs(b["bb"] - bb)) < 1e-11
    assert abs(b["zn"][0] - np.trace(Gc)) < 1e-12 and b["zn"][1] == 0
    assert abs(b["zb"] - sum(Gc[j, nn1[j]] + Gc[nn1[j], j] for j in range(N))) < 1e-12
    for key in ("pair_onsite", "jj", "pair_nn", "pair_sn"):
        assert np.all(b[key] == 0), key
    assert b["zj"] == 0


def test_cubic_lattice_block_of_dqmc_out():
    import sunhubbardmy_b200 as sb
    p = sb.DqmcParams.make(**kw_of(4, 2, 2))
    f = io.StringIO()
    sb.io.dqmc_initial_print(f, p, sb.io.wrap_step_of(p))
    txt = f.getvalue()
    assert " la     =    4\n lb     =    2\n lc     =    2\n" in txt
    assert "\ncubic_lattice\nlattice information: \n" in txt
    assert " primitive lattice vector a3_p(:) =   0.000000000000  0.000000000000  1.000000000000\n" in txt
    assert " primitive reciprocal vector bz3_p(:) / 2pi =   0.000000000000  0.000000000000  1.000000000000\n" in txt
    lines = txt.split("\n")
    k = lines.index(" The lattice nnlist ")
    assert lines[k + 3] == "     1   9   3   2   9   7   2"
    k = lines.index(" The lattice tnlist ")
    assert len(lines[k + 3].split()) == 9
    k = lines.index(" The lattice plq_cord ")
    assert lines[k + 3] == "     1   1   3   4   2   9  11  12  10"
    k = lines.index(" The momentum listk ")
    assert lines[k + 3] == "     1  -1   0   0" and lines[k + 18] == "    16   2   1   1"
    # the chain prints la only
    q = sb.DqmcParams.make(lattice=3, l1=8, l2=1, beta=1.0, dtau=0.1, rhub=4.0, nwrap=5)
    f = io.StringIO()
    sb.io.dqmc_initial_print(f, q, sb.io.wrap_step_of(q))
    assert " la     =    8\n beta" in f.getvalue()


def test_cubic_output_files(tmp_path):
    import sunhubbardmy_b200 as sb
    l1, l2, l3 = 4, 2, 2
    lq = l1 * l2 * l3
    rng = np.random.default_rng(0)

    def zr(*shape):
        return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    bins = []
    for _ in range(2):
        z = np.concatenate([zr(10), zr(16 * lq), zr(4 * lq), zr(4)])
        bins.append(sb.unpack_bins(z, lq, nobs=5))
    red = sb.equaltime_output3d(bins, l1, l2, l3, str(tmp_path))
    norm = 2 * 5
    cp = (bins[0]["cpcm"][0, 0] + bins[1]["cpcm"][0, 0]) / norm
    assert np.allclose(red["cpcm"], cp)
    r = np.loadtxt(tmp_path / "cpcm_r.bin")
    assert r.shape == (lq, 2) and np.allclose(r[:, 0] + 1j * r[:, 1], cp, atol=1e-7)
    k = np.loadtxt(tmp_path / "cpcm_k.bin")
    zq = sb.io.zexpiqr3d(l1, l2, l3)
    gk = (cp[None, :] / zq).sum(axis=1) / lq
    assert k.shape == (lq, 5) and np.allclose(k[:, 3] + 1j * k[:, 4], gk, atol=1e-7)
    assert np.allclose(k[0, :3], [-1 / l1, 0.0, 0.0])
    e = np.loadtxt(tmp_path / "energy.bin")
    assert e.shape == (8,)
    assert np.allclose(e[0::2] + 1j * e[1::2], (bins[0]["energy"][:4] + bins[1]["energy"][:4]) / norm, atol=1e-7)
    for name in ("n.bin", "b.bin", "spsm_r.bin", "nn_k.bin", "bb_r.bin"):
        assert os.path.exists(tmp_path / name)
    assert not os.path.exists(tmp_path / "jj_r.bin") and not os.path.exists(tmp_path / "nnnn.bin")
    # unequal-time files: tau = 0 is left out, three observables
    ntdm = 3
    dyn = [zr(ntdm + 1, 2, 2, lq) for _ in range(2)]
    out = sb.dyn_output3d(dyn, 4, l1, l2, l3, str(tmp_path))
    gr = (dyn[0] + dyn[1]) / 8.0
    assert np.allclose(out["gf"], gr[:, 1, 0, :]) and np.allclose(out["spsm"], gr[:, 0, 1, :])
    rt = np.loadtxt(tmp_path / "nn_rtau.bin")
    assert rt.shape == (lq * ntdm, 2)
    assert np.allclose(rt[0, 0] + 1j * rt[0, 1], gr[1, 0, 0, 0], atol=1e-7)
    with open(tmp_path / "gf_ktau.bin") as f:
        lines = f.read().splitlines()
    assert len(lines) == lq * (1 + ntdm) and len(lines[0].split()) == 3


# ---------------------------------------------------------------------------
# r_cubic
# ---------------------------------------------------------------------------
def reference_tables_rc(l1, l2, l3):
    """1-based r_cubic tables written from setup_r_cubic_sub's loops."""
    nc, ns = l1 * l2 * l3, 6 * l1 * l2 * l3

    def cellof(a, b, c):
        return (npbc(c, l3) - 1) * l1 * l2 + (npbc(a, l1) - 1) * l2 + npbc(b, l2)
    cord = np.zeros((ns, 3), int)
    lst = np.zeros((ns, 2), int)
    ind = 0
    for i3 in range(1, l3 + 1):
        for i1 in range(1, l1 + 1):
            for i2 in range(1, l2 + 1):
                for isub in range(1, 7):
                    lst[ind] = ((i3 - 1) * l1 * l2 + (i1 - 1) * l2 + i2, isub)
                    cord[ind] = (i1, i2, i3)
                    ind += 1
    nn = np.zeros((ns, 4), int)
    for i in range(1, ns + 1):
        c1, c2, c3 = cord[i - 1]
        r = i % 6
        if r in (3, 5):
            nn[i - 1] = (i + 1, (cellof(c1 - 1, c2, c3) - 1) * 6 + r + 1, (cellof(c1, c2 - 1, c3) - 1) * 6 + r + 1, i - 1)
        elif r == 1:
            nn[i - 1] = (i + 1, (cellof(c1 - 1, c2, c3) - 1) * 6 + r + 1, (cellof(c1, c2 - 1, c3) - 1) * 6 + r + 1,
                         (cellof(c1 - 1, c2 - 1, c3 - 1) - 1) * 6 + r + 1)
        elif r in (2, 4):
            nn[i - 1] = (i - 1, (cellof(c1 + 1, c2, c3) - 1) * 6 + r - 1, (cellof(c1, c2 + 1, c3) - 1) * 6 + r - 1, i + 1)
        else:
            nn[i - 1] = (i - 1, (cellof(c1 + 1, c2, c3) - 1) * 6 + 5, (cellof(c1, c2 + 1, c3) - 1) * 6 + 5,
                         (cellof(c1 + 1, c2 + 1, c3 + 1) - 1) * 6 + 1)
    cc = np.array([cord[6 * c] for c in range(nc)])
    imj = np.zeros((nc, nc), int)
    for j in range(nc):
        for i in range(nc):
            nx, ny, nz = (npbc(cc[i, k] - cc[j, k], (l1, l2, l3)[k]) for k in range(3))
            imj[i, j] = (nz - 1) * l1 * l2 + ny + (nx - 1) * l2
    return dict(nnlist=nn, nnlf_list=np.arange(1, 2 * 3 * nc, 2), list=lst, imj=imj,
                plq_cord=np.zeros((nc, 8), int), snlist=np.zeros((ns, 12), int))


RC_SIZES = [(2, 2, 2), (3, 2, 2), (2, 3, 4)]


def kw_rc(l1, l2, l3, **extra):
    kw = dict(lattice=5, l1=l1, l2=l2, l3=l3, beta=1.0, dtau=0.1, rhub=4.0, nflr=2, nwrap=5, rtd=0.7)
    kw.update(extra)
    return kw


@pytest.mark.parametrize("size", RC_SIZES)
def test_rcubic_tables_follow_reference_definitions(oracle, size):
    import sunhubbardmy_b200 as sb
    ref = reference_tables_rc(*size)
    kw = kw_rc(*size)
    p = sb.DqmcParams.make(**kw)
    assert (p.ndim, p.lq) == (6 * np.prod(size), np.prod(size))
    t = p.tables()
    to = oracle.Model(**kw).tables()
    for k, v in ref.items():
        assert np.array_equal(t[k], v), k
        assert np.array_equal(to[k], v), k
    # bond family 4 shares B1 sites: the rtd bonds of A2 and of A1 in the cell at (+1, +1, +1)
    b4 = ref["nnlist"][ref["nnlf_list"] - 1, 3]
    assert len(set(b4)) < len(b4)
    # urt of family 4 carries rtd, the others rt
    dtau, lf = kw["dtau"], len(ref["nnlf_list"])
    for f, hop in ((0, 1.0), (3, 0.7)):
        h = np.array([[0.0, -hop], [-hop, 0.0]])
        assert np.max(np.abs(t["urt"][f * lf] - expm(-0.5 * dtau * h))) < 1e-15


@pytest.mark.parametrize("kinetic", [0, 2])
@pytest.mark.parametrize("size", [(2, 2, 2), (3, 2, 2)])
def test_rcubic_free_fermion_green(oracle, size, kinetic):
    """U = 0: the slice B = K1 K2 K3 K4 K4 K3 K2 K1 with K_f the product of the
    family's bond exponentials in the reference's order (rtd on family 4), or
    exp(-dtau H0) with rt on every bond (seth0) for the dense kinetic term."""
    dtau, beta, mu, rtd = 0.1, 1.0, 0.3, 0.7
    kw = kw_rc(*size, rhub=0.0, mu=mu, kinetic=kinetic, beta=beta, dtau=dtau, rtd=rtd)
    c = oracle.Chain(oracle.Model(**kw), 5)
    c.sweep_start()
    ref = reference_tables_rc(*size)
    N = ref["nnlist"].shape[0]
    if kinetic == 0:
        K = []
        for f in range(4):
            t = rtd if f == 3 else 1.0
            Kf = np.eye(N)
            for a in ref["nnlf_list"]:
                b = ref["nnlist"][a - 1, f]
                h = np.zeros((N, N))
                h[a - 1, b - 1] = h[b - 1, a - 1] = -t
                h[a - 1, a - 1] += -mu / 4.0
                h[b - 1, b - 1] += -mu / 4.0
                Kf = expm(-0.5 * dtau * h) @ Kf
            K.append(Kf)
        B = K[0] @ K[1] @ K[2] @ K[3] @ K[3] @ K[2] @ K[1] @ K[0]
    else:
        H = np.zeros((N, N))
        for a in ref["nnlf_list"]:
            for f in range(4):
                b = ref["nnlist"][a - 1, f]
                H[a - 1, b - 1] += -1.0
                H[b - 1, a - 1] += -1.0
        H -= mu * np.eye(N)
        B = expm(-dtau * H)
    G = np.linalg.inv(np.eye(N) + np.linalg.matrix_power(B, int(round(beta / dtau))))
    assert np.max(np.abs(c.green() - G)) < 1e-12


def test_rcubic_measurement_formulas(oracle):
    """equaltime_measure3d.f90 on the r_cubic lattice: the site correlations
    summed over all orbital pairs of a cell pair, the bond correlation over
    the pairs (nu, nnlist(nu, 1)) with the cell index nu used as a site."""
    l1, l2, l3, nflr = 2, 2, 2, 2
    m = oracle.Model(**kw_rc(l1, l2, l3, nflr=nflr))
    c = oracle.Chain(m, 3)
    N, lq = m.ndim, m.lq
    rng = np.random.default_rng(12)
    G = np.asfortranarray(0.5 * np.eye(N) + 0.1 * (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))))
    c.set_green(G)
    c.set_phase(1.0 + 0.0j)
    c.obser_init()
    c.measure()
    b = c.bins()
    ref = reference_tables_rc(l1, l2, l3)
    Gc = np.eye(N) - G.T
    imj = ref["imj"] - 1
    cell = ref["list"][:, 0] - 1
    zk = sum(-2.0 * Gc[a - 1, ref["nnlist"][a - 1, f] - 1].real for a in ref["nnlf_list"] for f in range(4))
    e = b["energy"]
    assert abs(e[2] - zk) < 1e-11 and abs(e[3] - np.sum(np.diag(Gc) ** 2)) < 1e-11
    cp = np.zeros(lq, complex); nn = np.zeros(lq, complex); bb = np.zeros(lq, complex)
    fn = 1.0 / nflr
    for j in range(N):
        for i in range(N):
            k = imj[cell[i], cell[j]]
            cp[k] += Gc[i, j]
            nn[k] += Gc[i, i] * Gc[j, j] + fn * Gc[i, j] * G[i, j]
    nn1 = ref["nnlist"][:, 0] - 1
    for j0 in range(lq):
        jn = nn1[j0]
        for i0 in range(lq):
            i_n = nn1[i0]
            bb[imj[i0, j0]] += ((Gc[j0, jn] + Gc[jn, j0]) * (Gc[i0, i_n] + Gc[i_n, i0]) +
                                (Gc[i0, jn] * G[i_n, j0] + Gc[i_n, j0] * G[i0, jn] + Gc[i0, j0] * G[i_n, jn] +
                                 Gc[i_n, jn] * G[i0, j0]) * fn)
    assert np.max(np.abs(b["cpcm"][0, 0] - cp)) < 1e-11
    assert np.max(np.abs(b["nn"][0, 0] - nn)) < 1e-11
    assert np.max(np.abs(b["bb"] - bb)) < 1e-11


def test_rcubic_lattice_block_of_dqmc_out():
    import sunhubbardmy_b200 as sb
    p = sb.DqmcParams.make(**kw_rc(2, 2, 2))
    f = io.StringIO()
    sb.io.dqmc_initial_print(f, p, sb.io.wrap_step_of(p))
    txt = f.getvalue()
    assert " la     =    2\n lc     =    2\n beta" in txt          # no lb under -DR_CUBIC
    assert "\nrhombohedral_cubic_lattice\nlattice information: \n" in txt
    assert " primitive lattice vector a1_p(:) =   0.866025403784 -0.500000000000  0.000000000000\n" in txt
    assert " primitive reciprocal vector bz2_p(:) / 2pi =   0.577350269190  1.000000000000  0.000000000000\n" in txt
    lines = txt.split("\n")
    k = lines.index(" The lattice nnlist ")
    assert lines[k + 3] == "     1   2  14   8  44"
    k = lines.index(" The lattice snlist ")
    assert lines[k + 3].split()[1:] == ["0"] * 12
