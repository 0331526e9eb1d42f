"""CPU tests of the host side: the C ABI library loads and exports every
declared symbol, parameter derivation matches make_tables, the library fails
cleanly without a GPU, dqmc.in / conf files round-trip, and the replica bin
reduction works across two gloo ranks."""
import os
import re

import numpy as np
import pytest

from tests._cases import CASES

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "dqmc_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dqmc_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import ctypes
    import sunhubbardmy_b200 as sb
    lib = sb.load_library()
    names = _declared_symbols()
    assert len(names) > 30
    for n in names:
        assert hasattr(lib, n), n
        assert isinstance(getattr(lib, n), ctypes._CFuncPtr)
    # and the Python binding declares a signature for each of them
    assert set(names) <= set(sb.dqmc.SIGNATURES)


@pytest.mark.parametrize("case", list(CASES))
def test_params_derive_matches_oracle(oracle, case):
    import sunhubbardmy_b200 as sb
    p = sb.DqmcParams.make(**CASES[case])
    m = oracle.Model(**CASES[case])
    assert (p.ndim, p.lq, p.ltrot, p.nst, p.lcomp) == (m.ndim, m.lq, m.ltrot, m.nst, m.lcomp)
    if CASES[case]["update"] != 0:
        assert p.nublock == m.nublock


@pytest.mark.parametrize("kinetic", [0, 2])
def test_chain_tables_match_oracle(oracle, kinetic):
    """The library's chain (lattice 3) tables and bond exponentials equal the
    oracle's restatement of setup_chain_sub and expar1d."""
    import sunhubbardmy_b200 as sb
    kw = dict(lattice=3, l1=10, l2=1, beta=1.0, dtau=0.1, rhub=2.0, mu=0.1, flux_x=0.2, dimer=0.1, kinetic=kinetic)
    p = sb.DqmcParams.make(**kw)
    m = oracle.Model(**kw)
    t, to = p.tables(), m.tables()
    for k in ("nnlist", "nnlf_list", "list", "imj", "plq_cord", "snlist"):
        assert np.array_equal(t[k], to[k]), k
    if kinetic == 0:
        assert np.max(np.abs(t["urt"] - m.kinetic()["urt"])) < 1e-15
    with pytest.raises(sb.DqmcError):
        sb.DqmcParams.make(**dict(kw, l1=9))
    with pytest.raises(sb.DqmcError):
        sb.DqmcParams.make(**dict(kw, kinetic=1)).tables()     # the FFT pass is square-only


def test_params_defaults_like_make_tables():
    import sunhubbardmy_b200 as sb
    # nublock defaults (src/model_para.f90:384-415)
    assert sb.DqmcParams.make(l1=16, l2=16, update=sb.DELAY, nublock=0).nublock == 16   # 256/5 < 64
    assert sb.DqmcParams.make(l1=4, l2=4, update=sb.DELAY, nublock=0).nublock == 4
    assert sb.DqmcParams.make(l1=20, l2=20, update=sb.DELAY, nublock=0).nublock == 32   # 400/5 < 256
    assert sb.DqmcParams.make(l1=12, l2=12, lattice=sb.HONEYCOMB, update=sb.SUBMATRIX, nublock=0).nublock == 32
    p = sb.DqmcParams.make(beta=8.0, dtau=0.1, nwrap=10)
    assert (p.ltrot, p.nst) == (80, 8)
    p = sb.DqmcParams.make(beta=8.5, dtau=0.1, nwrap=10)
    assert (p.ltrot, p.nst) == (85, 9)
    with pytest.raises(sb.DqmcError):
        sb.DqmcParams.make(lattice=7)


def test_create_without_gpu_fails_cleanly():
    import torch
    import sunhubbardmy_b200 as sb
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = sb.DqmcParams.make(**CASES["sq4_cb_exact_fast"])
    with pytest.raises(sb.DqmcError, match="CUDA"):
        sb.Dqmc(p, 1)


def test_read_dqmc_in():
    import sunhubbardmy_b200 as sb
    text = """&model_para
  la = 6, lb = 6,
  beta = 8.d0, dtau = 0.1d0,
  rt = 1.0d0, rhub = 6.d0,
  nflr = 4, lproju = .false.,
/
&ctrl_para
  nwrap = 10, nsweep = 20, nbin = 5,
  nublock = 32, ltau = .false.
/
"""
    kw = sb.read_dqmc_in(text)
    assert kw["l1"] == 6 and kw["l2"] == 6 and kw["nflr"] == 4
    assert kw["beta"] == 8.0 and kw["dtau"] == 0.1 and kw["rhub"] == 6.0
    assert kw["nwrap"] == 10 and kw["nublock"] == 32 and kw["lproju"] == 0
    p = sb.DqmcParams.make(lattice=sb.HONEYCOMB, **kw)
    assert (p.ndim, p.ltrot) == (72, 80)


def test_conf_file_roundtrip(tmp_path):
    import sunhubbardmy_b200 as sb
    rng = np.random.default_rng(0)
    confs = [rng.integers(1, 5, size=(8, 16), dtype=np.int32) for _ in range(3)]
    path = tmp_path / "conf_u.out"
    sb.write_conf(str(path), confs)
    back = sb.read_conf(str(path), 8, 16, n_chains=4)
    for a, b in zip(confs, back):
        assert np.array_equal(a, b)
    assert np.array_equal(back[3], confs[0])        # missing chains copy chain 0
    (tmp_path / "fresh").write_text("0\n")
    assert sb.read_conf(str(tmp_path / "fresh"), 8, 16) is None


def test_equaltime_output_normalisation(tmp_path):
    import sunhubbardmy_b200 as sb
    lq = 4
    rng = np.random.default_rng(1)
    flat = [rng.standard_normal(10 + 20 * lq + 4) + 1j * rng.standard_normal(10 + 20 * lq + 4) for _ in range(2)]
    bins = [sb.unpack_bins(f, lq, nobs=5) for f in flat]
    red = sb.equaltime_output(bins, str(tmp_path))
    assert np.allclose(red["energy"], (flat[0][:10] + flat[1][:10]) / 10.0)
    line = (tmp_path / "energy.bin").read_text().strip()
    assert len(line.split()) == 16
    sb.equaltime_output(bins, str(tmp_path / "chain"), chain=True)      # equaltime_output1d: all ten
    assert len((tmp_path / "chain" / "energy.bin").read_text().split()) == 20


def _gloo_worker(rank, world, port, q):
    import torch.distributed as dist
    import sunhubbardmy_b200 as sb
    from sunhubbardmy_b200.replicas import reduce_bins, replica_seeds
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lq = 4
    flat = [np.full(10 + 20 * lq + 4, rank + 1.0 + c, complex) for c in range(2)]
    bins = [sb.unpack_bins(f, lq, nobs=3) for f in flat]
    red = reduce_bins(bins)
    q.put((rank, replica_seeds(rank, 2), red["energy"][0], red["chains"]))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_bin_reduction_two_gloo_ranks():
    import socket
    import torch.multiprocessing as mp
    s = socket.socket(); s.bind(("127.0.0.1", 0)); port = s.getsockname()[1]; s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # chain values 1,2 (rank 0) and 2,3 (rank 1): sum 8 over 4 chains, nobs 3
    for rank, seeds, e0, nch in res:
        assert nch == 4
        assert abs(e0 - 8.0 / (4 * 3)) < 1e-12
    assert res[0][1] == [1909706392, 501232835]
    assert set(res[0][1]).isdisjoint(res[1][1])


@pytest.mark.parametrize("kw", [
    dict(lattice=2, l1=3, l2=3, beta=2.0, dtau=0.1, rv=1.0, nflr=1, nwrap=5, proj=1, rndness=1e-3),
    dict(lattice=2, l1=3, l2=3, beta=2.0, dtau=0.1, rv=1.0, nflr=1, nwrap=5, proj=1, rndness=0.3, flux_x=0.3, mu=0.1),
    dict(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.1, rhub=4.0, nflr=2, nwrap=5, proj=1, rndness=0.2, xmag=1.0),
])
def test_trial_state_matches_oracle(oracle, kw):
    """The library's host eigensolver (tridiagonalisation + implicit QL) gives
    the trial state of dqmc_set_proj after the reference's draw order: same
    eigenvalues as zheev (scipy) and the same projector onto the ne lowest
    states (the basis inside a level may differ)."""
    import sunhubbardmy_b200 as sb
    oracle.use_scipy_lapack(True)
    try:
        p = sb.DqmcParams.make(**kw)
        for seed in (sb.test_seed(0), sb.test_seed(5)):
            P, w = sb.trial_state(p, seed)
            m = oracle.Model(**kw)
            c = oracle.Chain(m, seed)
            Po, wo = c.trial()
            ne = p.ne
            assert np.max(np.abs(w - wo)) < 1e-12
            assert np.max(np.abs(P.conj().T @ P - np.eye(p.ndim))) < 1e-13
            assert np.max(np.abs(P[:, :ne] @ P[:, :ne].conj().T - Po[:, :ne] @ Po[:, :ne].conj().T)) < 1e-10
    finally:
        oracle.use_scipy_lapack(False)


def test_projective_params():
    import sunhubbardmy_b200 as sb
    p = sb.DqmcParams.make(lattice=2, l1=12, l2=12, beta=20.0, dtau=0.1, rv=1.0, nflr=1, proj=1, update=2)
    assert (p.ndim, p.ne, p.ltrot, p.nst, p.obs_mid_len, p.nublock) == (288, 144, 200, 20, 1, 32)
    with pytest.raises(sb.DqmcError):
        sb.DqmcParams.make(rv=1.0, proj=0)       # t-V runs on the projective path only
    with pytest.raises(sb.DqmcError):
        sb.DqmcParams.make(rv=1.0, proj=1, lstabilize=0)


def test_dyn_output_files(tmp_path):
    """dyn_output: chains reduced and normalised by nsweep * n_chains; nn_rtau.bin
    holds, per distance and time index, the nsub x nsub block; nn_ktau.bin the
    transform with zexpiqr."""
    from sunhubbardmy_b200.io import dyn_output
    rng = np.random.default_rng(0)
    lq, ntp, nsub = 4, 3, 2
    bins = [rng.standard_normal((ntp, 2, 2, lq)) + 1j * rng.standard_normal((ntp, 2, 2, lq)) for _ in range(2)]
    zq = np.exp(1j * rng.uniform(0, 2 * np.pi, (lq, lq)))
    gr = dyn_output(bins, 5, nsub, str(tmp_path), zexpiqr=zq, listk=np.ones((lq, 2)), l1=2, l2=2)
    assert np.allclose(gr, (bins[0] + bins[1]) / 10.0)
    rows = [np.array(l.split(), float) for l in open(tmp_path / "nn_rtau.bin")]
    assert len(rows) == lq * ntp and all(len(r) == 8 for r in rows)
    r = rows[1 * ntp + 2]                                   # imj = 2, nt = 3
    z = r[0::2] + 1j * r[1::2]
    assert np.allclose(z, [gr[2, 0, 0, 1], gr[2, 0, 1, 1], gr[2, 1, 0, 1], gr[2, 1, 1, 1]], atol=1e-7)
    krows = open(tmp_path / "nn_ktau.bin").read().splitlines()
    assert len(krows) == lq * (ntp + 1)
    k1 = np.array(krows[1].split(), float)                  # nk = 1, nt = 1
    gk = (gr[0, 0, 0, :] / zq[0, :]).sum() / lq
    assert np.allclose(k1[0] + 1j * k1[1], gk, atol=1e-7)
    # the chain (dyn_output1d.f90) lists k1 / l1 only
    dyn_output(bins, 5, 1, str(tmp_path / "chain"), zexpiqr=zq, listk=np.ones((lq, 2)), l1=4, l2=1)
    assert open(tmp_path / "chain" / "nn_ktau.bin").read().splitlines()[0].split() == [f"{0.25:.8f}"]


def test_dqmc_out_writers():
    """dqmc.out pieces: Fortran E16.8 numbers, the parameter banner with the
    wrapping coordinates, wrap-error lines and the end-of-run acceptances."""
    import io as pyio
    import sunhubbardmy_b200 as sb
    from sunhubbardmy_b200.io import (dqmc_end_print, dqmc_initial_print, fortran_e, wrap_error_print,
                                      wrap_step_of)
    assert fortran_e(1.5) == "  0.15000000E+01"
    assert fortran_e(-1.23456789e-4) == " -0.12345679E-03"
    assert fortran_e(0.0) == "  0.00000000E+00"
    assert fortran_e(9.999999999) == "  0.10000000E+02"
    p = sb.DqmcParams.make(lattice=1, l1=4, l2=4, beta=4.0, dtau=0.1, rhub=4.0, nwrap=10, ltau=1, dyntau=4.0)
    ws = wrap_step_of(p)
    assert ws == [(1, 10), (11, 20), (21, 30), (31, 40)]
    f = pyio.StringIO()
    dqmc_initial_print(f, p, ws)
    txt = f.getvalue()
    assert " beta   =   4.00\n" in txt and " rhub      =   4.000\n" in txt and " ntdm =     40\n" in txt
    assert "              21              30               3\n" in txt and txt.endswith("square_lattice\n")
    diags = [dict(max_wrap_error=1e-11, max_phasediff=0.0, avglog10error=-22.0, logcount=2.0, avgexpphasediff=2.0,
                  accepted=30.0, proposed=100.0, accepted_v=0.0, proposed_v=0.0),
             dict(max_wrap_error=3e-11, max_phasediff=1e-14, avglog10error=-21.0, logcount=2.0, avgexpphasediff=2.0,
                  accepted=20.0, proposed=100.0, accepted_v=0.0, proposed_v=0.0)]
    f = pyio.StringIO()
    wrap_error_print(f, diags)
    lines = f.getvalue().splitlines()
    assert lines[0] == "--------------max_wrap_error  =   0.30000000E-10"
    assert lines[2] == f"--------------avglog10error     = {-10.75:16.8f}"
    for d, x in zip(diags, (1e-13, 4e-13)):
        d.update(max_dyn_error=x, dyn_log10_sum=2 * np.log10(x), dyn_count=2.0)
    f = pyio.StringIO()
    wrap_error_print(f, diags, ltau=True)
    lines = f.getvalue().splitlines()
    assert lines[4] == "--------------xmax_dyn        =   0.40000000E-12"
    assert lines[5] == f"--------------avglog10dynerror  = {(np.log10(1e-13) + np.log10(4e-13)) / 2:16.8f}"
    f = pyio.StringIO()
    dqmc_end_print(f, diags, 12.5, {"update": (100.0, 1), "stab": (50.0, 1), "green": (30.0, 1),
                                    "prop_left": (10.0, 1), "measure": (5.0, 1), "prop_right": (5.0, 1),
                                    "bprod": (0.0, 1), "other": (0.0, 1)})
    out = f.getvalue()
    assert " >>> accep_u     =   0.25000000E+00\n" in out and " >>> Total time spent:     12.50s\n" in out
    assert "The_time_of_ft_delay_update:         0.100s =  50.00%\n" in out


def _c_fields(header: str, name: str):
    import re
    i = header.index(f"typedef struct {name} {{")
    j = header.index(f"}} {name};")
    body = re.sub(r"/\*.*?\*/", "", header[i:j], flags=re.S)
    return [("i" if t == "int32_t" else "d", x.strip())
            for t, names in re.findall(r"(int32_t|double)\s+([^;]+);", body) for x in names.split(",")]


def _f_fields(doc: str, name: str):
    import re
    a = doc.index(f"type, bind(C) :: {name}")
    b = doc.index("end type", a)
    return [("i" if t.startswith("integer") else "d", x.strip())
            for t, names in re.findall(r"(integer\(c_int32_t\)|real\(c_double\))\s*::\s*(.+)", doc[a:b])
            for x in names.split(",")]


def test_fortran_binding_types_mirror_the_header():
    """The iso_c_binding types of the integration guide list the C structs'
    fields in the same order and kind, so dqmc_gpu_get_diag and
    dqmc_params_derive never write past a Fortran caller's variable."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    header = open(os.path.join(root, "include", "dqmc_gpu.h")).read()
    doc = open(os.path.join(root, "INTEGRATION.md")).read()
    assert _c_fields(header, "dqmc_params") == _f_fields(doc, "dqmc_params_c")
    assert _c_fields(header, "dqmc_diag") == _f_fields(doc, "dqmc_diag_c")
