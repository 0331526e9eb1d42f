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
    # every file equaltime_output appends, nnnn.bin and Crmax.bin (zeros) included
    for name in ("n.bin", "j.bin", "b.bin", "nnnn.bin", "Crmax.bin", "cpcm_r.bin", "pair_sn_r.bin"):
        assert (tmp_path / name).exists(), name
    assert (tmp_path / "nnnn.bin").read_text() == f"{0.0:16.8e}{0.0:16.8e}\n"


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
    ft = sb.DqmcParams.make(rv=1.0, proj=0)      # the bond field on the finite-temperature path
    assert (ft.proj, ft.rv) == (0, 1.0)
    with pytest.raises(sb.DqmcError):
        sb.DqmcParams.make(lattice=sb.R_CUBIC, l1=2, l2=2, l3=2, rv=1.0)
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
    assert "              21              30               3\n" in txt and "\nsquare_lattice\nlattice information: \n" in txt
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


@pytest.mark.parametrize("lattice,l1,l2", [(1, 4, 4), (2, 3, 3), (3, 8, 1)])
def test_print_latt_block(lattice, l1, l2):
    """The lattice block of dqmc.out (print_latt2d_sub / print_latt1d_sub,
    src/lattice.f90:146-226, 502-597): every section with one row per site
    (per cell for listk and plq_cord), the neighbour lists of the library's
    tables, and the third-neighbour and k lists of the reference's formulas."""
    import io as pyio
    import sunhubbardmy_b200 as sb
    from sunhubbardmy_b200.io import lattice_lists, print_latt
    p = sb.DqmcParams.make(lattice=lattice, l1=l1, l2=l2, beta=1.0, dtau=0.1, rhub=4.0)
    f = pyio.StringIO()
    print_latt(f, p)
    txt = f.getvalue()
    N, lq = int(p.ndim), int(p.lq)
    L = lattice_lists(p)
    secs = ["list", "cord", "nnlist", "snlist", "tnlist"] + ([] if lattice == 3 else ["plq_cord"]) + ["listk"]
    for name in secs:
        assert f" --------------------- \n" in txt and (f"     {name}(" in txt)
    rows = [ln for ln in txt.splitlines() if ln[:6].strip().isdigit() and len(ln) >= 10]
    assert len(rows) == 5 * N + (0 if lattice == 3 else lq) + lq
    # site 1's neighbour rows are the library's tables
    t = p.tables()
    nn_row = "     1" + "".join(f"{int(v):4d}" for v in t["nnlist"][0])
    assert nn_row in txt.splitlines()
    assert sorted(tuple(k) for k in L["listk"]) == sorted(set(tuple(k) for k in L["listk"])) and len(L["listk"]) == lq
    if lattice == 1:   # square: third neighbours at +-2 along each axis
        assert list(L["tnlist"][0]) == [1 + 2 * l2, 3, 1 + (l1 - 2) * l2, l2 - 1]
        assert " primitive lattice  vector a1_p(:) =    1.000000000000  0.000000000000\n" in txt
    if lattice == 2:   # honeycomb: reciprocal vectors of a1 = (1/2, -sqrt3/2), a2 = (1/2, sqrt3/2)
        assert np.allclose(L["bz1"] / (2 * np.pi), [1.0, -1.0 / np.sqrt(3.0)])


# the three greps of the reference's timing analysis
# (examples/run_square_time/ana_time.sh:24-26), run by bash on a dqmc.out
ANA_TIME = r"""
time=$(grep -E "The_time_of_update_ratio.*_update"  dqmc.out|awk -F: '{printf "%.2f\n", $2}')
time1=$(grep -E "The_time_of_update_gfunc.*_update"  dqmc.out|awk -F: '{printf "%.2f\n", $2}')
time3=$(grep 'The_time_of_sweep_in_total'  dqmc.out|awk -F: '{printf "%.2f\n", $2}')
echo ${time} ${time1} ${time3}
"""


@pytest.mark.parametrize("update,proj,name", [(1, 0, "ft_delay_update"), (2, 0, "ft_submatrix_update"),
                                              (2, 1, "proj_submatrix_update"), (1, 1, "proj_delay_update")])
def test_timing_lines_feed_the_reference_analysis(tmp_path, update, proj, name):
    """dqmc_end's -DTIMING lines carry the update flavour in their names, so
    the reference's ana_time.sh reads the ratio, gfunc and total times."""
    import subprocess
    import sunhubbardmy_b200 as sb
    from sunhubbardmy_b200.io import dqmc_end_print, update_flavour
    kw = dict(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.1, rhub=4.0, update=update, nwrap=5)
    if proj:
        kw.update(lattice=2, l1=3, l2=3, rhub=0.0, rv=1.0, nflr=1, proj=1)
    p = sb.DqmcParams.make(**kw)
    assert update_flavour(p) == name
    prof = {"update": (1234.0, 1), "stab": (500.0, 1), "green": (300.0, 1), "prop_left": (100.0, 1),
            "measure": (50.0, 1), "prop_right": (50.0, 1), "bprod": (10.0, 1), "other": (6.0, 1)}
    with open(tmp_path / "dqmc.out", "w") as f:
        dqmc_end_print(f, [dict(accepted=1.0, proposed=2.0)], 3.0, prof, params=p, gfunc_s=0.634)
    out = subprocess.run(["bash", "-c", ANA_TIME], cwd=tmp_path, capture_output=True, text=True, check=True)
    assert out.stdout.split() == ["0.60", "0.63", "2.25"]
    txt = (tmp_path / "dqmc.out").read_text()
    assert f"The_time_of_{name}:" in txt


def test_fast_update_timing_line(tmp_path):
    import sunhubbardmy_b200 as sb
    from sunhubbardmy_b200.io import dqmc_end_print
    import io as pyio
    p = sb.DqmcParams.make(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.1, rhub=4.0, update=0, nwrap=5)
    prof = {k: (10.0, 1) for k in ("update", "stab", "green", "prop_left", "measure", "prop_right", "bprod", "other")}
    f = pyio.StringIO()
    dqmc_end_print(f, [dict(accepted=1.0, proposed=2.0)], 1.0, prof, params=p)
    txt = f.getvalue()
    assert "The_time_of_ft_fast_update:          0.010s" in txt and "update_gfunc" not in txt


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
    """The iso_c_binding types of include/dqmc_gpu_f.f90 list the C structs'
    fields in the same order and kind, so dqmc_gpu_get_diag and
    dqmc_params_derive never write past a Fortran caller's variable."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    header = open(os.path.join(root, "include", "dqmc_gpu.h")).read()
    mod = open(os.path.join(root, "include", "dqmc_gpu_f.f90")).read()
    assert _c_fields(header, "dqmc_params") == _f_fields(mod, "dqmc_params_c")
    assert _c_fields(header, "dqmc_diag") == _f_fields(mod, "dqmc_diag_c")


def test_fortran_interfaces_match_the_header():
    """Every bind(C) interface of the Fortran module names a function of the C
    header with the same number of arguments, and its integer constants
    repeat the header's values."""
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    header = re.sub(r"/\*.*?\*/", "", open(os.path.join(root, "include", "dqmc_gpu.h")).read(), flags=re.S)
    mod = open(os.path.join(root, "include", "dqmc_gpu_f.f90")).read()
    c_funcs = {}
    for name, args in re.findall(r"\b(dqmc_\w+)\s*\(([^;{]*?)\)\s*;", header):
        a = args.strip()
        c_funcs[name] = 0 if a in ("", "void") else a.count(",") + 1
    f_funcs = re.findall(r"function\s+(dqmc_\w+)\s*\(([^)]*)\)\s*bind\(C\)", mod)
    assert len(f_funcs) >= 35
    for name, args in f_funcs:
        assert name in c_funcs, name
        n = 0 if not args.strip() else args.count(",") + 1
        assert n == c_funcs[name], (name, n, c_funcs[name])
    for name, val in re.findall(r"(DQMC_\w+) = (-?\d+)", mod):
        m = re.search(rf"#define {name} \(?(-?\d+)\)?", header)
        assert m and int(m.group(1)) == int(val), name


REPLAY_STUB = r"""
#include <stdio.h>
#include <string.h>
#include "dqmc_gpu.h"
/* handle-less stand-in for libdqmc_gpu.so: logs every call */
static int lg(const char* n) { printf("%s\n", n); return 0; }
int dqmc_params_derive(dqmc_params* p) {
    lg("dqmc_params_derive");
    p->ndim = p->l1 * p->l2 * (p->lattice == 2 ? 2 : 1);
    p->ltrot = (int)(p->beta / p->dtau + 0.5);
    return 0;
}
const char* dqmc_gpu_last_error(void) { return ""; }
int dqmc_gpu_create(const dqmc_params* p, int np, int nch, const int32_t* s, int d, dqmc_handle** h) {
    *h = (dqmc_handle*)1; printf("dqmc_gpu_create %d %d %d %d\n", np, nch, (int)s[0], d); return 0; }
int dqmc_gpu_destroy(dqmc_handle* h) { return lg("dqmc_gpu_destroy"); }
int dqmc_gpu_set_conf(dqmc_handle* h, int c, const int32_t* x) { return lg("dqmc_gpu_set_conf"); }
int dqmc_gpu_get_conf(dqmc_handle* h, int c, int32_t* x) { return lg("dqmc_gpu_get_conf"); }
int dqmc_gpu_sweep_start(dqmc_handle* h) { return lg("dqmc_gpu_sweep_start"); }
int dqmc_gpu_sweep_b0(dqmc_handle* h, int u, int m) { printf("dqmc_gpu_sweep_b0 %d %d\n", u, m); return 0; }
int dqmc_gpu_sweep_0b(dqmc_handle* h, int u, int m) { printf("dqmc_gpu_sweep_0b %d %d\n", u, m); return 0; }
int dqmc_gpu_sweep_dyn(dqmc_handle* h) { return lg("dqmc_gpu_sweep_dyn"); }
int dqmc_gpu_obser_init(dqmc_handle* h) { return lg("dqmc_gpu_obser_init"); }
int dqmc_gpu_nbins(dqmc_handle* h, int c) { lg("dqmc_gpu_nbins"); return 14; }
int dqmc_gpu_get_bins(dqmc_handle* h, int c, double* o) { memset(o, 0, 28 * sizeof(double)); return lg("dqmc_gpu_get_bins"); }
int dqmc_gpu_get_diag(dqmc_handle* h, int c, dqmc_diag* d) { memset(d, 0, sizeof(*d)); return lg("dqmc_gpu_get_diag"); }
"""


def test_replay_driver_makes_the_reference_call_order(tmp_path):
    """replay_ft (the reference's dqmc_main / dqmc_ft_ctrl call order through
    the C ABI) built against a logging stub: dqmc_start, dqmc_warmup, then
    nbin x (obser_init, nsweep x (b0, [dyn,] 0b), equaltime_output,
    dqmc_timing), dqmc_end."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    (tmp_path / "stub.c").write_text(REPLAY_STUB)
    exe = tmp_path / "replay_stub"
    subprocess.run(["gcc", "-std=c99", "-o", str(exe), os.path.join(root, "sunhubbardmy_b200", "csrc", "replay_ft.c"),
                    str(tmp_path / "stub.c"), "-I", os.path.join(root, "include")], check=True)
    (tmp_path / "dqmc.in").write_text("&model_para\nla = 4, lb = 4,\nbeta = 1.d0\ndtau = 0.1d0,\nrhub = 4.0\n/\n"
                                      "&ctrl_para\nnwrap = 5, nsweep = 2, nbin = 2, ltau = .true.\n/\n")
    out = subprocess.run([str(exe), "dqmc.in", "nwarmup=1"], cwd=tmp_path, capture_output=True, text=True, check=True)
    calls = out.stdout.split("\n")[:-1]
    sweep = ["dqmc_gpu_sweep_b0 1 1", "dqmc_gpu_sweep_dyn", "dqmc_gpu_sweep_0b 1 1"]
    binl = ["dqmc_gpu_obser_init"] + sweep * 2 + ["dqmc_gpu_nbins", "dqmc_gpu_get_bins", "dqmc_gpu_get_diag",
                                                   "dqmc_gpu_get_conf"]
    expect = (["dqmc_params_derive", "dqmc_gpu_create 1 1 1909706392 1", "dqmc_gpu_sweep_start",
               "dqmc_gpu_sweep_b0 1 0", "dqmc_gpu_sweep_0b 1 0"] + binl * 2
              + ["dqmc_gpu_get_diag", "dqmc_gpu_destroy"])
    assert calls == expect
    lines = (tmp_path / "replay.out").read_text().split("\n")
    assert lines[0].startswith("bin 1 ") and lines[1].startswith("bin 2 ")
    conf = (tmp_path / "conf_u.out").read_text().split()
    assert conf[0] == "1" and len(conf) == 1 + 16 * 10


def test_multi_handle_entry_points_check_their_arguments():
    """dqmc_gpu_sweep_start_multi and dqmc_gpu_sweeps_multi refuse an empty or
    oversized handle list (1..16) and null handles before any device work."""
    import ctypes as C
    import sunhubbardmy_b200 as sb
    L = sb.load_library()
    nulls = (C.c_void_p * 17)()
    for n in (0, 17):
        assert L.dqmc_gpu_sweep_start_multi(nulls, n) == sb.EINVAL
        assert L.dqmc_gpu_sweeps_multi(nulls, n, 1, 1, None) == sb.EINVAL
    assert L.dqmc_gpu_sweep_start_multi(None, 1) == sb.EINVAL
    assert L.dqmc_gpu_sweep_start_multi(nulls, 2) == sb.EINVAL      # null handles
    assert L.dqmc_gpu_sweeps_multi(nulls, 2, 1, 1, None) == sb.EINVAL
