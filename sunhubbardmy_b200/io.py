"""On-disk formats of the reference, written from the GPU sweep's results.

* ``conf_u.in`` / ``conf_u.out`` (src/dqmc_config_u/dqmc_input_conf.f90:36-102,
  dqmc_output_conf.f90:27-42): a first line with a nonzero integer, then
  ``ltrot*nsites`` integers, one per line, site fastest, chain (rank) after
  chain.  ``conf_plqu.in`` / ``conf_plqu.out`` of the plaquette field
  (src/dqmc_config_plqu/dqmc_input_plqconf.f90, dqmc_output_plqconf.f90) have
  the same layout with ``lq`` plaquettes per slice: ``write_conf`` and
  ``read_conf`` serve both (``Dqmc.conf_plq`` / ``set_conf_plq``).
* ``energy.bin`` and the ``*.bin`` files of equaltime_output
  (src/dqmc_measure/equaltime_output.f90:67-180): per bin, the bin sums
  reduced over chains and divided by ``n_chains * nobs``.
* ``dqmc.out``: the parameter banner (dqmc_initial_print), the wrap-error
  lines (wrap_error_print) and the end of run with the -DTIMING breakdown
  (dqmc_end), src/dqmc_util.f90.
* ``nn_rtau.bin`` / ``nn_ktau.bin`` of dyn_output
  (src/dqmc_measure/dyn_output.f90): the unequal-time density correlation
  reduced over chains and divided by ``nsweep * n_chains``.
"""
from __future__ import annotations

import os

import numpy as np


def unpack_bins(z: np.ndarray, lq: int, nobs: int = 0) -> dict:
    """Split the flat bin array of dqmc_gpu_get_bins (see include/dqmc_gpu.h)."""
    k = 0
    out = {"energy": z[k:k + 10].copy()}
    k += 10
    for name in ("cpcm", "spsm", "nn", "pair_onsite"):
        out[name] = z[k:k + 4 * lq].reshape(2, 2, lq).copy()   # [no_j][no_i][d]
        k += 4 * lq
    for name in ("jj", "bb", "pair_nn", "pair_sn"):
        out[name] = z[k:k + lq].copy()
        k += lq
    out["zn"] = z[k:k + 2].copy()
    out["zj"] = z[k + 2]
    out["zb"] = z[k + 3]
    out["nobs"] = nobs
    return out


def write_conf(path: str, confs) -> None:
    """conf_u.out: '1' then every chain's field, site fastest ((i4) per line)."""
    with open(path, "w") as f:
        f.write("           1\n")
        for conf in confs:
            for v in np.asarray(conf, np.int32).ravel():
                f.write(f"{int(v):4d}\n")


def read_conf(path: str, ltrot: int, nsites: int, n_chains: int = 1):
    """conf_u.in reader; returns None for a fresh start (first integer 0).
    Missing chains copy chain 0, as dqmc_input_conf does (lines 86-100)."""
    if not os.path.exists(path):
        return None
    with open(path) as f:
        vals = [int(x) for x in f.read().split()]
    if not vals or vals[0] == 0:
        return None
    body = np.asarray(vals[1:], np.int32)
    per = ltrot * nsites
    out = []
    for c in range(n_chains):
        if (c + 1) * per <= body.size:
            out.append(body[c * per:(c + 1) * per].reshape(ltrot, nsites).copy())
        else:
            out.append(out[0].copy())
    return out


def _fourier(gr: np.ndarray, zexpiqr: np.ndarray) -> np.ndarray:
    """k-space transform of a distance-binned array (fourier_trans_eqt)."""
    return zexpiqr @ gr


def equaltime_output(bins_per_chain, outdir: str = ".", zexpiqr: np.ndarray | None = None,
                     chain: bool = False) -> dict:
    """Reduce chain bins, normalise by n_chains*nobs and append to the
    reference's files (energy.bin '(16e16.8)', n.bin, j.bin, b.bin, nnnn.bin,
    Crmax.bin, *_r.bin);
    for the 1D chain energy.bin holds all ten energies ('(20e16.8)',
    equaltime_output1d.f90)."""
    n = len(bins_per_chain)
    nobs = bins_per_chain[0]["nobs"]
    rnorm = float(n * nobs)
    red = {}
    for key in bins_per_chain[0]:
        if key == "nobs":
            continue
        red[key] = sum(b[key] for b in bins_per_chain) / rnorm
    os.makedirs(outdir, exist_ok=True)
    with open(os.path.join(outdir, "energy.bin"), "a") as f:
        e = red["energy"][:10] if chain else red["energy"][:8]
        f.write("".join(f"{v:16.8e}" for z in e for v in (z.real, z.imag)) + "\n")
    with open(os.path.join(outdir, "n.bin"), "a") as f:
        f.write("".join(f"{v:16.8e}" for z in red["zn"] for v in (z.real, z.imag)) + "\n")
    for name, key in (("j.bin", "zj"), ("b.bin", "zb")):
        with open(os.path.join(outdir, name), "a") as f:
            z = red[key]
            f.write(f"{z.real:16.8e}{z.imag:16.8e}\n")
    # znnnn and zCrmax: the reference appends them every bin, but their
    # accumulation is commented out (equaltime_measure.f90:54-57), so they are 0
    for name in ("nnnn.bin", "Crmax.bin"):
        with open(os.path.join(outdir, name), "a") as f:
            f.write(f"{0.0:16.8e}{0.0:16.8e}\n")
    for key in ("cpcm", "spsm", "nn", "pair_onsite", "jj", "bb", "pair_nn", "pair_sn"):
        with open(os.path.join(outdir, f"{key}_r.bin"), "a") as f:
            arr = np.asarray(red[key]).reshape(-1)
            f.write("".join(f"{v:16.8e}" for z in arr for v in (z.real, z.imag)) + "\n")
        if zexpiqr is not None:
            with open(os.path.join(outdir, f"{key}_k.bin"), "a") as f:
                arr = np.asarray(red[key])
                kk = _fourier(arr.reshape(-1, arr.shape[-1]).T, zexpiqr).T.reshape(-1)
                f.write("".join(f"{v:16.8e}" for z in kk for v in (z.real, z.imag)) + "\n")
    return red


def dyn_output(dyn_bins_per_chain, nsweep: int, nsub: int, outdir: str = ".",
               zexpiqr: np.ndarray | None = None, listk: np.ndarray | None = None,
               l1: int = 1, l2: int = 1) -> np.ndarray:
    """dyn_output (src/dqmc_measure/dyn_output.f90:1-68, fourier_trans_tau_22):
    reduce the znn_tau bins of the chains (as Dqmc.dyn_bins returns them,
    [ntdm+1, 2 (no_j), 2 (no_i), lq]), normalise by nsweep * n_chains and
    append nn_rtau.bin (per distance imj, per time index: the nsub x nsub
    block, column-major) and, given zexpiqr[nk, imj] and listk[nk, 2],
    nn_ktau.bin (per momentum: its coordinates, then the block at every time
    index, gk = sum_imj gr / zexpiqr(nk, imj) / lq)."""
    gr = sum(np.asarray(b) for b in dyn_bins_per_chain) / float(nsweep * len(dyn_bins_per_chain))
    ntp, _, _, lq = gr.shape
    os.makedirs(outdir, exist_ok=True)

    def block(a, nt):        # a[nt, no_j, no_i] -> (no_i, no_j) column-major over 1..nsub
        return [a[nt, j, i] for j in range(nsub) for i in range(nsub)]

    with open(os.path.join(outdir, "nn_rtau.bin"), "a") as f:
        for imj in range(lq):
            for nt in range(ntp):
                f.write("".join(f"{v:16.8e}" for z in block(gr[..., imj], nt) for v in (z.real, z.imag)) + "\n")
    if zexpiqr is not None:
        gk = np.einsum("tjim,km->tjik", gr, 1.0 / np.asarray(zexpiqr)) / lq
        with open(os.path.join(outdir, "nn_ktau.bin"), "a") as f:
            for nk in range(lq):
                if listk is not None:     # the chain writes k1 / l1 only (dyn_output1d.f90)
                    f.write(f"{listk[nk][0] / l1:16.8f}{listk[nk][1] / l2:16.8f}\n" if l2 > 1
                            else f"{listk[nk][0] / l1:16.8f}\n")
                for nt in range(ntp):
                    f.write("".join(f"{v:16.8e}" for z in block(gk[..., nk], nt) for v in (z.real, z.imag)) + "\n")
    return gr


def equaltime_output3d(bins_per_chain, l1: int, l2: int, l3: int, outdir: str = ".") -> dict:
    """equaltime_output of the cubic lattice (src/dqmc_measure/equaltime_output3d.f90):
    the chain bins reduced and divided by n_chains * nobs; energy.bin gets
    energy_bin(1:4) ('(8e16.8)'), n.bin zn and b.bin zb ('(2e16.8)'); cpcm, spsm,
    nn and bb get *_r.bin (one '(2e16.8)' line per distance imj) and *_k.bin
    (per momentum '(3f16.8,2e16.8)': k1/l1, k2/l2, k3/l3 and gk = sum_imj
    gr(imj) / zexpiqr(nk, imj) / lq).  The cubic bins use the (no_i, no_j) =
    (1, 1) block of the library's site and bond bins."""
    n = len(bins_per_chain)
    nobs = bins_per_chain[0]["nobs"]
    rnorm = float(n * nobs)
    red = {}
    for key in ("energy", "cpcm", "spsm", "nn", "bb", "zn", "zb"):
        red[key] = sum(np.asarray(b[key]) for b in bins_per_chain) / rnorm
    for key in ("cpcm", "spsm", "nn"):
        red[key] = red[key][0, 0]
    red["zn"] = red["zn"][0]
    os.makedirs(outdir, exist_ok=True)
    lq = l1 * l2 * l3
    listk = momentum_list3d(l1, l2, l3)
    zq = zexpiqr3d(l1, l2, l3)
    for key in ("cpcm", "spsm", "nn", "bb"):
        gr = red[key]
        with open(os.path.join(outdir, f"{key}_r.bin"), "a") as f:
            for z in gr:
                f.write(f"{z.real:16.8e}{z.imag:16.8e}\n")
        gk = (gr[None, :] / zq).sum(axis=1) / lq
        with open(os.path.join(outdir, f"{key}_k.bin"), "a") as f:
            for nk in range(lq):
                f.write(f"{listk[nk][0] / l1:16.8f}{listk[nk][1] / l2:16.8f}{listk[nk][2] / l3:16.8f}"
                        f"{gk[nk].real:16.8e}{gk[nk].imag:16.8e}\n")
    with open(os.path.join(outdir, "energy.bin"), "a") as f:
        f.write("".join(f"{v:16.8e}" for z in red["energy"][:4] for v in (z.real, z.imag)) + "\n")
    for name, key in (("n.bin", "zn"), ("b.bin", "zb")):
        with open(os.path.join(outdir, name), "a") as f:
            z = red[key]
            f.write(f"{z.real:16.8e}{z.imag:16.8e}\n")
    return red


def dyn_output3d(dyn_bins_per_chain, nsweep: int, l1: int, l2: int, l3: int, outdir: str = ".") -> dict:
    """dyn_output of the cubic lattice (src/dqmc_measure/dyn_output3d.f90): the
    chains' znn_tau, zspsm_tau and gtau0 (slots (0, 0), (0, 1) and (1, 0) of
    Dqmc.dyn_bins' [ntdm+1, 2, 2, lq]) reduced and divided by nsweep *
    n_chains, written without tau = 0 as nn_, spsm_ and gf_rtau.bin (per
    distance, per time index a '(2e16.8)' line) and _ktau.bin (per momentum
    '(3f16.8)' coordinates, then the time indices)."""
    gr = sum(np.asarray(b) for b in dyn_bins_per_chain) / float(nsweep * len(dyn_bins_per_chain))
    lq = l1 * l2 * l3
    listk = momentum_list3d(l1, l2, l3)
    zq = zexpiqr3d(l1, l2, l3)
    out = {"nn": gr[:, 0, 0, :], "spsm": gr[:, 0, 1, :], "gf": gr[:, 1, 0, :]}
    os.makedirs(outdir, exist_ok=True)
    for tag in ("spsm", "nn", "gf"):
        a = out[tag]                       # [nt, imj]
        with open(os.path.join(outdir, f"{tag}_rtau.bin"), "a") as f:
            for imj in range(lq):
                for nt in range(1, a.shape[0]):
                    f.write(f"{a[nt, imj].real:16.8e}{a[nt, imj].imag:16.8e}\n")
        gk = (a[:, None, :] / zq[None, :, :]).sum(axis=2) / lq      # [nt, nk]
        with open(os.path.join(outdir, f"{tag}_ktau.bin"), "a") as f:
            for nk in range(lq):
                f.write(f"{listk[nk][0] / l1:16.8f}{listk[nk][1] / l2:16.8f}{listk[nk][2] / l3:16.8f}\n")
                for nt in range(1, a.shape[0]):
                    f.write(f"{gk[nt, nk].real:16.8e}{gk[nt, nk].imag:16.8e}\n")
    return out


# ----------------------------------------------------------------------------
# dqmc.out (src/dqmc_util.f90): parameter banner, wrap-error lines, end of run
# ----------------------------------------------------------------------------
def fortran_e(v: float, w: int = 16, d: int = 8) -> str:
    """Fortran Ew.d: 0.ddddddddE+xx, right-justified in w columns."""
    v = float(v)
    if v == 0.0 or not np.isfinite(v):
        s = f"{0.0:.{d}f}E+00" if v == 0.0 else str(v)
    else:
        e = int(np.floor(np.log10(abs(v)))) + 1
        m = abs(v) / 10.0 ** e
        if round(m, d) >= 1.0:
            m /= 10.0
            e += 1
        s = f"{'-' if v < 0 else ''}0.{int(round(m * 10 ** d)):0{d}d}E{'+' if e >= 0 else '-'}{abs(e):02d}"
    return s.rjust(w)


def _lg(b) -> str:
    return "T" if b else "F"


def dqmc_initial_print(f, p, wrap_step=None, nustock: int = 0) -> None:
    """dqmc_initial_print (src/dqmc_util.f90:208-285) for the parameter set p
    (DqmcParams or a dict of the same fields); wrap_step: (start, end) slice
    pairs of the stabilisation intervals, 1-based."""
    g = p if isinstance(p, dict) else p.as_dict()
    w = f.write
    w("\n --------------------- \n The input parameters  \n --------------------- \n\n")
    w(f" t      = {g['rt']:6.2f}\n")
    w(f" mu     = {g['mu']:7.3f}\n")
    w(f" rhub_plq  = {g.get('rhub_plq', 0.0):7.3f}\n")
    w(f" lprojplqu =  {_lg(g.get('lprojplqu', 0))}\n")
    w(f" rhub      = {g['rhub']:7.3f}\n")
    w(f" lproju    =  {_lg(g['lproju'])}\n")
    w(f" rv      = {g['rv']:7.3f}\n")
    w(f" lprojv   =  {_lg(g['lprojv'])}\n")
    w(f" la     = {g['l1']:4d}\n")
    if g["lattice"] in (1, 2, 4):   # lb under -DHONEYCOMB, -DSQUARE, -DCUBIC
        w(f" lb     = {g['l2']:4d}\n")
    if g["lattice"] in (4, 5):      # lc under -DCUBIC, -DR_CUBIC
        w(f" lc     = {g.get('l3', 1):4d}\n")
    w(f" beta   = {g['beta']:6.2f}\n")
    w(f" dtau   = {g['dtau']:7.3f}\n")
    for k, name in (("ndim", "ndim"), ("ne", "ne  "), ("nwrap", "nwrap "), ("nsweep", "nsweep"),
                    ("nbin", "nbin"), ("nublock", "nublock")):
        w(f" {name} = {g[k]:6d}\n")
    w(f" nustock = {nustock:6d}\n")
    w(f" B      = {g['xmag']:6.2f}\n")
    w(f" flux_x = {g['flux_x']:8.5f}\n")
    w(f" flux_y = {g['flux_y']:8.5f}\n")
    w(f" dimer  = {g['dimer']:8.5f}\n")
    w(f" alpha  = {g['alpha']:8.5f}\n")
    w(f" theta  = {g['theta']:8.5f}\n")
    w(f" nflr   = {g['nflr']:4d}\n")
    w(f"  ltau =  {_lg(g.get('ltau', 0))}\n")
    if g.get("ltau", 0):
        ntdm = g.get("ntdm", 0)
        w(f" ntauin = {(g['ltrot'] - ntdm) // 2:6d}\n")
        w(f" ntdm = {ntdm:6d}\n")
    w("\n --------------------- \n wrapping coordinates  \n --------------------- \n")
    w("       wrap_step(1,i)   wrap_step(2,i)   iwrap_nt(nt) \n")
    for i, (a, b) in enumerate(wrap_step or [], start=1):
        w(f"{a:16d}{b:16d}{i:16d}\n")
    w(" \n")
    w({2: "honeycomb_lattice", 3: "chain_lattice", 4: "cubic_lattice",
       5: "rhombohedral_cubic_lattice"}.get(g["lattice"], "square_lattice") + "\n")
    if not isinstance(p, dict):
        print_latt(f, p)


def _f16_12(v: float) -> str:
    """Fortran f16.12."""
    return f"{v:16.12f}"


def lattice_lists(p) -> dict:
    """The lattice tables that print_latt writes (1-based), for a DqmcParams p:
    list/cord (setup_honeycomb_sub, setup_square_sub, setup_chain_sub in
    src/lattice.f90), nnlist/snlist/plq_cord from the library's own tables,
    tnlist (third neighbours, src/lattice.f90:312-313, 716-731, 892-895), listk
    (the k list of setup_latt2d_sub / setup_latt1d_sub) and the primitive and
    reciprocal vectors (src/model_para.f90:342-357)."""
    t = p.tables()
    l1, l2, lat = int(p.l1), int(p.l2), int(p.lattice)
    N = int(p.ndim)

    def npbc(nr, l):
        return nr - l if nr > l else (nr + l if nr < 1 else nr)

    if lat == 4:      # cubic (setup_latt3d_sub, setup_cubic_sub: src/lattice.f90:1033-1157, 1280-1472)
        l3 = int(p.l3)
        cord = np.zeros((N, 3), dtype=np.int64)
        for i1 in range(1, l1 + 1):
            for i2 in range(1, l2 + 1):
                for i3 in range(1, l3 + 1):
                    cord[(i3 - 1) * l1 * l2 + (i1 - 1) * l2 + i2 - 1] = (i1, i2, i3)

        def cs(c1, c2, c3):
            return (npbc(c3, l3) - 1) * l1 * l2 + (npbc(c1, l1) - 1) * l2 + npbc(c2, l2)
        tn = np.zeros((N, 8), dtype=np.int64)
        steps = ((1, 1, 1), (-1, 1, 1), (-1, -1, 1), (1, -1, 1), (1, 1, -1), (-1, 1, -1), (-1, -1, -1), (1, -1, -1))
        for i in range(N):
            c1, c2, c3 = cord[i]
            tn[i] = [cs(c1 + a, c2 + b, c3 + c) for (a, b, c) in steps]
        listk = momentum_list3d(l1, l2, l3)
        eye = np.eye(3)
        return dict(list=t["list"], cord=cord, nnlist=t["nnlist"], snlist=t["snlist"], tnlist=tn,
                    plq_cord=t["plq_cord"], listk=listk, a1=eye[0], a2=eye[1], a3=eye[2],
                    bz1=2.0 * np.pi * eye[0], bz2=2.0 * np.pi * eye[1], bz3=2.0 * np.pi * eye[2])
    if lat == 5:      # r_cubic (setup_r_cubic_sub, src/lattice.f90:1486-1605; a_p of model_para.f90:366-371)
        l3 = int(p.l3)
        cord = np.zeros((N, 3), dtype=np.int64)
        for i3 in range(1, l3 + 1):
            for i1 in range(1, l1 + 1):
                for i2 in range(1, l2 + 1):
                    c = (i3 - 1) * l1 * l2 + (i1 - 1) * l2 + i2 - 1
                    cord[6 * c:6 * c + 6] = (i1, i2, i3)
        a = np.array([[0.5 * np.sqrt(3.0), -0.5, 0.0], [0.5 * np.sqrt(3.0), 0.5, 0.0], [0.0, 0.0, 1.0]])
        inv = np.linalg.inv(a)          # bz_j(:) = 2 pi inv(:, j)
        return dict(list=t["list"], cord=cord, nnlist=t["nnlist"], snlist=t["snlist"],
                    tnlist=np.zeros((N, 8), dtype=np.int64), plq_cord=t["plq_cord"],
                    listk=momentum_list3d(l1, l2, l3), a1=a[0], a2=a[1], a3=a[2],
                    bz1=2.0 * np.pi * inv[:, 0], bz2=2.0 * np.pi * inv[:, 1], bz3=2.0 * np.pi * inv[:, 2])
    if lat == 3:      # chain
        a1, a2 = np.array([1.0]), None
        cord = np.array([[i] for i in range(1, l1 + 1)], dtype=np.int64)
        tn = np.array([[npbc(i + 3, l1), npbc(i - 3, l1)] for i in range(1, l1 + 1)], dtype=np.int64)
        listk = np.array([[m] for m in range(-((l1 + 1) // 2) + 1, l1 // 2 + 1)], dtype=np.int64)
    else:
        hc = lat == 2
        if hc:
            a1 = np.array([0.5, -0.5 * np.sqrt(3.0)]); a2 = np.array([0.5, 0.5 * np.sqrt(3.0)])
        else:
            a1 = np.array([1.0, 0.0]); a2 = np.array([0.0, 1.0])
        nsub = 2 if hc else 1
        cord = np.zeros((N, 2), dtype=np.int64)
        tn = np.zeros((N, 3 if hc else 4), dtype=np.int64)
        for i1 in range(1, l1 + 1):
            for i2 in range(1, l2 + 1):
                for o in range(nsub):
                    cord[((i1 - 1) * l2 + i2 - 1) * nsub + o] = (i1, i2)

        def cs(c1, c2):
            return (npbc(c1, l1) - 1) * l2 + npbc(c2, l2)
        for i in range(N):
            c1, c2 = cord[i]
            if hc and i % 2 == 0:      # A site (1-based odd)
                tn[i] = (cs(c1 + 1, c2 - 1) * 2, cs(c1 - 1, c2 - 1) * 2, cs(c1 + 1, c2 + 1) * 2)
            elif hc:                    # B site
                tn[i] = (cs(c1 - 1, c2 + 1) * 2 - 1, cs(c1 + 1, c2 + 1) * 2 - 1, cs(c1 - 1, c2 - 1) * 2 - 1)
            else:
                tn[i] = (cs(c1 + 2, c2), cs(c1, c2 + 2), cs(c1 - 2, c2), cs(c1, c2 - 2))
        listk = np.array([[m, n] for m in range(-((l1 + 1) // 2) + 1, l1 // 2 + 1)
                          for n in range(-((l2 + 1) // 2) + 1, l2 // 2 + 1)], dtype=np.int64)
    if a2 is None:
        bz1, bz2 = np.array([2.0 * np.pi / a1[0]]), None
    else:
        x = a1[0] * a2[1] - a2[0] * a1[1]
        bz1 = 2.0 * np.pi * np.array([a2[1] / x, -a2[0] / x])
        bz2 = 2.0 * np.pi * np.array([-a1[1] / x, a1[0] / x])
    return dict(list=t["list"], cord=cord, nnlist=t["nnlist"], snlist=t["snlist"], tnlist=tn,
                plq_cord=None if lat == 3 else t["plq_cord"], listk=listk, a1=a1, a2=a2, bz1=bz1, bz2=bz2)


def momentum_list3d(l1: int, l2: int, l3: int) -> np.ndarray:
    """listk of setup_latt3d_sub (src/lattice.f90:1115-1127): (m, n, l) with l
    outermost, then m (along a1), then n (along a2)."""
    return np.array([[m, n, l] for l in range(-((l3 + 1) // 2) + 1, l3 // 2 + 1)
                     for m in range(-((l1 + 1) // 2) + 1, l1 // 2 + 1)
                     for n in range(-((l2 + 1) // 2) + 1, l2 // 2 + 1)], dtype=np.int64)


def zexpiqr3d(l1: int, l2: int, l3: int) -> np.ndarray:
    """zexpiqr(nk, i) = exp(i k_nk . R_i) of the cubic lattice (setup_latt3d_sub,
    src/lattice.f90:1143-1150): R_i the unit-cell coordinates (i1, i2, i3) of
    cell i = (i3-1) l1 l2 + (i1-1) l2 + i2, k = (m/l1, n/l2, l/l3) 2 pi."""
    lk = momentum_list3d(l1, l2, l3)
    c = np.array([(i1, i2, i3) for i3 in range(1, l3 + 1) for i1 in range(1, l1 + 1)
                  for i2 in range(1, l2 + 1)], dtype=float)
    k = 2.0 * np.pi * lk / np.array([l1, l2, l3], dtype=float)
    return np.exp(1j * (k @ c.T))


def print_latt(f, p) -> None:
    """print_latt2d_sub / print_latt1d_sub / print_latt3d_sub (src/lattice.f90:
    146-226, 502-597, 1169-1263): the lattice block of dqmc.out, without the
    PLEVEL2 imj table."""
    L = lattice_lists(p)
    w = f.write

    def vec(a):
        return "".join(_f16_12(float(v)) for v in a)

    def section(title, head, rows, fmt):
        w(" \n --------------------- \n")
        w(f" {title} \n --------------------- \n")
        w(f"{head} \n")
        for i, r in enumerate(rows, start=1):
            w(f"{i:6d}" + "".join(fmt.format(int(v)) for v in r) + "\n")

    if "a3" in L:
        w("lattice information: \n")
        for k in ("a1", "a2", "a3"):
            w(f" primitive lattice vector {k}_p(:) = " + vec(L[k]) + "\n")
        for k in ("bz1", "bz2", "bz3"):
            w(f" primitive reciprocal vector {k}_p(:) / 2pi = " + vec(L[k] / (2.0 * np.pi)) + "\n")
        section("The lattice sites list", "   i     list(i,:)", L["list"], "{:4d}")
        section("The lattice sites cord", "   i     cord(i,:)", L["cord"], "{:4d}")
        section("The lattice nnlist", "   i     nnlist(i,:)", L["nnlist"], "{:4d}")
        section("The lattice snlist", "   i     snlist(i,:)", L["snlist"], "{:4d}")
        section("The lattice tnlist", "   i     tnlist(i,:)", L["tnlist"], "{:4d}")
        section("The lattice plq_cord", "   i     plq_cord(:,i)", L["plq_cord"], "{:4d}")
        section("The momentum listk", "   i     listk(i,:)", L["listk"], "{:4d}")
        return

    w("lattice information: \n")
    w(" primitive lattice  vector a1_p(:) =  " + vec(L["a1"]) + "\n")
    if L["a2"] is not None:
        w(" primitive lattice  vector a2_p(:) =  " + vec(L["a2"]) + "\n")
    w(" primitive reciprocal vector bz1_p / 2pi = " + vec(L["bz1"] / (2.0 * np.pi)) + "\n")
    if L["bz2"] is not None:
        w(" primitive reciprocal vector bz2_p / 2pi = " + vec(L["bz2"] / (2.0 * np.pi)) + "\n")
    section("The lattice sites list", "   i     list(i,:)", L["list"], "{:4d}")
    section("The lattice sites cord", "   i     cord(i,:)", L["cord"], "{:4d}")
    section("The lattice nnlist", "   i     nnlist(i,:)", L["nnlist"], "{:4d}")
    section("The lattice snlist", "   i     snlist(i,:)", L["snlist"], "{:4d}")
    section("The lattice tnlist", "   i     tnlist(i,:)", L["tnlist"], "{:4d}")
    if L["plq_cord"] is not None:
        section("The lattice plq_cord", "   i     plq_cord(:,i)", L["plq_cord"], "{:4d}")
    section("The momentum listk", "   i     listk(i,:)", L["listk"], "{:4d}")


def wrap_step_of(p) -> list:
    """The stabilisation intervals (wrap_step(1:2, n), src/model_para.f90:420-452)."""
    g = p if isinstance(p, dict) else p.as_dict()
    lt, nw, nst = g["ltrot"], g["nwrap"], g["nst"]
    return [((n - 1) * nw + 1, min(n * nw, lt)) for n in range(1, nst + 1)]


def wrap_error_print(f, diags, ltau: bool = False) -> None:
    """wrap_error_print (src/dqmc_util.f90:15-57) of the chains' diagnostics
    (Dqmc.diag dicts): max over chains, averages over all wrap checks; with
    ltau also xmax_dyn and avglog10dynerror of the projective unequal-time
    pass (0/0 prints NaN, as the reference's division does)."""
    mw = max(d["max_wrap_error"] for d in diags)
    mp = max(d["max_phasediff"] for d in diags)
    cnt = sum(d["logcount"] for d in diags)
    a10 = sum(d["avglog10error"] for d in diags) / cnt if cnt else 0.0
    aph = sum(d["avgexpphasediff"] for d in diags) / cnt if cnt else 0.0
    f.write(f"--------------max_wrap_error  = {fortran_e(mw)}\n")
    f.write(f"--------------max_phasediff   = {fortran_e(mp)}\n")
    f.write(f"--------------avglog10error     = {a10:16.8f}\n")
    f.write(f"--------------avgexpphasediff = {aph:16.8f}\n")
    if ltau:
        xd = max(d.get("max_dyn_error", 0.0) for d in diags)
        dc = sum(d.get("dyn_count", 0.0) for d in diags)
        ad = sum(d.get("dyn_log10_sum", 0.0) for d in diags) / dc if dc else float("nan")
        f.write(f"--------------xmax_dyn        = {fortran_e(xd)}\n")
        f.write(f"--------------avglog10dynerror  = {ad:16.8f}\n" if dc else f"--------------avglog10dynerror  = {'NaN':>16}\n")


def update_flavour(p) -> str:
    """The -DTIMING name of the update of a parameter set: ft_ / proj_ and
    fast / delay / submatrix, as dqmc_end prints it (src/dqmc_util.f90:316-355)."""
    g = p if isinstance(p, dict) else p.as_dict()
    kind = {0: "fast", 1: "delay", 2: "submatrix"}[int(g.get("update", 1))]
    return f"{'proj' if g.get('proj', 0) else 'ft'}_{kind}_update"


def dqmc_end_print(f, diags, total_s: float, profile: dict | None = None, date: str = "", params=None,
                   gfunc_s: float = 0.0, dyn_s: float = 0.0, output_s: float = 0.0) -> None:
    """dqmc_end (src/dqmc_util.f90:287-369): acceptance of the U (and t-V bond)
    field over all chains, total time and, given a sweep profile
    (Dqmc.sweep_profile: {kind: (ms, groups)}), the -DTIMING breakdown with the
    reference's line names, the update named by its flavour (params: the
    handle's parameter set; default ft_delay_update).  gfunc_s is the part of
    the update spent updating G (the reference's timecalculation(18..21)); the
    ratio line is the rest, so the two lines add up to the update time as in
    the reference.  The propagation kernels apply the kinetic and the HS
    factors of a slice in one pass, so that pass is charged to H0 and the HI
    lines read zero."""
    def acc(a, p):
        return sum(d[a] for d in diags) / max(1.0, sum(d[p] for d in diags))
    if sum(d.get("proposed_v", 0.0) for d in diags) > 0:
        f.write(f" >>> accep_v     = {fortran_e(acc('accepted_v', 'proposed_v'))}\n")
    if sum(d["proposed"] for d in diags) > 0:
        f.write(f" >>> accep_u     = {fortran_e(acc('accepted', 'proposed'))}\n")
    f.write("\n")
    f.write(f" >>> Total time spent:{total_s:10.2f}s\n")
    f.write(f" >>> Happy ending at {date}\n\n")
    if profile:
        s = {k: v[0] * 1e-3 for k, v in profile.items()}
        inside = sum(s.values())
        tot = inside + output_s
        pct = (lambda t: 100.0 * t / tot if tot else 0.0)
        fl = update_flavour(params) if params is not None else "ft_delay_update"
        upd = s["update"]
        prop = s["prop_left"] + s["prop_right"] + s["bprod"]
        w = f.write
        w(f"The_time_of_sweep_in_total:     {tot:10.3f}s\n")
        w(f"The_time_of_sweep_inside:       {inside:10.3f}s = {pct(inside):6.2f}%\n")
        w(f"The_time_of_propagating:        {prop:10.3f}s = {pct(prop):6.2f}%\n")
        w(f"The_time_of_{fl}:".ljust(32) + f"{upd:10.3f}s = {pct(upd):6.2f}%\n")
        if not fl.endswith("fast_update"):
            w(f"The_time_of_update_gfunc_{fl}:  {gfunc_s:10.3f}s\n")
            w(f"The_time_of_update_ratio_{fl}:  {upd - gfunc_s:10.3f}s\n")
        stab = s["stab"] + s["green"] + s["other"]
        w(f"The_time_of_stabilization:      {stab:10.3f}s = {pct(stab):6.2f}%\n")
        w(f"The_time_of_measuring_equaltime:{s['measure']:10.3f}s = {pct(s['measure']):6.2f}%\n")
        w(f"The_time_of_measuring_dynamic:  {dyn_s:10.3f}s = {pct(dyn_s):6.2f}%\n")
        w(f"The_time_of_outputing_bins      {output_s:10.3f}s = {pct(output_s):6.2f}%\n")
        w(f"The_time_of_H0_left:            {s['prop_left']:10.3f}s\n")
        w(f"The_time_of_H0_right:           {s['prop_right']:10.3f}s\n")
        w(f"The_time_of_HI_left:            {0.0:10.3f}s\n")
        w(f"The_time_of_HI_right:           {0.0:10.3f}s\n")
    f.write(" The simulation done !!! \n")
