"""Batched chains of uneven sizes and the delay-depth autotuner.

A handle advances many independent chains in one launch per kernel (one CTA
per chain), the GPU form of the reference's one-chain-per-MPI-rank runs
(src/dqmc_main.f90).  Chains may have different lattice sizes as long as they
share ltrot, nwrap, the lattice kind and the kinetic propagator.

The flush depth (nublock: accepted flips folded into G by one tensor-core
GEMM) trades GEMM efficiency against the cost of building longer delayed
columns.  `tune_nublock` times one sweep per candidate for each size class on
the device and keeps the fastest; it never changes the accept sequence.

One handle runs every kernel over all its chains, so a kernel lasts as long as
its largest chain's CTA: with chains of N = 72, 162 and 288 in one handle, the
SMs of the small chains idle while the N = 288 CTAs finish.  `ChainGroup`
instead gives each size class (split into a few handles) its own stream
(dqmc_gpu_sweeps_multi): the small classes' kernels fill the SMs that the
large class's long kernels leave free.  Chains are independent and each
keeps its seed, so a group gives the same fields, Green's functions and bins
as one handle of all its chains.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .dqmc import Dqmc, DqmcParams, sweep_start_concurrent, sweeps_concurrent, test_seed


def with_nublock(p: DqmcParams, nb: int) -> DqmcParams:
    q = DqmcParams()
    C.memmove(C.byref(q), C.byref(p), C.sizeof(DqmcParams))
    q.nublock = nb
    return q


def tune_nublock(p: DqmcParams, chains: int, candidates=(16, 32, 64), sweeps: int = 1) -> tuple[int, dict]:
    """Device ms per sweep for each candidate depth on `chains` chains of p."""
    times = {}
    for nb in candidates:
        with Dqmc(with_nublock(p, nb), n_chains=chains) as g:
            g.sweep_start()
            g.sweeps(1, True)                  # captures the sweep graph
            times[nb] = g.sweeps(sweeps, True)
    best = min(times, key=times.get)
    return best, times


def batched(groups, tune: bool = True, candidates=(16, 32, 64), tune_chains: int = 8, seed0: int = 0):
    """One handle for groups = [(params, n_chains), ...]; returns (Dqmc, report).
    Chain order: all chains of the first group, then the second, ...  Seeds are
    the -DTEST formula for consecutive global chain indices."""
    plist, report = [], {}
    for p, n in groups:
        if tune:
            nb, t = tune_nublock(p, min(n, tune_chains), candidates)
            report[p.ndim] = {"nublock": nb, "ms_per_sweep": t}
            p = with_nublock(p, nb)
        plist += [p] * n
    seeds = [test_seed(seed0 + c) for c in range(len(plist))]
    return Dqmc(plist, n_chains=len(plist), seeds=seeds), report


class ChainGroup:
    """Several handles whose sweeps run concurrently, each on its own stream,
    behind the per-chain interface of one handle: chain c of the group is
    chain c - offset of the handle that holds it, in handle order."""

    MAX_HANDLES = 16        # dqmc_gpu_sweeps_multi

    def __init__(self, handles, params_per_chain=None, seeds=None):
        if not 1 <= len(handles) <= self.MAX_HANDLES:
            raise ValueError(f"1..{self.MAX_HANDLES} handles")
        self.handles = list(handles)
        self.offsets = []
        k = 0
        for h in self.handles:
            self.offsets.append(k)
            k += h.n_chains
        self.n_chains = k
        self.params = [q for h in self.handles for q in (h.params if len(h.params) > 1 else h.params * h.n_chains)]
        self._plist = params_per_chain if params_per_chain is not None else self.params
        self._seeds = seeds if seeds is not None else [int(s) for h in self.handles for s in h.seeds]

    def _h(self, c):
        for h, o in zip(reversed(self.handles), reversed(self.offsets)):
            if c >= o:
                return h, c - o
        raise IndexError(c)

    @property
    def ltrot(self) -> int:
        return self.handles[0].ltrot

    def sweeps(self, n: int, lmeasure: bool = True) -> float:
        return sweeps_concurrent(self.handles, n, lmeasure)

    def sweep_start(self) -> None:
        sweep_start_concurrent(self.handles)

    def obser_init(self) -> None:
        for h in self.handles:
            h.obser_init()

    def reset_diag(self) -> None:
        for h in self.handles:
            h.reset_diag()

    def close(self) -> None:
        for h in self.handles:
            h.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def sweep_kernels(self) -> int:
        return sum(h.sweep_kernels() for h in self.handles)

    def ndim(self, c: int = 0) -> int:
        h, cc = self._h(c)
        return h.ndim(cc)

    def diag(self, c: int = 0) -> dict:
        h, cc = self._h(c)
        return h.diag(cc)

    def bins_raw(self, c: int = 0):
        h, cc = self._h(c)
        return h.bins_raw(cc)

    def conf(self, c: int = 0):
        h, cc = self._h(c)
        return h.conf(cc)

    def green(self, c: int = 0):
        h, cc = self._h(c)
        return h.green(cc)

    def vconf(self, c: int = 0):
        h, cc = self._h(c)
        return h.vconf(cc)

    def set_vconf(self, v, c: int = 0) -> None:
        h, cc = self._h(c)
        h.set_vconf(v, cc)

    def _conf_sizes(self):
        return [sum(h.ltrot * h.ndim(c) for c in range(h.n_chains)) for h in self.handles]

    def conf_all(self, out=None):
        """Every chain's HS field in group chain order (the layout of
        Dqmc.conf_all for one handle of all the chains)."""
        sizes = self._conf_sizes()
        if out is None:
            out = np.zeros(sum(sizes), np.int32)
        o = 0
        for h, n in zip(self.handles, sizes):
            h.conf_all(out[o:o + n])
            o += n
        return out

    def set_conf_all(self, conf) -> None:
        o = 0
        for h, n in zip(self.handles, self._conf_sizes()):
            h.set_conf_all(np.ascontiguousarray(conf[o:o + n]))
            o += n

    def sweep_profile(self, n: int = 1, lmeasure: bool = True) -> dict:
        """The per-kind profile of one handle holding all the group's chains
        (built for it, one sweep after sweep_start): the kernels' own times,
        which concurrent streams would mix."""
        g = Dqmc(self._plist, n_chains=self.n_chains, seeds=self._seeds)
        try:
            g.sweep_start()
            g.obser_init()
            g.sweeps(1, True)
            return g.sweep_profile(n, lmeasure)
        finally:
            g.close()


def size_classes(groups, tune: bool = True, candidates=(16, 32, 64), tune_chains: int = 8, seed0: int = 0,
                 split: int = 0) -> tuple[ChainGroup, dict]:
    """groups = [(params, n_chains), ...] as for `batched`, run as a ChainGroup:
    each group (a size class) in `split` handles of its own (0: as many as
    keep the total at 16 or below, at most 4 per class).  Same chain order
    and seeds as `batched`."""
    if split <= 0:
        split = max(1, min(4, ChainGroup.MAX_HANDLES // max(1, len(groups))))
    handles, plist, seeds, report = [], [], [], {}
    c0 = seed0
    for p, n in groups:
        if tune:
            nb, t = tune_nublock(p, min(n, tune_chains), candidates)
            report[p.ndim] = {"nublock": nb, "ms_per_sweep": t}
            p = with_nublock(p, nb)
        parts = [n // split + (1 if j < n % split else 0) for j in range(min(split, n))]
        for k in parts:
            sd = [test_seed(c0 + c) for c in range(k)]
            handles.append(Dqmc(p, n_chains=k, seeds=sd))
            plist += [p] * k
            seeds += sd
            c0 += k
    return ChainGroup(handles, plist, seeds), report
