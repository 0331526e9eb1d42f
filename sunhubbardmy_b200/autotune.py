"""Batched chains of uneven sizes and the delay-depth autotuner.

A handle advances many independent chains in one launch per kernel (one CTA
per chain), the GPU form of the reference's one-chain-per-MPI-rank runs
(src/dqmc_main.f90).  Chains may have different lattice sizes as long as they
share ltrot, nwrap, the lattice kind and the kinetic propagator.

The flush depth (nublock: accepted flips folded into G by one tensor-core
GEMM) trades GEMM efficiency against the cost of building longer delayed
columns.  `tune_nublock` times one sweep per candidate for each size class on
the device and keeps the fastest; it never changes the accept sequence.
"""
from __future__ import annotations

import ctypes as C

from .dqmc import Dqmc, DqmcParams, test_seed


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
