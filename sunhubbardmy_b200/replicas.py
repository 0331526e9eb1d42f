"""Replica parallelism across processes (one per GPU).

The reference's only parallelism is independent Markov chains on MPI ranks;
at the end of a bin, equaltime_output (src/dqmc_measure/equaltime_output.f90:14-27)
sums every rank's bins with MPI_Reduce and normalises by isize*nobs.  Here
every process owns a batch of chains on its GPU; the bin buffers (<= 100 KB)
are reduced over ranks with one all-reduce (NCCL over NVLink, or gloo on CPU),
outside any sweep.  Nothing is exchanged while a sweep runs.
"""
from __future__ import annotations

import numpy as np

from .dqmc import test_seed


def replica_seeds(rank: int, chains_per_rank: int) -> list[int]:
    """Seeds of this rank's chains: the reference's -DTEST seed formula for
    global chain index rank*chains_per_rank + c (src/dqmc_util.f90:72)."""
    return [test_seed(rank * chains_per_rank + c) for c in range(chains_per_rank)]


def reduce_bins(local_bins: list[dict], group=None, device: str = "cpu") -> dict:
    """Sum the bin dicts (as returned by Dqmc.bins) of this rank's chains and
    all-reduce them over the process group; returns the normalised averages
    (bin sums / (total chains * nobs)), as equaltime_output writes them."""
    import torch
    import torch.distributed as dist

    keys = [k for k in local_bins[0] if k != "nobs"]
    flat = np.concatenate([np.sum([np.asarray(b[k], complex).ravel() for b in local_bins], axis=0)
                           for k in keys])
    nobs = local_bins[0]["nobs"]
    t = torch.from_numpy(np.concatenate([flat.view(np.float64), [float(len(local_bins))]])).to(device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    arr = t.cpu().numpy()
    nchains = arr[-1]
    z = arr[:-1].view(complex) / (nchains * nobs)
    out, off = {}, 0
    for k in keys:
        shape = np.asarray(local_bins[0][k]).shape
        size = int(np.prod(shape)) if shape else 1
        out[k] = z[off:off + size].reshape(shape) if shape else z[off]
        off += size
    out["chains"] = int(round(nchains))
    out["nobs"] = nobs
    return out
