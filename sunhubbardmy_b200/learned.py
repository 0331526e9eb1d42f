"""Learned effective action and global block proposals (host side).

A 3-layer periodic convolutional network S(s) over the (ltrot x L x L) HS
field approximates -log |W(s)|.  It is trained by the library's own
tensor-core forward and backward kernels (kern_nn.cu) on (field, log weight)
pairs recorded at every stabilisation of the plain sweeps, and then proposes
global 8 x 4 x 4 block flips that the exact determinant ratio accepts or
rejects (dqmc_gpu_sweep_learned).  The plain local updates keep running in
every learned sweep, so the method without the network is also the fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .dqmc import DqmcError, _check, _ptr, load_library


class EffectiveAction:
    """The network; parameters and Adam state live on the GPU."""

    def __init__(self, ltrot: int, L: int, max_batch: int = 64, seed: int = 1):
        self.ltrot, self.L, self.max_batch = int(ltrot), int(L), int(max_batch)
        h = C.c_void_p()
        _check(load_library().dqmc_nn_create(self.ltrot, self.L, self.max_batch, C.c_uint64(seed), C.byref(h)),
               "dqmc_nn_create")
        self.h = h
        self.nparams = load_library().dqmc_nn_nparams()

    def close(self):
        if getattr(self, "h", None):
            load_library().dqmc_nn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.zeros(self.nparams, np.float32)
        _check(load_library().dqmc_nn_get_params(self.h, _ptr(out)), "get_params")
        return out

    def set_params(self, theta) -> None:
        a = np.ascontiguousarray(theta, np.float32)
        if a.size != self.nparams:
            raise DqmcError(f"expected {self.nparams} parameters")
        _check(load_library().dqmc_nn_set_params(self.h, _ptr(a)), "set_params")

    def _fields(self, fields) -> np.ndarray:
        f = np.ascontiguousarray(fields, np.int8)
        if f.ndim == 3:
            f = f[None]
        if f.shape[1:] != (self.ltrot, self.L, self.L):
            raise DqmcError("fields must be int8 [B][ltrot][L][L]")
        return f

    def forward(self, fields) -> np.ndarray:
        f = self._fields(fields)
        S = np.zeros(f.shape[0])
        _check(load_library().dqmc_nn_forward(self.h, _ptr(f), f.shape[0], _ptr(S)), "nn_forward")
        return S

    def gradient(self, fields, r):
        f = self._fields(fields)
        rr = np.ascontiguousarray(r, np.float64)
        S = np.zeros(f.shape[0])
        g = np.zeros(self.nparams, np.float32)
        _check(load_library().dqmc_nn_gradient(self.h, _ptr(f), f.shape[0], _ptr(rr), _ptr(S), _ptr(g)), "nn_gradient")
        return S, g

    def train_step(self, fields, y, lr: float = 1e-3) -> float:
        f = self._fields(fields)
        yy = np.ascontiguousarray(y, np.float64)
        loss = C.c_double()
        _check(load_library().dqmc_nn_train_step(self.h, _ptr(f), _ptr(yy), f.shape[0], float(lr), C.byref(loss)),
               "nn_train_step")
        return loss.value

    def train_recorded(self, g, idx, y, lr: float = 1e-3) -> float:
        ii = np.ascontiguousarray(idx, np.int32)
        yy = np.ascontiguousarray(y, np.float64)
        loss = C.c_double()
        _check(load_library().dqmc_nn_train_recorded(self.h, g.h, _ptr(ii), _ptr(yy), len(ii), float(lr),
                                                     C.byref(loss)), "nn_train_recorded")
        return loss.value

    def train_recorded_pairs(self, g, idx_a, idx_b, dy, lr: float = 1e-3) -> float:
        """One Adam step on (S(b) - S(a) - dy)^2 over recorded pairs."""
        ia = np.ascontiguousarray(idx_a, np.int32)
        ib = np.ascontiguousarray(idx_b, np.int32)
        yy = np.ascontiguousarray(dy, np.float64)
        loss = C.c_double()
        _check(load_library().dqmc_nn_train_recorded_pairs(self.h, g.h, _ptr(ia), _ptr(ib), _ptr(yy), len(ia),
                                                           float(lr), C.byref(loss)), "nn_train_recorded_pairs")
        return loss.value


def collect(g, sweeps: int, capacity: int) -> np.ndarray:
    """Run `sweeps` plain sweeps recording (field, nflr Re log W) at every
    stabilisation; returns the targets -log|W| of the filled slots."""
    g.record(capacity)
    g.sweeps(sweeps, False)
    n = g.record_count()
    vals = g.record_values(capacity)[:n]
    g.record(0)
    return -vals


def train(nn: EffectiveAction, g, targets: np.ndarray, steps: int, batch: int = 32, lr: float = 1e-3,
          seed: int = 0, slots=None, pair_lag: int = 0, diff_every: int = 0) -> list:
    """Adam on minibatches of the recorded pairs; returns the loss history.
    targets[k] is the target of record slot slots[k] (slots defaults to
    0..len(targets)-1, i.e. all recorded pairs in order).  With pair_lag > 0
    and diff_every = d > 0, every d-th step instead fits the difference of the
    targets of slots s and s + pair_lag (the same chain one stabilisation later
    when pair_lag = n_chains), among the slots given."""
    rng = np.random.default_rng(seed)
    n = len(targets)
    slots = np.arange(n, dtype=np.int32) if slots is None else np.asarray(slots, np.int32)
    if len(slots) != n:
        raise ValueError("slots and targets differ in length")
    by_slot = {int(sl): t for sl, t in zip(slots, targets)}
    pairs = np.array([sl for sl in slots if int(sl) + pair_lag in by_slot], np.int32) if pair_lag > 0 else None
    losses = []
    for step in range(steps):
        if diff_every > 0 and pairs is not None and len(pairs) and step % diff_every == diff_every - 1:
            a = pairs[rng.integers(0, len(pairs), size=min(batch // 2, len(pairs)))]
            b = a + pair_lag
            dy = np.array([by_slot[int(y)] - by_slot[int(x)] for x, y in zip(a, b)])
            losses.append(nn.train_recorded_pairs(g, a, b, dy, lr))
        else:
            k = rng.integers(0, n, size=min(batch, n))
            losses.append(nn.train_recorded(g, slots[k], targets[k], lr))
    return losses
