"""CPU restatement of the learned effective action (test infrastructure only).

The checker for the tensor-core kernels of sunhubbardmy_b200/csrc/kern_nn.cu:
the forward value S(s) of the 3-layer periodic convolutional network and the
gradient of sum_b r_b S(s_b) with respect to its parameters, in float64 numpy,
with optional rounding to bfloat16 at the points where the CUDA kernels store
bfloat16 (W2, h1, the stored h2, dpre2), so that the comparison isolates the
FP32-versus-FP64 accumulation.

This network has no counterpart in the reference (it is the learned proposal
the build adds beside the reference's local updates); the layout of the flat
parameter vector follows include/dqmc_gpu.h:
  W1[27][32], b1[32], W2[27][32 in][32 out], b2[32], w3[32], b3,
tap = 9 (dt+1) + 3 (dy+1) + (dx+1), out(v) = sum_tap W[tap] in(v + off(tap)).
"""
from __future__ import annotations

import numpy as np

C = 32
NP = 27 * C + C + 27 * C * C + C + C + 1
OFFS = [(dt, dy, dx) for dt in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float64 values to bfloat16 (round to nearest even), returned as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = (u + 0x7FFF + lsb) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(theta: np.ndarray):
    th = np.asarray(theta, np.float64)
    k = 0
    W1 = th[k:k + 27 * C].reshape(27, C); k += 27 * C
    b1 = th[k:k + C]; k += C
    W2 = th[k:k + 27 * C * C].reshape(27, C, C); k += 27 * C * C
    b2 = th[k:k + C]; k += C
    w3 = th[k:k + C]; k += C
    b3 = th[k]
    return W1, b1, W2, b2, w3, b3


def shift(a: np.ndarray, off) -> np.ndarray:
    """a(v + off) for a[..., t, y, x] with periodic boundaries (channel-last
    arrays [t, y, x, c] are handled by the caller)."""
    dt, dy, dx = off
    return np.roll(a, (-dt, -dy, -dx), axis=(0, 1, 2))


def forward(theta, s, emulate_bf16=True, keep=False):
    """S for one field s[t, y, x] = +-1."""
    W1, b1, W2, b2, w3, b3 = unpack(theta)
    rb = bf16 if emulate_bf16 else (lambda x: np.asarray(x, np.float64))
    s = np.asarray(s, np.float64)
    pre1 = np.zeros(s.shape + (C,)) + b1
    for tap, off in enumerate(OFFS):
        pre1 += shift(s, off)[..., None] * W1[tap]
    h1 = rb(np.tanh(pre1))
    W2r = rb(W2)
    pre2 = np.zeros(s.shape + (C,)) + b2
    for tap, off in enumerate(OFFS):
        pre2 += shift(h1, off) @ W2r[tap]
    h2 = np.tanh(pre2)
    S = float(np.sum(h2 @ w3) + b3 * s.size)
    if keep:
        return S, dict(s=s, h1=h1, h2=h2, W2r=W2r)
    return S


def gradient(theta, fields, r, emulate_bf16=True):
    """(S_b, d/dtheta sum_b r_b S_b) by backpropagation."""
    W1, b1, W2, b2, w3, b3 = unpack(theta)
    rb = bf16 if emulate_bf16 else (lambda x: np.asarray(x, np.float64))
    g = np.zeros(NP)
    gW1 = np.zeros((27, C)); gb1 = np.zeros(C); gW2 = np.zeros((27, C, C)); gb2 = np.zeros(C)
    gw3 = np.zeros(C); gb3 = 0.0
    Ss = []
    for f, rr in zip(fields, r):
        S, a = forward(theta, f, emulate_bf16, keep=True)
        Ss.append(S)
        s, h1, h2, W2r = a["s"], a["h1"], a["h2"], a["W2r"]
        h2s = rb(h2)                            # the stored h2
        gw3 += rr * h2s.reshape(-1, C).sum(0)
        gb3 += rr * s.size
        dp2 = rb(rr * w3 * (1.0 - h2s * h2s))
        gb2 += dp2.reshape(-1, C).sum(0)
        dh1 = np.zeros_like(h1)
        for tap, off in enumerate(OFFS):
            gW2[tap] += np.einsum("tyxi,tyxo->io", shift(h1, off), dp2)
            # h1 at u feeds out(u - off): dh1(u) += W2 dpre2(u - off)
            dh1 += shift(dp2, tuple(-o for o in off)) @ W2r[tap].T
        dp1 = dh1 * (1.0 - h1 * h1)
        gb1 += dp1.reshape(-1, C).sum(0)
        for tap, off in enumerate(OFFS):
            gW1[tap] += np.einsum("tyx,tyxc->c", shift(s, off), dp1)
    k = 0
    for part in (gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]):
        part = np.asarray(part, np.float64)
        g[k:k + part.size] = part
        k += part.size
    return np.array(Ss), g
