"""Exact Trotterised expectation values of a small Hubbard ring, for tests.

DQMC samples the Trotterised partition function Z = Tr B^Lt exactly (the
discrete HS decoupling of exp(-dtau U/2 (n - 1)^2) is an identity), so its
equal-time averages must agree, within statistical error only, with
Tr[B^Lt O] / Tr[B^Lt] computed in Fock space.  Here B is the slice operator of
the sweep's B products for the chain lattice: the two checkerboard families'
half steps around the interaction, B = K1 K2 V K2 K1 (K_f = exp(-dtau k_f / 2)
of bond family f, V = exp(-dtau U/2 sum_i (n_i - 1)^2)), or with the dense
kinetic term B = K V K, K = exp(-dtau k / 2).  The Fock space is split into
sectors of fixed (N_up, N_dn), which every factor conserves.
"""
from itertools import combinations

import numpy as np
from scipy.linalg import expm


def _hop(states, index, bonds, t):
    """One-spin hopping -t sum_bonds (c_a^+ c_b + h.c.) in the basis `states`."""
    H = np.zeros((len(states), len(states)))
    for k, s in enumerate(states):
        occ = set(s)
        for (i, j) in bonds:
            for (a, b) in ((i, j), (j, i)):
                if b in occ and a not in occ:
                    new = tuple(sorted((occ - {b}) | {a}))
                    lo, hi = min(a, b), max(a, b)
                    sgn = (-1) ** sum(1 for x in occ if lo < x < hi)
                    H[index[new], k] += -t * sgn
    return H


def chain_bonds(L):
    """The chain's two bond families (0-based sites): bonds (A, A+1) and (A, A-1)
    from the A sites, the odd 0-based (even 1-based) sites."""
    A = [i for i in range(L) if (i + 1) % 2 == 0]
    return [[(a, (a + 1) % L) for a in A], [(a, (a - 1) % L) for a in A]]


def trotter_ring(L, t, U, beta, dtau, dense=False):
    """(double occupancy per site, kinetic energy per site) of the Trotterised
    SU(2) Hubbard ring of L sites at mu = 0."""
    fam = chain_bonds(L)
    allb = fam[0] + fam[1]
    Lt = int(round(beta / dtau))
    z = dsum = ksum = 0.0
    for nu in range(L + 1):
        for nd in range(L + 1):
            ups = list(combinations(range(L), nu))
            dns = list(combinations(range(L), nd))
            iu = {s: k for k, s in enumerate(ups)}
            idn = {s: k for k, s in enumerate(dns)}
            du, dd = len(ups), len(dns)
            if dense:
                Ku = expm(-0.5 * dtau * _hop(ups, iu, allb, t))
                Kd = expm(-0.5 * dtau * _hop(dns, idn, allb, t))
                Lu, Ru, Ld, Rd = Ku, Ku, Kd, Kd
            else:
                k1u, k2u = (expm(-0.5 * dtau * _hop(ups, iu, f, t)) for f in fam)
                k1d, k2d = (expm(-0.5 * dtau * _hop(dns, idn, f, t)) for f in fam)
                Lu, Ru, Ld, Rd = k1u @ k2u, k2u @ k1u, k1d @ k2d, k2d @ k1d
            nu_occ = np.array([[1.0 if i in s else 0.0 for i in range(L)] for s in ups]).reshape(du, L)
            nd_occ = np.array([[1.0 if i in s else 0.0 for i in range(L)] for s in dns]).reshape(dd, L)
            n = nu_occ[:, None, :] + nd_occ[None, :, :]
            V = np.exp(-0.5 * dtau * U * ((n - 1.0) ** 2).sum(-1)).ravel()
            D = ((nu_occ[:, None, :] * nd_occ[None, :, :]).sum(-1) / L).ravel()
            left = np.kron(Lu, Ld)
            right = np.kron(Ru, Rd)
            B = left @ (V[:, None] * right)
            P = np.linalg.matrix_power(B, Lt)
            hu, hd = _hop(ups, iu, allb, t), _hop(dns, idn, allb, t)
            K = np.kron(hu, np.eye(dd)) + np.kron(np.eye(du), hd)
            z += np.trace(P)
            dsum += np.trace(P * D[None, :])
            ksum += np.trace(P @ K)
    return dsum / z, ksum / z / L


def trotter_tv_ring(L, t, V, beta, dtau):
    """(density per site, kinetic energy per site) of the Trotterised spinless
    t-V ring of L sites at mu = 0, as sampled by the bond field.

    The field of bond b = (i, j) enters the slice as exp(a eta K_b), K_b =
    c_i^+ c_j + c_j^+ c_i and cosh a = exp(dtau V / 2) (the Hadamard mix, the
    scale by exp(+-a eta), the mix again).  Summed over eta = +-1 it gives
    2 cosh(a K_b) = 2 exp(dtau V / 2 K_b^2) with K_b^2 = n_i + n_j - 2 n_i n_j
    diagonal in the occupation basis, so the slice operator is
    B = K1 K2 W K2 K1 with W = prod_b exp(dtau V / 2 (n_i + n_j - 2 n_i n_j))."""
    fam = chain_bonds(L)
    allb = fam[0] + fam[1]
    Lt = int(round(beta / dtau))
    z = nsum = ksum = 0.0
    for n in range(L + 1):
        sts = list(combinations(range(L), n))
        idx = {s: k for k, s in enumerate(sts)}
        k1, k2 = (expm(-0.5 * dtau * _hop(sts, idx, f, t)) for f in fam)
        occ = np.array([[1.0 if i in s else 0.0 for i in range(L)] for s in sts]).reshape(len(sts), L)
        ksq = sum(occ[:, i] + occ[:, j] - 2.0 * occ[:, i] * occ[:, j] for (i, j) in allb)
        W = np.exp(0.5 * dtau * V * ksq)
        B = (k1 @ k2) @ (W[:, None] * (k2 @ k1))
        P = np.linalg.matrix_power(B, Lt)
        z += np.trace(P)
        nsum += np.trace(P) * n / L
        ksum += np.trace(P @ _hop(sts, idx, allb, t))
    return nsum / z, ksum / z / L


def binned_mean(x, nbins=20):
    """Mean and standard error from nbins consecutive bins of the series x."""
    x = np.asarray(x, float)
    m = len(x) // nbins * nbins
    b = x[:m].reshape(nbins, -1).mean(axis=1)
    return float(b.mean()), float(b.std(ddof=1) / np.sqrt(nbins))
