"""Exact energy of the 2D Ising ferromagnet on an L x L torus -- TEST
INFRASTRUCTURE (the physics reference of the long-run statistical tests).

``kaufman_energy``: Kaufman's (1949) partition function of the finite torus in
the form of Ferdinand and Fisher (1969),
    Z = 1/2 (2 sinh 2K)^(L^2/2) (Z1 + Z2 + Z3 + Z4),
    Z1 = prod_{r=0}^{L-1} 2 cosh(L g_{2r+1}/2),  Z2 = prod 2 sinh(L g_{2r+1}/2),
    Z3 = prod_{r=0}^{L-1} 2 cosh(L g_{2r}/2),    Z4 = prod 2 sinh(L g_{2r}/2),
    cosh g_l = cosh 2K coth 2K - cos(pi l / L) (l >= 1),  g_0 = 2K + ln tanh K,
evaluated in log space with signs; the energy per site e = -(1/L^2) d ln Z/dK
(H = -sum_<ij> s_i s_j, K = beta J) by a central difference.
``transfer_energy`` (column transfer matrix, exact for small L) and
``brute_energy`` (all 2^(L^2) states, L <= 4) pin it.
"""
from __future__ import annotations

import itertools

import numpy as np


def _log_sum_signed(terms):
    """log |sum_i sign_i exp(a_i)| for (sign, a) pairs."""
    m = max(a for _, a in terms)
    return m + np.log(abs(sum(sg * np.exp(a - m) for sg, a in terms)))


def kaufman_lnZ(L: int, K: float) -> float:
    c = np.cosh(2 * K) / np.tanh(2 * K)
    l = np.arange(2 * L)
    g = np.arccosh(c - np.cos(np.pi * l / L))
    g[0] = 2 * K + np.log(np.tanh(K))
    odd, even = g[1::2], g[0::2]

    def lnprod(x, f):
        v = f(L * x / 2)
        return int(np.prod(np.sign(v))), float(np.sum(np.log(2 * np.abs(v))))

    terms = [lnprod(odd, np.cosh), lnprod(odd, np.sinh), lnprod(even, np.cosh), lnprod(even, np.sinh)]
    return -np.log(2.0) + 0.5 * L * L * np.log(2 * np.sinh(2 * K)) + _log_sum_signed(terms)


def kaufman_energy(L: int, K: float, h: float = 1e-6) -> float:
    return -(kaufman_lnZ(L, K + h) - kaufman_lnZ(L, K - h)) / (2 * h) / (L * L)


def transfer_lnZ(L: int, K: float) -> float:
    states = np.array(list(itertools.product([1, -1], repeat=L)), dtype=np.float64)
    intra = (states * np.roll(states, 1, axis=1)).sum(1)
    inter = states @ states.T
    T = np.exp(K * (0.5 * intra[:, None] + 0.5 * intra[None, :] + inter))
    w = np.linalg.eigvalsh(T)
    m = np.abs(w).max()
    return L * np.log(m) + np.log(np.sum((w / m) ** L))


def transfer_energy(L: int, K: float, h: float = 1e-6) -> float:
    return -(transfer_lnZ(L, K + h) - transfer_lnZ(L, K - h)) / (2 * h) / (L * L)


def brute_energy(L: int, K: float) -> float:
    n = L * L
    idx = np.arange(1 << n, dtype=np.int64)
    s = 1 - 2 * ((idx[:, None] >> np.arange(n)) & 1)
    g = s.reshape(-1, L, L)
    bonds = (g * np.roll(g, 1, axis=1)).sum((1, 2)) + (g * np.roll(g, 1, axis=2)).sum((1, 2))
    w = np.exp(K * (bonds - bonds.max()))
    return -float(np.sum(w * bonds) / np.sum(w)) / n
