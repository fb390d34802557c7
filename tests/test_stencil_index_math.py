"""The index arithmetic of the compile-time stencils (StencilDim in
marqov_b200/csrc/engine.h), restated in Python and checked on the CPU against
plain modular arithmetic for every site of small lattices: coordinates by
shifts on power-of-two sides, by multiply-high with the 64-bit reciprocal
ceil(2^64 / len) otherwise (the last coordinate without a remainder), and the
periodic neighbours +x, -x, +y, -y, ... of FixedDimRegularHypercubic::nbrs
(src/lattice/regular_hypercubic.h:31-66) in 32-bit arithmetic; and the
checkerboard site of position t of a colour (parity_site)."""
import numpy as np
import pytest


def _divlen(u, mlen):
    return (u * mlen) >> 64


def _coord(i, j, L, D, lg, mlen):
    u = i
    if lg >= 0:
        v = u >> (lg * j)
        return v if j == D - 1 else v & (L - 1)
    if j >= 1:
        u = _divlen(u, mlen)
    if j >= 2:
        u = _divlen(u, mlen)
    if j == D - 1:
        return u
    return u - _divlen(u, mlen) * L


def _nbr(i, slot, L, D, lg, mlen):
    j = slot >> 1
    p = L ** j
    w = ((L - 1) * p) & 0xFFFFFFFF
    x = _coord(i, j, L, D, lg, mlen)
    if slot & 1 == 0:
        return (i - w) & 0xFFFFFFFF if x == L - 1 else (i + p) & 0xFFFFFFFF
    return (i + w) & 0xFFFFFFFF if x == 0 else (i - p) & 0xFFFFFFFF


def _parity_site(t, colour, L, D, lg, mlen):
    i0 = 2 * t
    par = sum(_coord(i0, j, L, D, lg, mlen) for j in range(1, D))
    return i0 + (1 if (par & 1) != colour else 0)


@pytest.mark.parametrize("D,L", [(2, 6), (2, 10), (2, 12), (2, 16), (2, 48), (3, 6), (3, 8), (3, 10), (3, 12),
                                 (3, 14)])
def test_stencil_coordinates_and_neighbours(D, L):
    lg = L.bit_length() - 1 if L & (L - 1) == 0 else -1
    mlen = ((1 << 64) - 1) // L + 1  # as the host computes it: ceil(2^64 / L) for L not a power of two
    n = L ** D
    idx = np.arange(n)
    coords = [(idx // L ** j) % L for j in range(D)]
    for i in range(n):
        for j in range(D):
            assert _coord(i, j, L, D, lg, mlen) == coords[j][i]
        for slot in range(2 * D):
            j, sgn = slot >> 1, (1 if slot % 2 == 0 else -1)
            c = [coords[k][i] for k in range(D)]
            c[j] = (c[j] + sgn) % L
            assert _nbr(i, slot, L, D, lg, mlen) == sum(c[k] * L ** k for k in range(D))
    # the two colours of the checkerboard partition the sites
    for colour in (0, 1):
        sites = {_parity_site(t, colour, L, D, lg, mlen) for t in range(n // 2)}
        assert len(sites) == n // 2
        assert all(sum(coords[k][s] for k in range(D)) % 2 == colour for s in sites)


def test_multiply_high_division_is_exact_for_32_bit_indices():
    rng = np.random.default_rng(7)
    for L in (3, 6, 10, 12, 48, 96, 192, 320, 384, 1000, 1290):
        mlen = ((1 << 64) - 1) // L + 1
        for u in list(rng.integers(0, 1 << 32, 2000)) + [0, L - 1, L, (1 << 32) - 1]:
            u = int(u)
            assert _divlen(u, mlen) == u // L
