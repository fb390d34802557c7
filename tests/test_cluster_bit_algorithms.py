"""The bit-parallel steps of the cluster kernels, restated lane by lane in
Python and checked against breadth-first search on random bond sets (CPU).

* The single-warp flood fill of the resident path (smem_emcs.cu,
  resident_fill_warp2): 2D lattices of at most 64 x 64 sites, two rows per
  lane; per pass, prefix scans over the lanes upwards and downwards from the
  same start (with the loop-invariant propagate masks of every scan step),
  the periodic y bond of the last row, then every row closed as a line by
  additions (row_close_up on the row and on its bit reversal), joined through
  its periodic x bond and closed again; until no lane changes.
* The bonds the labelling hook takes one thread each (wolff_ccl.cuh,
  ccl_hook): exactly the forward bonds that leave a 16 x 16 (2D) or
  8 x 8 x 4 (3D) tile.
"""
import collections

import numpy as np
import pytest

LANES = 32
STEPS = (1, 2, 4, 8, 16)


def _brev(x: int, bits: int) -> int:
    return int(format(x, f"0{bits}b")[::-1], 2)


def _close_up(S: int, A: int, M: int) -> int:
    E = (S << 1) & A & M
    return (S | E | ((((A + E) & M) ^ A) & A)) & M


def _row_close(S: int, Aup: int, Adn: int, T: int) -> int:
    M = (1 << T) - 1
    return _brev(_close_up(_brev(_close_up(S, Aup, M), T), Adn, M), T)


def fill_warp2(F, Bx, By, R, L):
    """Lane-by-lane restatement of resident_fill_warp2 (words of 32 sites,
    WR words per row); returns the closed flood plane and the passes used."""
    WR = (L + 31) // 32
    T = 32 * WR
    M = (1 << T) - 1
    ra, ka = (R - 1) >> 1, (R - 1) & 1
    top = 1 << (L - 1)
    ends = top | 1

    def row(a, r):
        return sum(a[r * WR + q] << (32 * q) for q in range(WR))

    G = [[0, 0] for _ in range(LANES)]
    Aup = [[0, 0] for _ in range(LANES)]
    Adn = [[0, 0] for _ in range(LANES)]
    wrap = [[False, False] for _ in range(LANES)]
    up = [[[0, 0], [0, 0]] for _ in range(LANES)]
    for ln in range(LANES):
        for k in range(2):
            r = 2 * ln + k
            if r >= R:
                continue
            G[ln][k] = row(F, r)
            b = row(Bx, r)
            wrap[ln][k] = bool(b & top)
            b &= ~top
            Aup[ln][k] = (b << 1) & M
            Adn[ln][k] = _brev(b, T)
            for q in range(WR):
                up[ln][k][q] = By[r * WR + q] if r < R - 1 else 0
    wb = [By[(R - 1) * WR + q] for q in range(WR)]
    pin = [[0] * WR for _ in range(LANES)]
    Pu = [[[0] * 5 for _ in range(WR)] for _ in range(LANES)]
    Pd = [[[0] * 5 for _ in range(WR)] for _ in range(LANES)]
    for q in range(WR):
        b01 = [up[ln][0][q] for ln in range(LANES)]
        b1n = [up[ln][1][q] for ln in range(LANES)]
        p_in = [0] + b1n[:-1]
        P = [p_in[ln] & b01[ln] for ln in range(LANES)]
        for s, o in enumerate(STEPS):
            for ln in range(LANES):
                Pu[ln][q][s] = P[ln]
            P = [(P[ln] & P[ln - o]) if ln >= o else P[ln] for ln in range(LANES)]
        P = [b1n[ln] & b01[ln] for ln in range(LANES)]
        for s, o in enumerate(STEPS):
            for ln in range(LANES):
                Pd[ln][q][s] = P[ln]
            P = [(P[ln] & P[ln + o]) if ln + o < LANES else P[ln] for ln in range(LANES)]
        for ln in range(LANES):
            pin[ln][q] = p_in[ln]
    passes = 0
    while True:
        passes += 1
        moved = False
        Y = [[0, 0] for _ in range(LANES)]
        for q in range(WR):
            g0 = [(G[ln][0] >> (32 * q)) & 0xFFFFFFFF for ln in range(LANES)]
            g1 = [(G[ln][1] >> (32 * q)) & 0xFFFFFFFF for ln in range(LANES)]
            b01 = [up[ln][0][q] for ln in range(LANES)]
            b1n = [up[ln][1][q] for ln in range(LANES)]
            x0 = [g0[ln] | (g1[ln] & b01[ln]) for ln in range(LANES)]
            x1 = [g1[ln] | (g0[ln] & b01[ln]) for ln in range(LANES)]
            Xu, Xd = x1[:], x0[:]
            for s, o in enumerate(STEPS):
                Uo = [Xu[ln - o] if ln >= o else Xu[ln] for ln in range(LANES)]
                Do = [Xd[ln + o] if ln + o < LANES else Xd[ln] for ln in range(LANES)]
                Xu = [(Xu[ln] | (Pu[ln][q][s] & Uo[ln])) if ln >= o else Xu[ln] for ln in range(LANES)]
                Xd = [(Xd[ln] | (Pd[ln][q][s] & Do[ln])) if ln + o < LANES else Xd[ln] for ln in range(LANES)]
            below, above = [0] + Xu[:-1], Xd[1:] + [0]
            n0 = [x0[ln] | (below[ln] & pin[ln][q]) for ln in range(LANES)]
            n1 = [x1[ln] | (above[ln] & b1n[ln]) for ln in range(LANES)]
            y0 = [n0[ln] | (n1[ln] & b01[ln]) for ln in range(LANES)]
            y1 = [n1[ln] | (n0[ln] & b01[ln]) for ln in range(LANES)]
            last, first = (y1 if ka else y0)[ra], y0[0]
            y0[0] |= last & wb[q]
            if ka:
                y1[ra] |= first & wb[q]
            else:
                y0[ra] |= first & wb[q]
            for ln in range(LANES):
                moved |= bool((y0[ln] ^ g0[ln]) | (y1[ln] ^ g1[ln]))
                Y[ln][0] |= y0[ln] << (32 * q)
                Y[ln][1] |= y1[ln] << (32 * q)
        for ln in range(LANES):
            for k in range(2):
                X = _row_close(Y[ln][k], Aup[ln][k], Adn[ln][k], T)
                if wrap[ln][k] and (X & ends):
                    X |= ends
                X = _row_close(X, Aup[ln][k], Adn[ln][k], T)
                moved |= X != Y[ln][k]
                G[ln][k] = X
        if not moved:
            break
    out = [0] * (R * WR)
    for ln in range(LANES):
        for k in range(2):
            r = 2 * ln + k
            if r < R:
                for q in range(WR):
                    out[r * WR + q] = (G[ln][k] >> (32 * q)) & 0xFFFFFFFF
    return out, passes


def _component(bx, by, L, sy, sx):
    seen = np.zeros((L, L), bool)
    seen[sy, sx] = True
    todo = collections.deque([(sy, sx)])
    while todo:
        y, x = todo.popleft()
        for ny, nx, b in ((y, (x + 1) % L, bx[y, x]), (y, (x - 1) % L, bx[y, (x - 1) % L]),
                          ((y + 1) % L, x, by[y, x]), ((y - 1) % L, x, by[(y - 1) % L, x])):
            if b and not seen[ny, nx]:
                seen[ny, nx] = True
                todo.append((ny, nx))
    return seen


def _pack(m, L):
    WR = (L + 31) // 32
    return [int(sum(1 << b for b in range(32) if 32 * q + b < L and m[r, 32 * q + b])) for r in range(L)
            for q in range(WR)]


@pytest.mark.parametrize("L", [2, 3, 5, 16, 31, 32, 33, 48, 63, 64])
@pytest.mark.parametrize("p", [0.3, 0.55, 0.8, 1.0])
def test_single_warp_fill_is_the_component(L, p):
    rng = np.random.default_rng(1000 * L + int(100 * p))
    for _ in range(2):
        bx, by = rng.random((L, L)) < p, rng.random((L, L)) < p
        sy, sx = int(rng.integers(L)), int(rng.integers(L))
        F = [0] * (L * ((L + 31) // 32))
        F[sy * ((L + 31) // 32) + sx // 32] = 1 << (sx % 32)
        out, passes = fill_warp2(F, _pack(bx, L), _pack(by, L), L, L)
        assert out == _pack(_component(bx, by, L, sy, sx), L)
        assert passes <= L * L + 1


def _leaving_bonds(tile, L):
    """(offset, direction) of every forward bond of tile 0 whose other end
    lies in another tile (the neighbour's coordinate, periodic, in another
    tile along that direction)."""
    out = set()
    for o in range(256):
        if tile == 2:
            c, w = (o & 15, o >> 4), (16, 16)
        else:
            c, w = (o & 7, (o >> 3) & 7, o >> 6), (8, 8, 4)
        for d in range(len(c)):
            n = (c[d] + 1) % L
            if n // w[d] != c[d] // w[d]:
                out.add((o, d))
    return out


def _face_threads(tile):
    """The (offset, direction) ccl_hook gives its thread t of a tiled block."""
    out = set()
    for t in range(32 if tile == 2 else 128):
        if tile == 2:
            d = 0 if t < 16 else 1
            o = (t << 4) | 15 if d == 0 else (15 << 4) | (t - 16)
        elif t < 32:
            d, o = 0, ((t >> 3) << 6) | ((t & 7) << 3) | 7
        elif t < 64:
            d, o = 1, (((t >> 3) & 3) << 6) | (7 << 3) | (t & 7)
        else:
            d, o = 2, (3 << 6) | (((t >> 3) & 7) << 3) | (t & 7)
        out.add((o, d))
    return out


@pytest.mark.parametrize("tile,L", [(2, 16), (2, 32), (2, 64), (3, 8), (3, 16), (3, 64)])
def test_hook_face_threads_cover_the_leaving_bonds(tile, L):
    leaving = _leaving_bonds(tile, L)
    faces = _face_threads(tile)
    assert len(faces) == (32 if tile == 2 else 128)  # one thread each
    assert leaving <= faces
    # the face threads left over are bonds that wrap into the same tile (the
    # lattice is one tile wide in that direction); the kernel skips them
    widths = (16, 16) if tile == 2 else (8, 8, 4)
    assert all(widths[d] == L for _, d in faces - leaving)
