"""Handles driven from several host threads at once, each on its own
non-blocking stream, must give the chains they give one after the other:
nothing a handle's kernels read may be uploaded outside its stream's order,
and the host-side launch caches are shared between threads."""
from concurrent.futures import ThreadPoolExecutor

import pytest

pytestmark = pytest.mark.gpu

SIZES = [32, 96, 384, 512, 64, 512, 256, 384, 48, 512, 128, 192]


def members(M):
    return [(M.RegularHypercubic(L, 2), M.Config(seed=700 + i, repid=i, resident=(i % 3 == 0)), M.Potts(3, -1.0),
             0.98 + 0.005 * i) for i, L in enumerate(SIZES)]


def run_one(M, lat, cfg, ham, beta):
    c = M.makeCore(lat, cfg, ham, beta)
    try:
        c.init()
        c.emcs(20, 1, 1, measure=False)
        obs, mc = c.emcs(15, 1, 1)
        return obs, mc, c.state
    finally:
        c.close()


def test_threaded_handles_equal_sequential():
    import marqov_b200 as M
    ms = members(M)
    seq = [run_one(M, *m) for m in ms]
    with ThreadPoolExecutor(8) as ex:
        par = list(ex.map(lambda m: run_one(M, *m), ms))
    for i, (a, b) in enumerate(zip(seq, par)):
        assert (a[0] == b[0]).all(), f"observables of member {i}"
        assert (a[1] == b[1]).all(), f"cluster sizes of member {i}"
        assert (a[2] == b[2]).all(), f"state of member {i}"
