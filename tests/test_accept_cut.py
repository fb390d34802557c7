"""The closed-form acceptance cut of the sweep kernels (host self test of the
engine library, no device needed) equals the oracle's bisection over the
reference rule update_accepted<pref>: for every word, accept iff
word >> 11 < cut."""
import ctypes as C

import numpy as np


def cuts(pref, dE, beta):
    from marqov_b200 import _lib as L
    dE = np.ascontiguousarray(dE, np.float64)
    beta = np.ascontiguousarray(beta, np.float64)
    out = np.zeros(dE.size, np.uint64)
    L.check(L.load().mqv_selftest_accept_cut(pref, dE.size, dE.ctypes.data, beta.ctypes.data, out.ctypes.data))
    return out


def test_closed_form_cut_equals_bisection(orc):
    rng = np.random.default_rng(5)
    dE = np.concatenate([rng.uniform(0, 1, 300), rng.uniform(0, 20, 300), 10.0 ** rng.uniform(-12, 3, 300),
                         [0.0, -1.0, 1e-300, 4.0, 8.0, 12.0, 700.0, 740.0, 800.0, 1e6, np.inf, np.nan]])
    beta = np.concatenate([rng.uniform(0, 3, 900), [0.44, 0.44, 0.44, 0.44, 0.44, 0.44, 1.0, 1.0, 1.0, 1.0, 1.0,
                                                    1.0]])
    for pref in (1, 2):
        got = cuts(pref, dE, beta)
        want = np.array([orc.threshold(pref, float(d), float(b)) for d, b in zip(dE, beta)], np.uint64)
        bad = np.nonzero(got != want)[0]
        assert bad.size == 0, [(dE[i], beta[i], int(got[i]), int(want[i])) for i in bad[:5]]


def test_cut_is_the_decision_boundary(orc):
    rng = np.random.default_rng(9)
    for _ in range(200):
        pref = int(rng.integers(1, 3))
        d, b = float(rng.uniform(0.01, 30)), float(rng.uniform(0.05, 2))
        c = int(cuts(pref, [d], [b])[0])
        if 0 < c < 2 ** 53:
            assert orc.update_accepted(pref, d, b, (c - 1) << 11)
            assert not orc.update_accepted(pref, d, b, c << 11)
            u = int(rng.integers(0, 2 ** 53))
            assert orc.update_accepted(pref, d, b, u << 11) == (u < c)
