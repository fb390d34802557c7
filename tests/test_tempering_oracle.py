"""Replica exchange, CPU side: the oracle's restatement of the reference
scheduler's exchange rule against the reference's own calcMHratio and
calcprob (compiled from its sources into oracle/_ref), the exchange plans,
and the 64-bit Mersenne twister behind the reference's plan."""
import math
import os
import sys

import numpy as np
import pytest

from oracle import tempering as T
from marqov_b200 import tempering as P


@pytest.fixture(scope="module")
def ref():
    from oracle.oracle import RefHarness, ref_path
    if not os.path.exists(ref_path()):
        pytest.skip("reference harness not built")
    return RefHarness()


def test_mt19937_64_known_answer(orc):
    """std::mt19937_64's required value: the 10000th output of a
    default-seeded engine is 9981545732273789042; and the oracle's words."""
    r = P.Mt19937_64()
    for _ in range(9999):
        r()
    assert r() == 9981545732273789042
    r = P.Mt19937_64(0)
    assert [r() for _ in range(64)] == [int(w) for w in orc.mt_words(0, 64)]


def test_mh_ratio_matches_reference(ref):
    lo, hi = math.log(sys.float_info.min), math.log(sys.float_info.max)
    vals = [-1e300, -800.0, lo - 1e-9, lo, lo + 1e-9, -700.0, -30.5, -1.0, -1e-12, 0.0, 1e-12, 0.5, 3.0,
            700.0, hi - 1e-9, hi, hi + 1e-9, 800.0, 1e300]
    vals += list(np.random.default_rng(3).uniform(-50, 50, 200))
    for en in vals:
        assert T.mh_ratio(en) == ref.calc_mh_ratio(en), en


def test_calcprob_matches_reference(ref):
    """Random (beta, total energy) pairs, integer-valued energies as the
    int8 models have and general doubles: bit-equal ratios."""
    rng = np.random.default_rng(11)
    n = 400
    ba = rng.uniform(0.05, 2.0, n)
    bb = rng.uniform(0.05, 2.0, n)
    ea = np.concatenate([rng.integers(-5000, 5000, n // 2).astype(float), rng.normal(0, 300, n - n // 2)])
    eb = np.concatenate([rng.integers(-5000, 5000, n // 2).astype(float), rng.normal(0, 300, n - n // 2)])
    got = ref.pt_calcprob(ba, ea, bb, eb)
    mine = np.array([T.calcprob(*x) for x in zip(ba, ea, bb, eb)])
    assert (got == mine).all()
    # an exchange towards the Boltzmann-favoured order is always accepted
    assert T.calcprob(1.0, -10.0, 0.5, -20.0) >= 1.0


def test_uniform_stream(orc):
    u = [T.uniform(orc, 99, t, p) for t in range(50) for p in range(4)]
    assert all(0.0 <= x < 1.0 for x in u)
    assert len(set(u)) == len(u)
    assert abs(np.mean(u) - 0.5) < 0.1


def test_neighbour_plan_alternates_and_is_disjoint():
    for n in (1, 2, 5, 8):
        plan = P.neighbour_plan(n, 6, first=1)
        assert plan.shape == (6, max(n // 2, 1), 2)
        for t in range(6):
            real = [tuple(p) for p in plan[t] if p[0] != p[1]]
            ids = [i for p in real for i in p]
            assert len(ids) == len(set(ids))
            assert all(b == a + 1 and a % 2 == (1 + t) % 2 for a, b in real)


def test_reference_plan_shifts_the_reference_steps():
    """Step t of the device plan holds the reference's pair t + 1 (pair 0 is
    never used: the first exchange follows the first game loop); the last
    step has none."""
    n, maxpt, seed = 5, 40, 17
    r = P.Mt19937_64(seed)
    ref = [(r() % n, r() % n) for _ in range(maxpt)]
    plan = P.reference_plan(n, maxpt, seed)
    assert plan.shape == (maxpt, 1, 2)
    assert [tuple(p) for p in plan[:-1, 0]] == ref[1:]
    assert plan[-1, 0, 0] == plan[-1, 0, 1]
