"""Exchange plans for replica exchange between batch members.

The exchanges themselves run on the device (``Batch.tempering``); a plan
lists, per exchange step, the disjoint member pairs that attempt one.

- ``reference_plan`` is the reference scheduler's plan: ``maxpt`` random
  ordered pairs ``(x % len, y % len)`` from a 64-bit Mersenne twister
  (CXX11Scheduler::createPTplan / start, src/libmarqov/marqovscheduler.h:203-210,
  231-234), one pair per step, self pairs included and skipped.  Each member
  runs ``maxpt`` game loops and the pair of step t >= 1 exchanges after the
  t-th (ptstep is reached only with npt > 0, marqovscheduler.h:251-256), so
  step t of the device plan holds the reference's pair t + 1 and the last
  step none.
- ``neighbour_plan`` pairs members adjacent in the given order, even pairs
  (0,1), (2,3), ... on even steps and odd pairs (1,2), (3,4), ... on odd
  steps; with members ordered by beta this is the usual ladder.  It has no
  counterpart in the reference.
"""
import numpy as np

MASK64 = (1 << 64) - 1


class Mt19937_64:
    """The 64-bit Mersenne twister MT19937-64 (Matsumoto and Nishimura,
    published parameters; the engine std::mt19937_64 of C++11)."""

    N, M = 312, 156
    A = 0xB5026F5AA96619E9
    UPPER, LOWER = 0xFFFFFFFF80000000, 0x7FFFFFFF

    def __init__(self, seed: int = 5489):
        self.mt = [0] * self.N
        self.mt[0] = seed & MASK64
        for i in range(1, self.N):
            prev = self.mt[i - 1]
            self.mt[i] = (6364136223846793005 * (prev ^ (prev >> 62)) + i) & MASK64
        self.idx = self.N

    def _twist(self):
        mt = self.mt
        for i in range(self.N):
            x = (mt[i] & self.UPPER) | (mt[(i + 1) % self.N] & self.LOWER)
            xa = x >> 1
            if x & 1:
                xa ^= self.A
            mt[i] = mt[(i + self.M) % self.N] ^ xa
        self.idx = 0

    def __call__(self) -> int:
        if self.idx >= self.N:
            self._twist()
        y = self.mt[self.idx]
        self.idx += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & MASK64


def reference_plan(n_members: int, maxpt: int, seed: int = 0) -> np.ndarray:
    """The reference's plan as device steps: int32 [maxpt, 1, 2]."""
    if n_members < 1 or maxpt < 1:
        raise ValueError("need at least one member and one step")
    rng = Mt19937_64(seed)
    ref = []
    for _ in range(maxpt):
        a = rng() % n_members
        b = rng() % n_members
        ref.append((a, b))
    plan = np.zeros((maxpt, 1, 2), np.int32)
    for t in range(maxpt - 1):
        plan[t, 0] = ref[t + 1]
    return plan


def neighbour_plan(n_members: int, n_steps: int, first: int = 0) -> np.ndarray:
    """Alternating adjacent pairs: int32 [n_steps, n_members // 2, 2]; steps
    with fewer pairs are padded with self pairs (skipped)."""
    if n_members < 1 or n_steps < 0:
        raise ValueError("need at least one member")
    width = max(n_members // 2, 1)
    plan = np.zeros((n_steps, width, 2), np.int32)
    for t in range(n_steps):
        off = (first + t) & 1
        pairs = [(i, i + 1) for i in range(off, n_members - 1, 2)]
        for k in range(width):
            plan[t, k] = pairs[k] if k < len(pairs) else (0, 0)
    return plan
