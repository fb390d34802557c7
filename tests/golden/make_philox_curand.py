"""Generate tests/golden/philox_curand.npz on a machine with a CUDA GPU.

The fixture pins the oracle's Philox4x32-10 (oracle/oracle.c) to an
independent implementation: cuRAND's Philox4_32_10, called on the device
through the engine's self-test entry point mqv_selftest_philox (a state
initialised with seed, subsequence = c2 | c3 << 32, offset = 4 * (c0 | c1 << 32)
yields the block of counter (c0, c1, c2, c3) under key (lo32 seed, hi32 seed)).
The CPU test then compares the oracle with these cuRAND words.

    python tests/golden/make_philox_curand.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# (seed, c1, c2, c3): zero, and counters of the engine's streams (c3 =
# stream << 24 | replica).  cuRAND reaches counter word c1 through the 64-bit
# offset 4 * (c0 | c1 << 32), so c1 must stay below 2^30.
CASES = [
    (0, 0, 0, 0),
    (0x123456789ABCDEF0, 7, 11, (1 << 24) | 5),
    (20240601, 3, 1, (5 << 24) | 0),
]
N = 64  # counters c0 = 0 .. N-1 per case


def main():
    from marqov_b200 import _lib

    lib = _lib.load()
    seeds, ctrs, words = [], [], []
    for seed, c1, c2, c3 in CASES:
        eng = np.zeros(4 * N, np.uint32)
        cur = np.zeros(4 * N, np.uint32)
        _lib.check(lib.mqv_selftest_philox(seed, c1, c2, c3, N, eng.ctypes.data, cur.ctypes.data))
        for i in range(N):
            seeds.append(seed)
            ctrs.append([i, c1, c2, c3])
            words.append(cur[4 * i:4 * i + 4])
    out = os.path.join(HERE, "philox_curand.npz")
    np.savez_compressed(out, seed=np.array(seeds, np.uint64), ctr=np.array(ctrs, np.uint32),
                        out=np.array(words, np.uint32))
    print("wrote", out, len(seeds), "blocks")


if __name__ == "__main__":
    main()
