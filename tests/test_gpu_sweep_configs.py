"""Every candidate kernel of the fused 2D Ising sweep, forced one at a time
(MARQOV_B200_SWEEP_CONFIG), against the oracle: two sweeps with measurements
at sizes where the band kernels apply (L = 8192, 16384)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BETA = 0.44068679

CONFIGS = [
    ("ising2d_band<256,4,2>", 16384),
    ("ising2d_band<256,2,2>", 16384),
    ("ising2d_band<256,4,3>", 16384),
    ("ising2d_band<256,4,4>", 16384),
    ("ising2d_band<128,4,2>", 8192),
    ("ising2d_band<128,4,4>", 8192),
    ("ising2d_band<128,4,2,2>", 16384),
    ("ising2d_band<128,2,2,2>", 16384),
    ("ising2d_band<128,1,2,2>", 16384),
    ("ising2d_band<128,3,2,2>", 16384),
    ("ising2d_band<64,4,2,2>", 8192),
    ("ising2d_band_rs<128,1,2,5>", 16384),
    ("ising2d_band_rs<128,1,2,6>", 16384),
    ("ising2d_band_rs<128,2,2,5>", 16384),
    ("ising2d_band_rs<256,1,1,3>", 16384),
    ("ising2d_band_rs<256,1,1,4>", 16384),
    ("ising2d_band_rs<64,2,4,4>", 16384),
    ("ising2d_band_rs<64,2,4,6>", 16384),
    ("ising2d_band_rs<64,2,4,8>", 16384),
    ("ising2d_band_rs<64,1,4,6>", 16384),
    ("ising2d_band_rs<64,1,4,8>", 16384),
    ("ising2d_sweep<512,32,4>", 8192),
    ("ising2d_sweep<256,32,4>", 8192),
    ("ising2d_sweep<512,32,2>", 8192),
    ("ising2d_sweep<256,32,8>", 8192),
    ("ising2d_sweep<1024,32,2>", 8192),
    ("ising2d_sweep<128,32,4>", 8192),
    ("ising2d_sweep<64,32,4>", 8192),
]


def energy_per_site(s: np.ndarray, L: int) -> float:
    g = s.reshape(L, L).astype(np.int64)
    bonds = int((g * np.roll(g, 1, axis=0)).sum() + (g * np.roll(g, 1, axis=1)).sum())
    return -bonds / (L * L)  # J = -1 in the reference sign convention


@pytest.mark.parametrize("name,L", CONFIGS)
def test_forced_config_matches_oracle(orc, name, L, monkeypatch):
    import marqov_b200 as M
    monkeypatch.setenv("MARQOV_B200_SWEEP_CONFIG", name)
    cfg = M.Config(seed=4242, repid=3, ncluster=0, nmetro=1)
    with M.makeCore(M.RegularHypercubic(L, 2), cfg, M.Ising(-1.0), BETA) as c:
        c.init()
        s = c.state
        obs, _ = c.emcs(2, ncluster=0, nmetro=1)
        assert c.describe().endswith(name)
        g = c.state
    for sweep in range(2):
        orc.ising2d_sweep(L, -1.0, s, BETA, 4242, 3, sweep)
    assert (s == g).all()
    assert obs[-1, 1] == abs(float(s.astype(np.int64).sum())) / (L * L)
    assert abs(obs[-1, 0] - energy_per_site(s, L)) <= 1e-12
