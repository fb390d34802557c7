"""Long-run statistics of the engine: 2D Ising L = 64 at beta_c, one Wolff
cluster + one checkerboard sweep per EMCS, 10^4 measured EMCS after 10^3.

* <e> within 2 sigma of the exact finite-torus energy (Kaufman's partition
  function, oracle/exact2d.py);
* <e>, <|m|>, chi = beta N (<m^2> - <|m|>^2) and U4 against the reference's
  own EMCS loop (random-site order, mt19937_64; oracle/_ref): every one within
  3 sigma of the combined error and at least three of the four within 2 sigma.
Errors: batch means and jackknife over 50 batches of 200 EMCS."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BETA_C = 0.44068679


def test_engine_matches_exact_energy_and_reference():
    import marqov_b200 as M
    from oracle import exact2d as X
    from oracle import stats as S
    from oracle.oracle import RefHarness, ref_path
    L, N = 64, 64 * 64
    cfg = M.Config(seed=99, repid=0, ncluster=1, nmetro=1)
    with M.makeCore(M.RegularHypercubic(L, 2), cfg, M.Ising(-1.0), BETA_C) as c:
        c.init()
        c.emcs(1000, measure=False)
        obs, mc = c.emcs(10000)
    eng = S.ising_summary(obs[:, 0], obs[:, 1], N, BETA_C)
    exact = X.kaufman_energy(L, BETA_C)
    e, de = eng["e"]
    assert abs(e - exact) < 2 * de, f"<e> = {e} +- {de}, exact {exact}"
    if not os.path.exists(ref_path()):
        pytest.skip("reference harness not present")
    robs, rmc = RefHarness().emcs_ising2d(L, -1.0, BETA_C, 2024, 1, 1, 1000, 10000)
    ref = S.ising_summary(robs[:, 0], robs[:, 1], N, BETA_C)
    z = {k: abs(eng[k][0] - ref[k][0]) / np.hypot(eng[k][1], ref[k][1]) for k in ("e", "m", "chi", "u4")}
    assert all(v < 3 for v in z.values()) and sum(v < 2 for v in z.values()) >= 3, z
    # same cluster-size law: mean Wolff cluster within 3 sigma
    m1, s1 = S.mean_err(mc)
    m2, s2 = S.mean_err(rmc)
    assert abs(m1 - m2) < 3 * np.hypot(s1, s2), (m1, s1, m2, s2)
