"""Long-run statistics of the engine against exact results and against the
reference's own EMCS loop (random-site order, mt19937_64, its Wolff).

* 2D Ising L = 64 at beta_c, one Wolff cluster + one checkerboard sweep per
  EMCS, 10^4 measured EMCS after 10^3: <e> within 2 sigma of the exact
  finite-torus energy (Kaufman's partition function, oracle/exact2d.py), and
  <e>, <|m|>, chi = beta N (<m^2> - <|m|>^2), U4 and the mean cluster size
  each within 2 sigma of the reference's run (oracle/_ref).
* q = 3 Potts (2D L = 16, beta_c), Heisenberg (3D L = 8, beta = 0.693, five
  sweeps per cluster) and scalar phi^4 (3D L = 8): the same five quantities
  within 2 sigma of the reference's runs stored in tests/golden/ref_emcs_*.
Errors: the larger of batch means (50 batches; jackknife for chi and U4) and
the integrated-autocorrelation-time estimate (oracle/stats.py), combined in
quadrature between the two runs."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BETA_C = 0.44068679
KEYS = ("e", "m", "chi", "u4")


def zscores(a, b):
    return {k: abs(a[k][0] - b[k][0]) / np.hypot(a[k][1], b[k][1]) for k in KEYS}


def test_ising_matches_exact_energy_and_reference():
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
    eng = S.summary(obs[:, 0], obs[:, 1], N, BETA_C)
    exact = X.kaufman_energy(L, BETA_C)
    e, de = eng["e"]
    assert abs(e - exact) < 2 * de, f"<e> = {e} +- {de}, exact {exact}"
    if not os.path.exists(ref_path()):
        pytest.skip("reference harness not present")
    robs, rmc = RefHarness().emcs_ising2d(L, -1.0, BETA_C, 2024, 1, 1, 1000, 10000)
    ref = S.summary(robs[:, 0], robs[:, 1], N, BETA_C)
    z = zscores(eng, ref)
    assert all(v < 2 for v in z.values()), z
    m1, s1 = S.mean_err(mc)
    m2, s2 = S.mean_err(rmc)
    assert abs(m1 - m2) < 2 * np.hypot(s1, s2), (m1, s1, m2, s2)


@pytest.mark.parametrize("case", ["ref_emcs_potts2d_L16", "ref_emcs_heis3d_L8", "ref_emcs_phi4_3d_L8"])
def test_models_match_reference_long_runs(golden, case):
    import marqov_b200 as M
    from oracle import stats as S
    g = golden(case)
    kind, dim, L, beta = int(g["kind"]), int(g["dim"]), int(g["L"]), float(g["beta"])
    if kind == 3:
        ham = M.Potts(3, -1.0)
    elif kind == 6:
        ham = M.Heisenberg(-1.0, "fresh")
    else:
        ham = M.Phi4(beta, float(g["p0"]), float(g["p1"]), amp=float(g["p2"]))
    ncl, nmet = int(g["ncluster"]), int(g["nmetro"])
    cfg = M.Config(seed=7, repid=0, ncluster=ncl, nmetro=nmet)
    with M.makeCore(M.RegularHypercubic(L, dim), cfg, ham, beta) as c:
        c.init()
        c.emcs(int(g["ntherm"]), measure=False)
        obs, mc = c.emcs(int(g["nmeas"]))
    eng = S.summary(obs[:, 0], obs[:, 1], L ** dim, beta)
    ref = {k: tuple(g[k]) for k in KEYS}
    z = zscores(eng, ref)
    assert all(v < 2 for v in z.values()), (case, z)
    m1, s1 = S.mean_err(mc)
    m2, s2 = g["cluster"]
    assert abs(m1 - m2) < 2 * np.hypot(s1, s2), (case, m1, s1, m2, s2)
