"""The CPU oracle against the reference: golden vectors generated from the
reference's own templates (tests/golden/make_golden.py), the reference's
acceptance known-answer test, and the published Philox KAT."""
import hashlib
import os

import numpy as np
import pytest

from oracle import oracle as O

INT_CASES = ["ising2d_L16", "ising2d_L64", "ising3d_L8", "potts2d_L16", "bc2d_L16", "bcbip2d_L16", "ea3d_L8"]
F32_CASES = ["heis3d_L8_fresh", "heis3d_L8_cap", "phi4_3d_L8", "xxz3d_L8", "xxzsa3d_L8_bip"]
# float cases: per-sweep e and |m| within this relative tolerance of the reference
F32_RTOL = 1e-5


def model_of(g):
    kind = int(g["kind"])
    return O.OrcModel(kind=kind, q=int(g["q"]), J=float(g["J"]), h=float(g["D"]), h2=float(g.get("D2", 0.0)),
                      k=float(g["J"]), termsel=int(g.get("bipartite", 0)))


def f32_model_of(g):
    """The oracle model of a float fixture (ref_kind as in ref_harness.cpp)."""
    rk, beta = int(g["ref_kind"]), float(g["beta"])
    ts = int(g.get("bipartite", 0))
    if rk == 8:
        return O.OrcModel(kind=O.PHI4, J=-1.0, h=float(g["p1"]) / beta, h2=float(g["p0"]) / beta,
                          cap=float(g["cap"]), termsel=ts)
    if rk in (9, 10):
        return O.OrcModel(kind=O.XXZ, J=float(g["J"]), delta=float(g["p0"]), h=float(g["p1"]),
                          h2=float(g["p2"]) if rk == 10 else 0.0, termsel=ts)
    return O.OrcModel(kind=O.HEISENBERG, J=-1.0, proposal=1 if rk == 7 else 0, cap=float(g["cap"]))


def close(a, b, rtol=F32_RTOL, floor=1e-3):
    return abs(a - b) <= rtol * max(abs(b), floor)


def test_philox_matches_curand_fixture(orc, golden):
    """The oracle's Philox4x32-10 against cuRAND's Philox4_32_10 blocks."""
    g = golden("philox_curand")
    for seed, c, o in zip(g["seed"], g["ctr"], g["out"]):
        seed = int(seed)
        assert (orc.philox(c, [seed & 0xFFFFFFFF, seed >> 32]) == o).all()


def test_mt19937_64_words(orc, golden):
    g = golden("mt19937_64_words")
    assert (orc.mt_words(0, len(g["words"])) == g["words"]).all()


def test_metro_exp_kat(orc, golden):
    """testsuite/components/5-metro_exp.cpp: same accept decisions, one by one."""
    g = golden("metro_exp")
    acc, dec = orc.metro_exp(int(g["N"]), int(g["reps"]), float(g["beta"]), want_decisions=True)
    assert acc == int(g["accepted"])
    assert acc == int(g["accepted_plain"])  # the reference test's own criterion
    assert hashlib.sha256(np.packbits(dec).tobytes()).hexdigest() == str(g["sha256"])


@pytest.mark.parametrize("pref", [1, 2])
def test_acceptance_is_a_threshold_on_u53(orc, pref):
    rng = np.random.default_rng(pref)
    for _ in range(60):
        dE = float(rng.uniform(0.01, 30))
        beta = float(rng.uniform(0.05, 2.0))
        t = orc.threshold(pref, dE, beta)
        for u53 in [0, 1, max(t - 1, 0), t, min(t + 1, 2 ** 53 - 1), 2 ** 53 - 1] + \
                list(rng.integers(0, 2 ** 53, 20)):
            u53 = int(u53)
            w = (u53 << 11) | int(rng.integers(0, 2 ** 11))
            assert orc.update_accepted(pref, dE, beta, w) == (u53 < t)


def test_acceptance_edge_cases(orc):
    assert orc.update_accepted(1, 0.0, 1.0, 2 ** 64 - 1)
    assert orc.update_accepted(1, -5.0, 1.0, 2 ** 64 - 1)
    assert orc.threshold(1, -1.0, 0.5) == 2 ** 53
    # huge action: truncation saturates, every nonzero draw is rejected
    assert not orc.update_accepted(1, 1e300, 1e10, 1 << 40)
    assert orc.threshold(1, 1e300, 1e10) <= 1


@pytest.mark.parametrize("case", INT_CASES)
def test_int_case_bit_exact(orc, golden, case):
    """Initial state, final state and every per-sweep energy and |m| equal the
    reference's, bit for bit.  The energy is the one the reference's moves see
    (column 0); it equals the reference's Energy observable (column 2) except
    where that observable is a stub (Potts) or ignores bnds() (bond lattices)."""
    g = golden(case)
    dim, L = int(g["dim"]), int(g["L"])
    graph = orc.hypercubic(dim, L, g.get("bonds"))
    m = model_of(g)
    if "bonds" not in g:
        assert (orc.init_int8(m, graph.n, int(g["seed"]), int(g["replica"])) == g["init"]).all()
    s = g["init"].copy()
    for t in range(int(g["nsweeps"])):
        orc.sweep_int8(m, graph, s, float(g["beta"]), int(g["seed"]), int(g["replica"]), t)
        e, mm, _, _ = orc.measure_int8(m, graph, s)
        assert mm == g["obs"][t, 1]
        assert e == g["obs"][t, 0]
        if not (case.startswith("potts") or "bonds" in g):
            assert g["obs"][t, 0] == g["obs"][t, 2]
    assert (s == g["final"]).all()


def test_potts_and_bond_energies_differ_from_the_stub_observable(golden):
    """The reference's Energy<Potts<3>> reads 0 (PottsInteraction::energy is a
    stub) and Energy<Ising> on a bond lattice ignores the bonds; the fixtures
    keep both readings, and the parity energy is the one the moves see."""
    assert (golden("potts2d_L16")["obs"][:, 2] == 0).all()
    g = golden("ea3d_L8")
    assert (g["obs"][:, 0] != g["obs"][:, 2]).any()


@pytest.mark.parametrize("case", F32_CASES)
def test_f32_case_tolerance(orc, golden, case):
    """Float models: per-sweep energy and |m| within F32_RTOL of the
    reference's, final state within 1e-5."""
    g = golden(case)
    dim, L, symd = int(g["dim"]), int(g["L"]), int(g["symd"])
    graph = orc.hypercubic(dim, L)
    beta = float(g["beta"])
    m = f32_model_of(g)
    s = g["init"].copy()
    for t in range(int(g["nsweeps"])):
        orc.sweep_f32(m, graph, s, symd, beta, int(g["seed"]), 0, t)
        e, mm, _, _ = orc.measure_f32(m, graph, s, symd)
        assert close(mm, g["obs"][t, 1]), (t, mm, g["obs"][t, 1])
        assert close(e, g["obs"][t, 0]), (t, e, g["obs"][t, 0])
        assert close(e, g["obs"][t, 2]), (t, e, g["obs"][t, 2])
    assert np.allclose(s, g["final"], rtol=0, atol=1e-5)


def test_xxz_weights_delta_on_x_and_y(orc, golden):
    """The restatement must fail the XXZ fixture if Delta weights z instead."""
    g = golden("xxz3d_L8")
    graph = orc.hypercubic(3, 8)
    m = f32_model_of(g)
    s = g["init"].copy()
    orc.sweep_f32(m, graph, s, 3, float(g["beta"]), int(g["seed"]), 0, 0)
    e_x, _, _, _ = orc.measure_f32(m, graph, s, 3)
    assert close(e_x, g["obs"][0, 0])
    # the same energy function with the anisotropy moved onto z misses
    s3 = s.reshape(-1, 3)
    d = float(g["p0"])
    rp, ci = graph.row_ptr, graph.col_idx
    wrong = 0.0
    for i in range(graph.n):
        nb = s3[ci[rp[i]:rp[i + 1]]].sum(axis=0, dtype=np.float64)
        wrong += s3[i, 0] * nb[0] + s3[i, 1] * nb[1] + d * d * s3[i, 2] * nb[2]
    wrong = wrong / (2 * graph.n) + float(g["p1"]) * s3[:, 2].astype(np.float64).sum() / graph.n
    assert not close(wrong, g["obs"][0, 0])


def _batch_err(x, nb=20):
    b = np.array_split(np.asarray(x, float), nb)
    means = np.array([v.mean() for v in b])
    return means.std(ddof=1) / np.sqrt(nb)


@pytest.mark.parametrize("case,kind,q", [("wolff_ising_L16", O.ISING, 0), ("wolff_potts_L16", O.POTTS, 3)])
def test_wolff_restatement_statistics(orc, golden, case, kind, q):
    """Bond-keyed clusters have the reference clusters' size distribution."""
    g = golden(case)
    beta = float(g["beta"])
    graph = orc.hypercubic(2, 16)
    m = O.OrcModel(kind=kind, q=q, J=-1.0, k=-1.0)
    s = orc.init_int8(m, graph.n, 99, 0)
    for t in range(200):
        orc.sweep_int8(m, graph, s, beta, 99, 0, t)
    sizes = []
    for t in range(4000):
        sizes.append(orc.wolff_int8(m, graph, s, beta, 7, 0, t))
        orc.sweep_int8(m, graph, s, beta, 7, 0, 1000 + t)
    a, b = np.asarray(sizes, float), g["sizes"].astype(float)
    err = np.hypot(_batch_err(a), _batch_err(b))
    assert abs(a.mean() - b.mean()) < 4 * err, (a.mean(), b.mean(), err)


@pytest.mark.parametrize("case,kind,symd", [("wolff_heis_L8", O.HEISENBERG, 3), ("wolff_phi4_L8", O.PHI4, 1)])
def test_wolff_f32_restatement_statistics(orc, golden, case, kind, symd):
    """The bond-keyed float clusters (orc_wolff_f32: Embedder<Heisenberg> /
    scalar Embedder<Phi4>) against the reference's generic Wolff driven by
    those embedders with sequential draws: mean cluster size, <e> and <|m|>
    within 3 sigma (batch-means errors), same Metropolis in between."""
    g = golden(case)
    beta, p0, p1, amp = float(g["beta"]), float(g["p0"]), float(g["p1"]), float(g["amp"])
    graph = orc.hypercubic(3, 8)
    m = O.OrcModel(kind=kind, J=-1.0, h=p1 / beta, h2=p0 / beta, cap=amp)
    s = orc.init_f32(m, graph.n, symd, 77, 0)
    for t in range(200):
        orc.sweep_f32(m, graph, s, symd, beta, 77, 0, t)
    sizes, es, ms = [], [], []
    for t in range(len(g["sizes"])):
        sizes.append(orc.wolff_f32(m, graph, s, symd, beta, 5, 0, t))
        orc.sweep_f32(m, graph, s, symd, beta, 5, 0, 1000 + t)
        e, mm, _, _ = orc.measure_f32(m, graph, s, symd)
        es.append(e)
        ms.append(mm)
    for mine, theirs in ((sizes, g["sizes"]), (es, g["e"]), (ms, g["m"])):
        a, b = np.asarray(mine, float), np.asarray(theirs, float)
        err = np.hypot(_batch_err(a), _batch_err(b))
        assert abs(a.mean() - b.mean()) < 3 * err, (case, a.mean(), b.mean(), err)


def test_ref_harness_live_matches_oracle(orc):
    """Where the reference build is present, re-check a fresh case directly."""
    path = O.ref_path()
    if not os.path.exists(path):
        pytest.skip("reference build oracle/_ref not present")
    ref = O.RefHarness(path)
    graph = orc.hypercubic(2, 12)
    m = O.OrcModel(kind=O.ISING, J=-1.0)
    s = orc.init_int8(m, graph.n, 1234, 9)
    s2 = s.copy()
    for t in range(25):
        orc.sweep_int8(m, graph, s, 0.3, 1234, 9, 100 + t)
    ref.sweeps_int(1, graph, s2, -1.0, 0.0, 0.3, 1234, 9, 100, 25, want_obs=False)
    assert (s == s2).all()


@pytest.mark.parametrize("case", ["ref_emcs_potts2d_L16", "ref_emcs_heis3d_L8", "ref_emcs_phi4_3d_L8"])
def test_restatement_long_runs_match_reference(orc, golden, case):
    """The restatement's EMCS (colour order, keyed Philox, bond-keyed clusters)
    samples what the reference's own loop samples: <e>, <|m|>, chi, U4 and the
    mean cluster size within 2 sigma (tau_int-corrected) over 10^4 EMCS."""
    from oracle import stats as S
    g = golden(case)
    kind, dim, L, beta = int(g["kind"]), int(g["dim"]), int(g["L"]), float(g["beta"])
    graph = orc.hypercubic(dim, L)
    if kind == 3:
        m, symd = O.OrcModel(kind=O.POTTS, q=3, k=-1.0), 0
    elif kind == 6:
        m, symd = O.OrcModel(kind=O.HEISENBERG, J=-1.0), 3
    else:
        m, symd = O.OrcModel(kind=O.PHI4, J=-1.0, h=float(g["p1"]) / beta, h2=float(g["p0"]) / beta,
                             cap=float(g["p2"])), 1
    ncl, nmet, nth, nmeas = int(g["ncluster"]), int(g["nmetro"]), int(g["ntherm"]), int(g["nmeas"])
    s = orc.init_f32(m, graph.n, symd, 7, 0) if symd else orc.init_int8(m, graph.n, 7, 0)
    obs, mc = [], []
    sweep = cluster = 0
    for t in range(nth + nmeas):
        tot = 0
        for _ in range(ncl):
            tot += (orc.wolff_f32(m, graph, s, symd, beta, 7, 0, cluster) if symd
                    else orc.wolff_int8(m, graph, s, beta, 7, 0, cluster))
            cluster += 1
        for _ in range(nmet):
            if symd:
                orc.sweep_f32(m, graph, s, symd, beta, 7, 0, sweep)
            else:
                orc.sweep_int8(m, graph, s, beta, 7, 0, sweep)
            sweep += 1
        if t >= nth:
            obs.append(orc.measure_f32(m, graph, s, symd) if symd else orc.measure_int8(m, graph, s))
            mc.append(tot / ncl)
    obs = np.array(obs)
    mine = S.summary(obs[:, 0], obs[:, 1], graph.n, beta)
    for k in ("e", "m", "chi", "u4"):
        a, da = mine[k]
        b, db = g[k]
        assert abs(a - b) < 2 * np.hypot(da, db), (case, k, a, da, b, db)
    m1, s1 = S.mean_err(mc)
    m2, s2 = g["cluster"]
    assert abs(m1 - m2) < 2 * np.hypot(s1, s2), (case, m1, s1, m2, s2)
