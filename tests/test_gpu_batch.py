"""Batched EMCS (mqv_batch_*): a batch of members with uneven lattice sizes,
models and temperatures equals the same members run one handle at a time,
bit for bit -- states, per-EMCS observables and cluster sizes -- over
consecutive calls and for every number of EMCS per graph launch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TC_POTTS3 = 1.0 / np.log(1.0 + np.sqrt(3.0))


def members(M):
    out = []
    rng = np.random.default_rng(7)
    sizes = [16, 24, 32, 48, 10, 64]
    for i, L in enumerate(sizes):
        beta = 1.0 / (TC_POTTS3 * rng.uniform(0.9, 1.1))
        out.append((M.RegularHypercubic(L, 2), M.Config(seed=100 + i, repid=i), M.Potts(3, -1.0), beta))
    out.append((M.RegularHypercubic(64, 2), M.Config(seed=11, repid=40), M.Ising(-1.0), 0.44068679))
    out.append((M.RegularHypercubic(8, 3), M.Config(seed=12, repid=41), M.Ising(-1.0), 0.2216))
    out.append((M.RegularHypercubic(20, 2), M.Config(seed=13, repid=42), M.Ising(-1.0, "int8"), 0.42))
    return out


def solo(M, m):
    lat, cfg, ham, beta = m
    return M.makeCore(lat, cfg, ham, beta)


@pytest.mark.parametrize("graph_steps", [1, 3, 8])
def test_batch_equals_single_handles(graph_steps):
    import marqov_b200 as M
    ms = members(M)
    singles = [solo(M, m) for m in ms]
    try:
        with M.Batch(ms, graph_steps=graph_steps) as b:
            b.init()
            for c in singles:
                c.init()
            for i, c in enumerate(singles):
                assert (b.member(i).state == c.state).all()
            for call, n in enumerate((7, 5)):
                obs, mc = b.emcs(n, ncluster=1, nmetro=2)
                for i, c in enumerate(singles):
                    o, m = c.emcs(n, ncluster=1, nmetro=2)
                    assert (obs[:, i, :] == o).all(), f"call {call} member {i}: observables differ"
                    assert (mc[:, i] == m).all(), f"call {call} member {i}: cluster sizes differ"
                    assert (b.member(i).state == c.state).all(), f"call {call} member {i}: states differ"
                    assert b.member(i).counters == c.counters
            assert b.launches > 0
    finally:
        for c in singles:
            c.close()


def test_batch_blume_capel_metropolis_only():
    import marqov_b200 as M
    ms = [(M.RegularHypercubic(L, 2), M.Config(seed=5 + L, repid=L), M.BlumeCapel(-1.0, 0.5), 0.6)
          for L in (8, 12, 16)]
    singles = [solo(M, m) for m in ms]
    try:
        with M.Batch(ms) as b:
            b.init()
            for c in singles:
                c.init()
            obs, mc = b.emcs(6, ncluster=0, nmetro=3)
            assert (mc == 0).all()
            for i, c in enumerate(singles):
                o, _ = c.emcs(6, ncluster=0, nmetro=3)
                assert (obs[:, i, :] == o).all()
                assert (b.member(i).state == c.state).all()
    finally:
        for c in singles:
            c.close()


def test_batch_csr_members_equal_single_handles():
    """int8 members on CSR lattices (EA disorder realisations, a random
    geometric graph) beside hypercubic ones."""
    import marqov_b200 as M
    ms = [(M.RegularRandomBond(6, 3, 0.5, seed=s), M.Config(seed=300 + s, repid=s), M.EdwardsAndersonIsing(-1.0), 0.9)
          for s in range(3)]
    ms.append((M.RegularRandomBond(6, 3, 0.5, seed=7).to_csr(), M.Config(seed=307, repid=7),
               M.EdwardsAndersonIsing(-1.0), 0.9))
    ms.append((M.RandomGeometricGraph2D(500, 8.0, seed=4), M.Config(seed=9, repid=9), M.Ising(-1.0, "int8"), 0.5))
    ms.append((M.RegularHypercubic(16, 2), M.Config(seed=8, repid=8), M.Potts(3, -1.0), 1.0))
    singles = [solo(M, m) for m in ms]
    try:
        with M.Batch(ms, graph_steps=4) as b:
            b.init()
            for c in singles:
                c.init()
            obs, _ = b.emcs(9, ncluster=0, nmetro=2)
            for i, c in enumerate(singles):
                o, _ = c.emcs(9, ncluster=0, nmetro=2)
                assert (obs[:, i, :] == o).all(), f"member {i}"
                assert (b.member(i).state == c.state).all(), f"member {i}"
    finally:
        for c in singles:
            c.close()


def test_batch_float_members_equal_single_handles():
    """phi^4 at several couplings and small-cap Heisenberg, Metropolis + Wolff."""
    import marqov_b200 as M
    ms = [(M.RegularHypercubic(L, 3), M.Config(seed=70 + i, repid=i), M.Phi4(b, 1.1), b)
          for i, (L, b) in enumerate(((6, 0.36), (8, 0.37), (4, 0.38)))]
    ms.append((M.RegularHypercubic(8, 3), M.Config(seed=80, repid=7), M.Heisenberg(-1.0, "smallcap", 0.3), 0.693))
    singles = [solo(M, m) for m in ms]
    try:
        with M.Batch(ms, graph_steps=3) as b:
            b.init()
            for c in singles:
                c.init()
            for call in range(2):
                obs, mc = b.emcs(5, ncluster=1, nmetro=2)
                for i, c in enumerate(singles):
                    o, m = c.emcs(5, ncluster=1, nmetro=2)
                    np.testing.assert_allclose(obs[:, i, :], o, rtol=1e-5, atol=1e-7)
                    np.testing.assert_array_equal(mc[:, i], m)
                    np.testing.assert_allclose(b.member(i).state, c.state, rtol=1e-5, atol=1e-6)
    finally:
        for c in singles:
            c.close()


@pytest.mark.parametrize("kind", ["int8", "float"])
def test_batch_labelling_clusters_equal_single_handles(kind):
    """Clusters by connected-component labelling equal the breadth-first
    clusters of single handles (same bond draws), int8 and float members."""
    import marqov_b200 as M
    if kind == "int8":
        ms = [(M.RegularHypercubic(L, 2), M.Config(seed=40 + i, repid=i), M.Potts(3, -1.0), b)
              for i, (L, b) in enumerate(((16, 1.0), (24, 1.1), (256, 1.005)))]
        ms.append((M.RegularHypercubic(32, 2), M.Config(seed=50, repid=50), M.Ising(-1.0), 0.44068679))
        ms.append((M.RegularRandomBond(6, 3, 0.5, seed=2), M.Config(seed=51, repid=51), M.Ising(-1.0, "int8"), 0.3))
    else:
        ms = [(M.RegularHypercubic(L, 3), M.Config(seed=60 + i, repid=i), M.Phi4(b, 1.1), b)
              for i, (L, b) in enumerate(((6, 0.36), (8, 0.38)))]
        ms.append((M.RegularHypercubic(8, 3), M.Config(seed=70, repid=9), M.Heisenberg(-1.0), 0.693))
    singles = [solo(M, m) for m in ms]
    try:
        with M.Batch(ms, graph_steps=2) as b:
            b.set_wolff("label")
            b.init()
            for c in singles:
                c.init()
            for call in range(2):
                obs, mc = b.emcs(4, ncluster=2, nmetro=1)
                for i, c in enumerate(singles):
                    o, m = c.emcs(4, ncluster=2, nmetro=1)
                    np.testing.assert_array_equal(mc[:, i], m, err_msg=f"call {call} member {i}: cluster sizes")
                    if kind == "int8":
                        assert (obs[:, i, :] == o).all() and (b.member(i).state == c.state).all()
                    else:
                        np.testing.assert_allclose(obs[:, i, :], o, rtol=1e-5, atol=1e-7)
                        np.testing.assert_allclose(b.member(i).state, c.state, rtol=1e-5, atol=1e-6)
    finally:
        for c in singles:
            c.close()


def test_batch_labelling_equals_bfs_on_a_potts_farm():
    """The 256-member Potts farm (L up to 512, near Tc): both cluster
    algorithms give the same clusters, observables and states."""
    import marqov_b200 as M
    sizes = [32, 48, 64, 96, 128, 192, 256, 384, 512]
    rng = np.random.default_rng(3)
    tc = 1.0 / np.log(1.0 + np.sqrt(3.0))
    ms = []
    for i in range(256):
        L = int(rng.choice(sizes))
        ms.append((M.RegularHypercubic(L, 2), M.Config(seed=9000 + i, repid=i), M.Potts(3, -1.0),
                   1.0 / (tc * float(rng.uniform(0.9, 1.1)))))
    out = {}
    for alg in ("bfs", "label", "auto"):
        with M.Batch(ms) as b:
            b.set_wolff(alg)
            b.init()
            o1, m1 = b.emcs(12, 1, 1)
            o2, m2 = b.emcs(8, 2, 0)
            out[alg] = (m1, m2, o1, o2, [b.member(i).state for i in range(len(ms))])
            # auto: timed both on the first call, then kept one of them
            assert b.wolff == (alg if alg != "auto" else b.wolff) and b.wolff in ("bfs", "label")
    for alg in ("label", "auto"):
        for k in range(4):
            np.testing.assert_array_equal(out["bfs"][k], out[alg][k])
        assert all((x == y).all() for x, y in zip(out["bfs"][4], out[alg][4]))


def test_batch_samples_match_member_samples():
    import ctypes as C
    import torch
    import marqov_b200 as M
    ms = [(M.RegularHypercubic(4, 3), M.Config(seed=5, repid=i), M.Phi4(b, 1.1), b) for i, b in enumerate((0.36, 0.38))]
    singles = [solo(M, m) for m in ms]
    try:
        with M.Batch(ms) as b:
            b.init()
            for c in singles:
                c.init()
            d = torch.zeros((2, 7, 4), dtype=torch.float64, device="cuda")
            M._lib.check(M._lib.load().mqv_batch_emcs_samples(b._h, 7, 1, 1, C.c_void_p(d.data_ptr())))
            for i, c in enumerate(singles):
                ds = torch.zeros((7, 4), dtype=torch.float64, device="cuda")
                M._lib.check(M._lib.load().mqv_emcs_samples(c.handle, 7, 1, 1, C.c_void_p(ds.data_ptr())))
                c.synchronize()
                np.testing.assert_allclose(d[i].cpu().numpy(), ds.cpu().numpy(), rtol=1e-9)
    finally:
        for c in singles:
            c.close()


def test_batch_rejects_mixed_or_unsupported_members():
    import marqov_b200 as M
    with pytest.raises(M.MarqovError) as ei:
        M.Batch([(M.RegularHypercubic(8, 3), M.Config(), M.Heisenberg(-1.0), 0.7),
                 (M.RegularHypercubic(8, 2), M.Config(), M.Ising(-1.0), 0.4)])
    assert ei.value.status == M._lib.ERR_UNSUPPORTED_TERM
    with M.Batch([(M.RegularHypercubic(8, 3), M.Config(), M.XXZAntiferro(1.0, 0.5), 0.7)]) as b:
        b.init()
        with pytest.raises(M.MarqovError) as ei:
            b.emcs(1, ncluster=1, nmetro=1)
        assert ei.value.status == M._lib.ERR_UNSUPPORTED_TERM
        obs, _ = b.emcs(2, ncluster=0, nmetro=1)
        assert np.isfinite(obs).all()
