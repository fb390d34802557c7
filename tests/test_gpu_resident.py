"""The resident path -- a small int8 lattice kept in one CTA's shared memory
for a whole chunk of EMCS, clusters by connected-component labelling -- must
give what the launch-per-step path gives (clusters grown breadth first, one
launch per colour and per measurement), bit for bit: states, cluster sizes,
energies and magnetisations."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def run(M, lat, ham, beta, seed, resident, n, ncluster, nmetro):
    cfg = M.Config(seed=seed, repid=3, ncluster=ncluster, nmetro=nmetro, resident=resident)
    with M.makeCore(lat, cfg, ham, beta) as c:
        c.init()
        obs, mc = c.emcs(n, ncluster=ncluster, nmetro=nmetro)
        return obs, mc, c.state, c.describe()


CASES = [
    ("ising2d_L16", lambda M: (M.RegularHypercubic(16, 2), M.Ising(-1.0), 0.44068679)),
    ("ising2d_L64", lambda M: (M.RegularHypercubic(64, 2), M.Ising(-1.0), 0.44068679)),
    ("ising2d_L96_embed", lambda M: (M.RegularHypercubic(96, 2), M.Ising(-1.0, "int8"), 0.44068679)),
    ("ising2d_L180", lambda M: (M.RegularHypercubic(180, 2), M.Ising(-1.0), 0.5)),
    ("ising2d_L256", lambda M: (M.RegularHypercubic(256, 2), M.Ising(-1.0), 0.44068679)),
    ("ising3d_L32", lambda M: (M.RegularHypercubic(32, 3), M.Ising(-1.0), 0.2216544)),
    ("ising3d_L40", lambda M: (M.RegularHypercubic(40, 3), M.Ising(-1.0), 0.2216544)),
    ("potts2d_L48", lambda M: (M.RegularHypercubic(48, 2), M.Potts(3, -1.0), 1.0050525)),
    ("potts3d_L8_q5", lambda M: (M.RegularHypercubic(8, 3), M.Potts(5, -1.0), 0.9)),
    ("potts2d_L256", lambda M: (M.RegularHypercubic(256, 2), M.Potts(3, -1.0), 1.0050525)),
    # thread-block clusters (distributed shared memory): 2 .. 8 CTAs
    ("ising2d_L384_cluster", lambda M: (M.RegularHypercubic(384, 2), M.Ising(-1.0), 0.44068679)),
    ("potts2d_L512_cluster", lambda M: (M.RegularHypercubic(512, 2), M.Potts(3, -1.0), 1.0050525)),
    ("ising3d_L48_cluster", lambda M: (M.RegularHypercubic(48, 3), M.Ising(-1.0, "int8"), 0.2216544)),
    ("ising2d_L320_cluster", lambda M: (M.RegularHypercubic(320, 2), M.Ising(-1.0), 0.5)),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("ncluster,nmetro", [(1, 1), (2, 3), (1, 0)])
def test_resident_equals_launch_path(name, make, ncluster, nmetro):
    import marqov_b200 as M
    lat, ham, beta = make(M)
    a = run(M, lat, ham, beta, 77, True, 25, ncluster, nmetro)
    b = run(M, lat, ham, beta, 77, False, 25, ncluster, nmetro)
    assert "resident" in a[3] and "resident" not in b[3], (a[3], b[3])
    assert (a[0] == b[0]).all(), "observables"
    assert (a[1] == b[1]).all(), "cluster sizes"
    assert (a[2] == b[2]).all(), "state"


@pytest.mark.parametrize("make", [lambda M: (M.RegularHypercubic(16, 2), M.BlumeCapel(-1.0, 0.5), 0.6),
                                  lambda M: (M.SimpleBipartite(16, 2), M.BlumeCapelBipartite(-1.0, 0.7, -0.4), 0.6),
                                  lambda M: (M.RegularRandomBond(8, 3, 0.5, seed=4), M.EdwardsAndersonIsing(-1.0), 0.9)])
def test_resident_metropolis_only_models(make):
    import marqov_b200 as M
    lat, ham, beta = make(M)
    a = run(M, lat, ham, beta, 5, True, 30, 0, 2)
    b = run(M, lat, ham, beta, 5, False, 30, 0, 2)
    assert (a[0] == b[0]).all() and (a[2] == b[2]).all()


def test_resident_wolff_only_equals_oracle(orc):
    """mqv_wolff on the resident path: the oracle's bond-keyed clusters."""
    import marqov_b200 as M
    L, beta, seed = 64, 0.44068679, 8
    cfg = M.Config(seed=seed, repid=0, ncluster=1, nmetro=0)
    with M.makeCore(M.RegularHypercubic(L, 2), cfg, M.Ising(-1.0), beta) as c:
        c.init()
        s = c.state.copy()
        sizes = c.wolff(200)
        final = c.state
    g = orc.hypercubic(2, L)
    m = O.OrcModel(kind=O.ISING, J=-1.0)
    ref = np.array([orc.wolff_int8(m, g, s, beta, seed, 0, k) for k in range(200)])
    assert (np.asarray(sizes) == ref).all()
    assert (final == s).all()


@pytest.mark.parametrize("make", [lambda M: (M.RegularHypercubic(1024, 2), M.Ising(-1.0), 0.44068679, 0),
                                  lambda M: (M.RegularHypercubic(256, 2), M.Potts(3, -1.0), 1.0050525, 0),
                                  lambda M: (M.RegularHypercubic(32, 3), M.Heisenberg(-1.0, "smallcap", 0.5), 0.693, 3),
                                  lambda M: (M.RegularHypercubic(32, 3), M.Phi4(0.37, 1.1, 1.0), 0.37, 1)])
def test_labelling_equals_breadth_first(make):
    """One large lattice on the launch-per-step path: clusters by
    whole-lattice labelling equal the breadth-first ones (the same draws),
    states and sizes bit for bit (float states: the same arithmetic, so equal
    too).  Float observables are sums of FP64 atomics, whose order differs
    between runs: they agree to rounding."""
    import marqov_b200 as M
    lat, ham, beta, symd = make(M)
    out = []
    for algo in ("label", "bfs"):
        cfg = M.Config(seed=12, repid=1, ncluster=1, nmetro=1, resident=False)
        with M.makeCore(lat, cfg, ham, beta) as c:
            c.set_wolff(algo)
            assert ("clusters=" + algo) in c.describe()
            c.init()
            obs, mc = c.emcs(12)
            sizes = c.wolff(5)
            out.append((obs, mc, sizes, c.state))
    assert (out[0][1] == out[1][1]).all() and (out[0][2] == out[1][2]).all()
    if symd == 0:
        assert (out[0][0] == out[1][0]).all()
    else:
        assert np.allclose(out[0][0], out[1][0], rtol=1e-12, atol=1e-12)
    assert (out[0][3] == out[1][3]).all()


def test_batch_resident_members_equal_launch_path():
    """A farm of resident members (both size classes) beside graph members
    (too large, or asked for the launch path) equals the members run one by
    one on the launch path, bit for bit, with and without replica exchange."""
    import marqov_b200 as M
    sizes = [32, 48, 64, 128, 192, 256, 384, 512, 96]
    # resident=True: nine members fill too few SMs for the default choice
    ms = [(M.RegularHypercubic(L, 2), M.Config(seed=40 + i, repid=i, resident=True), M.Potts(3, -1.0),
           1.0 + 0.01 * i) for i, L in enumerate(sizes)]
    solo = []
    try:
        for lat, cfg, ham, beta in ms:
            cfg1 = M.Config(seed=cfg.seed, repid=cfg.repid, resident=False, per_colour=True)
            c = M.makeCore(lat, cfg1, ham, beta)
            c.init()
            solo.append(c)
        with M.Batch(ms, graph_steps=4) as b:
            b.init()
            obs, mc = b.emcs(11, 1, 2)
            for i, c in enumerate(solo):
                o, m = c.emcs(11, 1, 2)
                assert (obs[:, i, :] == o).all(), f"member {i}"
                assert (mc[:, i] == m).all(), f"member {i}"
                assert (b.member(i).state == c.state).all(), f"member {i}"
    finally:
        for c in solo:
            c.close()
