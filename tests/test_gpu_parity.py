"""Engine parity on the GPU, through the C ABI.

Integer models must be bit-exact with the reference (golden fixtures) and the
oracle: final configuration and every per-sweep energy and |m|.  Float models
agree within 1e-5 relative per sweep over short runs.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

INT_CASES = ["ising2d_L16", "ising2d_L64", "ising3d_L8", "potts2d_L16", "bc2d_L16", "bcbip2d_L16", "ea3d_L8"]
F32_CASES = ["heis3d_L8_fresh", "heis3d_L8_cap", "phi4_3d_L8", "xxz3d_L8", "xxzsa3d_L8_bip"]
# float models: per-sweep energy and |m| within this relative tolerance of the reference
F32_RTOL = 1e-5


def mb():
    import marqov_b200 as M
    return M


def ham_of(g):
    M = mb()
    kind = int(g["kind"])
    if kind == O.ISING:
        return M.Ising(float(g["J"]))
    if kind == O.POTTS:
        return M.Potts(int(g["q"]), float(g["J"]))
    if kind == O.BLUME_CAPEL and int(g.get("bipartite", 0)):
        return M.BlumeCapelBipartite(float(g["J"]), float(g["D"]), float(g["D2"]))
    if kind == O.BLUME_CAPEL:
        return M.BlumeCapel(float(g["J"]), float(g["D"]))
    if kind == O.EA:
        return M.EdwardsAndersonIsing(float(g["J"]))
    raise ValueError(kind)


def lattice_of(g, stencil_bonds=False):
    M = mb()
    dim, L = int(g["dim"]), int(g["L"])
    if "bonds" in g:
        if stencil_bonds:
            return M.BondedHypercubic(L, dim, g["bonds"])
        base = M.RegularHypercubic(L, dim).to_csr()
        return M.CSRLattice(base.row_ptr, base.col_idx, g["bonds"], base.colours)
    if int(g.get("bipartite", 0)):
        return M.SimpleBipartite(L, dim)
    return M.RegularHypercubic(L, dim)


def core_for(lat, ham, beta, seed, replica=0, per_colour=False):
    M = mb()
    cfg = M.Config(seed=int(seed), repid=int(replica), ncluster=0, nmetro=1, per_colour=per_colour)
    return M.makeCore(lat, cfg, ham, float(beta))


@pytest.mark.parametrize("case", INT_CASES)
def test_int_golden_bit_exact(golden, case):
    """Initial state (the reference's init rule), final state and every
    per-sweep energy and |m| equal the reference's, bit for bit."""
    g = golden(case)
    with core_for(lattice_of(g), ham_of(g), g["beta"], g["seed"], g["replica"]) as c:
        if "bonds" not in g:
            c.init()
            assert (c.state == g["init"]).all(), "initstatespace rule"
        c.state = g["init"]
        obs, _ = c.emcs(int(g["nsweeps"]), ncluster=0, nmetro=1)
        assert (obs[:, 1] == g["obs"][:, 1]).all()
        assert (obs[:, 0] == g["obs"][:, 0]).all()
        assert (c.state == g["final"]).all()
        assert c.launches > 0


def test_ea_golden_on_the_stencil_path(golden):
    """The EA fixture's bonds on the hypercubic stencil (one plane of +d bonds
    per dimension) give the reference's states and energies, bit for bit."""
    g = golden("ea3d_L8")
    with core_for(lattice_of(g, stencil_bonds=True), ham_of(g), g["beta"], g["seed"], g["replica"]) as c:
        assert "hypercubic" in c.describe()
        c.state = g["init"]
        obs, _ = c.emcs(int(g["nsweeps"]), ncluster=0, nmetro=1)
        assert (obs[:, 0] == g["obs"][:, 0]).all() and (obs[:, 1] == g["obs"][:, 1]).all()
        assert (c.state == g["final"]).all()


def f32_ham_of(g):
    M = mb()
    rk, beta = int(g["ref_kind"]), float(g["beta"])
    if rk == 8:
        return M.Phi4(beta, float(g["p0"]), float(g["p1"]), amp=float(g["cap"]))
    if rk == 9:
        return M.XXZAntiferro(float(g["p0"]), float(g["p1"]))
    if rk == 10:
        return M.XXZAntiferroSingleAniso(float(g["p1"]), float(g["p0"]), float(g["p2"]))
    return M.Heisenberg(-1.0, proposal="smallcap" if rk == 7 else "fresh", cap=float(g["cap"]))


def rel_close(a, b, rtol=F32_RTOL, floor=1e-3):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return (np.abs(a - b) <= rtol * np.maximum(np.abs(b), floor)).all()


@pytest.mark.parametrize("case", F32_CASES)
def test_f32_golden_tolerance(golden, case):
    """Float models against the reference: per-sweep energy and |m| within
    F32_RTOL relative, final state within 1e-5."""
    g = golden(case)
    beta = float(g["beta"])
    with core_for(lattice_of(g), f32_ham_of(g), beta, g["seed"]) as c:
        c.init()
        assert np.allclose(c.state, g["init"], rtol=0, atol=1e-6)
        c.state = g["init"]
        obs, _ = c.emcs(int(g["nsweeps"]), ncluster=0, nmetro=1)
        assert rel_close(obs[:, 1], g["obs"][:, 1])
        assert rel_close(obs[:, 0], g["obs"][:, 0])
        assert np.allclose(c.state, g["final"], rtol=0, atol=1e-5)


def test_philox_matches_oracle_and_curand(orc):
    M = mb()
    import ctypes as C
    lib = M._lib.load()
    n = 4096
    for seed, c1, c2, c3 in ((0, 0, 0, 0), (0x123456789ABCDEF0, 7, 11, (1 << 24) | 5), (42, 3, 0, 0)):
        eng = np.zeros(4 * n, np.uint32)
        cur = np.zeros(4 * n, np.uint32)
        M._lib.check(lib.mqv_selftest_philox(seed, c1, c2, c3, n, eng.ctypes.data, cur.ctypes.data))
        eng = eng.reshape(n, 4)
        key = [seed & 0xffffffff, seed >> 32]
        for i in (0, 1, 17, n - 1):
            assert (eng[i] == orc.philox([i, c1, c2, c3], key)).all()
        assert (eng == cur.reshape(n, 4)).all(), "engine Philox differs from cuRAND Philox4_32_10"


@pytest.mark.parametrize("L", [16, 32, 48, 64, 96, 320, 512])
@pytest.mark.parametrize("spintype", ["int", "int8"])
def test_fused_tiles_equal_per_colour_and_oracle(orc, L, spintype):
    M = mb()
    beta, seed = 0.44068679, 5 + L
    res = []
    for per_colour in (False, True):
        with core_for(M.RegularHypercubic(L, 2), M.Ising(-1.0, spintype), beta, seed, 3, per_colour) as c:
            c.init()
            obs, _ = c.emcs(12, ncluster=0, nmetro=1)
            res.append((c.state, obs))
    assert (res[0][0] == res[1][0]).all() and (res[0][1] == res[1][1]).all()
    g = orc.hypercubic(2, L)
    m = O.OrcModel(kind=O.ISING, J=-1.0)
    s = orc.init_int8(m, g.n, seed, 3)
    for t in range(12):
        orc.sweep_int8(m, g, s, beta, seed, 3, t)
        e, mm, _, _ = orc.measure_int8(m, g, s)
        assert res[0][1][t, 0] == e and res[0][1][t, 1] == mm
    assert (s == res[0][0]).all()


def test_csr_path_equals_stencil_path():
    M = mb()
    lat = M.RegularHypercubic(8, 3)
    out = []
    for l in (lat, lat.to_csr()):
        with core_for(l, M.Potts(3, -1.0), 1.0, 77) as c:
            c.init()
            c.emcs(10, ncluster=0, nmetro=1)
            out.append(c.state)
    assert (out[0] == out[1]).all()


def run_oracle_emcs(orc, m, g, s, beta, seed, replica, nsteps, ncluster, nmetro, symd=0):
    sizes, obs = [], []
    sweep = cluster = 0
    for _ in range(nsteps):
        for _ in range(ncluster):
            if symd:
                sizes.append(orc.wolff_f32(m, g, s, symd, beta, seed, replica, cluster))
            else:
                sizes.append(orc.wolff_int8(m, g, s, beta, seed, replica, cluster))
            cluster += 1
        for _ in range(nmetro):
            if symd:
                orc.sweep_f32(m, g, s, symd, beta, seed, replica, sweep)
            else:
                orc.sweep_int8(m, g, s, beta, seed, replica, sweep)
            sweep += 1
        obs.append(orc.measure_f32(m, g, s, symd) if symd else orc.measure_int8(m, g, s))
    return np.array(sizes), np.array(obs)


@pytest.mark.parametrize("name,L,beta", [("ising", 16, 0.44068679), ("ising", 64, 0.44068679),
                                         ("ising8", 32, 0.5), ("potts", 32, 1.0050525)])
def test_wolff_emcs_bit_exact(orc, name, L, beta):
    """EMCS = 1 Wolff cluster + 1 sweep (config 1 shape), engine vs oracle."""
    M = mb()
    seed, replica, nsteps = 31337, 2, 60
    if name == "potts":
        ham, m = M.Potts(3, -1.0), O.OrcModel(kind=O.POTTS, q=3, k=-1.0)
    elif name == "ising8":
        ham, m = M.Ising(-1.0, "int8"), O.OrcModel(kind=O.ISING_EMBED, J=-1.0)
    else:
        ham, m = M.Ising(-1.0), O.OrcModel(kind=O.ISING, J=-1.0)
    lat = M.RegularHypercubic(L, 2)
    cfg = M.Config(seed=seed, repid=replica, ncluster=1, nmetro=1)
    with M.makeCore(lat, cfg, ham, beta) as c:
        c.init()
        s0 = c.state
        obs, mc = c.emcs(nsteps)
        final = c.state
    g = orc.hypercubic(2, L)
    s = s0.copy()
    sizes, oobs = run_oracle_emcs(orc, m, g, s, beta, seed, replica, nsteps, 1, 1)
    assert (mc == sizes).all()
    assert (obs[:, 1] == oobs[:, 1]).all()
    assert (obs[:, 0] == oobs[:, 0]).all()
    assert (final == s).all()
    assert sizes.max() > 1


def test_config1_eleven_thousand_emcs_bit_exact(orc):
    """The parity configuration over its whole run: 2D Ising L = 64 at beta_c,
    EMCS = one Wolff cluster + one checkerboard sweep, 10^3 thermalisation +
    10^4 measured EMCS from the reference's initial-state rule -- every
    cluster size, every per-EMCS energy and |m|, and the final state equal
    the oracle's, bit for bit."""
    M = mb()
    L, beta, seed, replica, nsteps = 64, 0.44068679, 2024, 5, 11000
    cfg = M.Config(seed=seed, repid=replica, ncluster=1, nmetro=1)
    with M.makeCore(M.RegularHypercubic(L, 2), cfg, M.Ising(-1.0), beta) as c:
        c.init()
        s0 = c.state
        obs, mc = c.emcs(nsteps)
        final = c.state
    g = orc.hypercubic(2, L)
    m = O.OrcModel(kind=O.ISING, J=-1.0)
    assert (orc.init_int8(m, g.n, seed, replica) == s0).all()
    s = s0.copy()
    sizes, oobs = run_oracle_emcs(orc, m, g, s, beta, seed, replica, nsteps, 1, 1)
    assert (mc == sizes).all()
    assert (obs[:, 0] == oobs[:, 0]).all() and (obs[:, 1] == oobs[:, 1]).all()
    assert (final == s).all()


@pytest.mark.parametrize("model", ["heisenberg", "phi4"])
def test_wolff_f32_vs_oracle(orc, model):
    M = mb()
    seed, nsteps = 4242, 8
    if model == "heisenberg":
        L, beta, symd = 8, 0.6930, 3
        ham = M.Heisenberg(-1.0, "smallcap", cap=0.5)
        m = O.OrcModel(kind=O.HEISENBERG, J=-1.0, proposal=1, cap=0.5)
    else:
        L, beta, symd = 8, 0.37, 1
        ham = M.Phi4(beta, 1.1, 1.0, amp=0.5)
        m = O.OrcModel(kind=O.PHI4, J=-1.0, h=1.0 / beta, h2=1.1 / beta, cap=0.5)
    cfg = M.Config(seed=seed, ncluster=1, nmetro=2)
    with M.makeCore(M.RegularHypercubic(L, 3), cfg, ham, beta) as c:
        c.init()
        s0 = c.state
        obs, mc = c.emcs(nsteps)
        final = c.state
    g = orc.hypercubic(3, L)
    s = s0.copy()
    sizes, oobs = run_oracle_emcs(orc, m, g, s, beta, seed, 0, nsteps, 1, 2, symd=symd)
    assert (mc == sizes).all()
    assert np.allclose(obs[:, 0], oobs[:, 0], rtol=1e-5, atol=1e-6)
    assert np.allclose(obs[:, 1], oobs[:, 1], rtol=1e-5, atol=1e-6)
    assert np.allclose(final, s, rtol=0, atol=1e-5)


def test_csr_ea_and_rgg_vs_oracle(orc):
    """General graphs: greedy-coloured CSR sweeps (config 5 shapes, small)."""
    M = mb()
    rgg = M.RandomGeometricGraph2D(4096, 8.0, seed=3)
    col = rgg.greedy_colours()
    ncol = int(col.max()) + 1
    order = np.concatenate([np.flatnonzero(col == c) for c in range(ncol)]).astype(np.int32)
    cptr = np.concatenate([[0], np.cumsum([np.sum(col == c) for c in range(ncol)])]).astype(np.int32)
    g = O.Graph(rgg.row_ptr, rgg.col_idx, cptr, order)
    m = O.OrcModel(kind=O.ISING, J=-1.0)
    with core_for(rgg, M.Ising(-1.0), 0.5, 9) as c:
        c.init()
        s = c.state.copy()
        obs, _ = c.emcs(20, ncluster=0, nmetro=1)
        final = c.state
    for t in range(20):
        orc.sweep_int8(m, g, s, 0.5, 9, 0, t)
        e, mm, _, _ = orc.measure_int8(m, g, s)
        assert obs[t, 0] == e and obs[t, 1] == mm
    assert (final == s).all()


def test_checkpoint_resume_bit_exact():
    M = mb()
    lat = M.RegularHypercubic(32, 2)
    cfg = M.Config(seed=5, ncluster=1, nmetro=2)
    with M.makeCore(lat, cfg, M.Ising(-1.0), 0.44) as a:
        a.init()
        a.emcs(20, measure=False)
        ref = a.state
    with M.makeCore(lat, cfg, M.Ising(-1.0), 0.44) as b:
        b.init()
        b.emcs(8, measure=False)
        st, ctr = b.state, b.counters
    with M.makeCore(lat, cfg, M.Ising(-1.0), 0.44) as c:
        c.state = st
        c.counters = ctr
        c.emcs(12, measure=False)
        assert (c.state == ref).all()


def test_error_statuses():
    M = mb()
    E = M.MarqovError
    with pytest.raises(E) as ei:
        core_for(M.RegularHypercubic(15, 2), M.Ising(-1.0), 0.4, 1)
    assert ei.value.status == M._lib.ERR_BAD_DESCRIPTOR
    with pytest.raises(E) as ei:
        core_for(M.RegularHypercubic(16, 2), M.Potts(200, -1.0), 0.4, 1)
    assert ei.value.status == M._lib.ERR_UNSUPPORTED_TERM
    with core_for(M.RegularHypercubic(16, 2), M.Ising(-1.0), 0.4, 1) as c:
        with pytest.raises(E) as ei:
            c.metropolis(1)
        assert ei.value.status == M._lib.ERR_STATE
        with pytest.raises(E) as ei:
            c.state = np.zeros(256, np.int8)
        assert ei.value.status == M._lib.ERR_INVALID_ARG
    bad = M.CSRLattice(np.array([0, 1, 1], np.int32), np.array([1], np.int32))
    with pytest.raises(E) as ei:
        core_for(bad, M.Ising(-1.0), 0.4, 1)
    assert ei.value.status == M._lib.ERR_BAD_DESCRIPTOR
    with core_for(M.RegularHypercubic(16, 2), M.BlumeCapel(-1.0, 0.5), 0.4, 1) as c:
        c.init()
        with pytest.raises(E) as ei:
            c.wolff(1)
        assert ei.value.status == M._lib.ERR_UNSUPPORTED_TERM


@pytest.mark.parametrize("L", [64, 192])
def test_set_state_rejects_illegal_spins_and_keeps_the_state(L):
    """The fused 2D path checks uploaded spins on the device; an illegal value
    is refused and the current state is kept."""
    M = mb()
    with M.makeCore(M.RegularHypercubic(L, 2), M.Config(seed=3), M.Ising(-1.0), 0.4) as c:
        c.init()
        before = c.state
        bad = before.copy()
        bad[L * L - 5] = 0
        with pytest.raises(M.MarqovError) as ei:
            c.state = bad
        assert ei.value.status == M._lib.ERR_INVALID_ARG
        assert (c.state == before).all()
        good = np.where(np.random.default_rng(L).random(L * L) < 0.5, 1, -1).astype(np.int8)
        c.state = good
        assert (c.state == good).all()
