"""The dump container (marqov_b200.checkpoint): the reference's step-group
layout as a directory tree, and a run continued from it equal to one that
never stopped."""
import json
import os

import numpy as np
import pytest

from marqov_b200 import checkpoint as CP
from marqov_b200.core import Config


def test_step_layout_roundtrip(tmp_path):
    import marqov_b200 as M
    cfg = Config(outpath=str(tmp_path) + "/", outname="run", seed=5, repid=2)
    path = CP.container_path(cfg)
    assert path.endswith("run.mqv") and not CP.dump_present(cfg) and CP.last_step(path) == -1
    st = CP.Step(path, 0).create(0.44, cfg, M.RegularHypercubic(8, 2), M.Ising(-1.0), "test")
    assert CP.last_step(path) == 0 and not st.complete
    s = np.arange(64, dtype=np.int8) % 2 * 2 - 1
    st.write_state(s, 5, 2, 40, 20)
    st.write_observables({"e": [-1.0, -1.5], "m": [0.1, 0.2]})
    assert st.complete and CP.dump_present(cfg)
    s2, rng, h = CP.Step(path, 0).read_state()
    assert (s2 == s).all() and s2.dtype == np.int8 and rng == (5, 2, 40, 20) and h is None
    assert list(CP.Step(path, 0).read_observables()) == ["e", "m"]
    mc = json.load(open(os.path.join(path, "step0", "config", "marqovconfig.json")))
    assert mc["beta"] == 0.44 and mc["seed"] == 5 and mc["repid"] == 2
    ham = json.load(open(os.path.join(path, "step0", "config", "hamiltonian.json")))
    assert ham["name"] == "Ising" and ham["J"] == -1.0
    os.makedirs(os.path.join(path, "step3"))
    assert CP.last_step(path) == 3


@pytest.mark.gpu
def test_continued_run_equals_uninterrupted(tmp_path):
    """Two Cores on one container (step0, then step1 continuing from it) give
    the observables and final state of one Core running both game loops."""
    import marqov_b200 as M
    kw = dict(seed=77, repid=3, warmupsteps=20, gameloopsteps=30, ncluster=1, nmetro=2)
    cfg = Config(outpath=str(tmp_path) + "/", outname="ising", **kw)
    lat, ham, beta = M.RegularHypercubic(32, 2), M.Ising(-1.0), 0.44
    with M.makeCore(lat, cfg, ham, beta) as c:
        c.init()
        c.wrmploop()
        c.gameloop()
    with M.makeCore(lat, cfg, ham, beta) as c:
        c.init()  # a continued step keeps the state it read
        c.gameloop()
    ref = M.makeCore(lat, Config(**kw), ham, beta)
    try:
        ref.init()
        ref.wrmploop()
        ref.gameloop()
        first = ref.obs.arrays()
        ref.obs = type(ref.obs)()
        ref.gameloop()
        second = ref.obs.arrays()
        path = CP.container_path(cfg)
        assert CP.last_step(path) == 1
        o0 = CP.Step(path, 0).read_observables()
        o1 = CP.Step(path, 1).read_observables()
        for k in ("e", "m", "m2", "m4", "clustersize"):
            assert (o0[k] == first[k]).all() and (o1[k] == second[k]).all(), k
        s1, rng, h = CP.Step(path, 1).read_state()
        assert (s1 == ref.state).all() and h is not None
        assert rng == (77, 3) + ref.counters
    finally:
        ref.close()


def test_truncated_state_is_refused(tmp_path):
    """A step whose state file was cut short is refused with CHECKSUM."""
    import marqov_b200 as M
    cfg = Config(outpath=str(tmp_path) + "/", outname="t", seed=1)
    path = CP.container_path(cfg)
    st = CP.Step(path, 0).create(0.4, cfg, M.RegularHypercubic(8, 2), M.Ising(-1.0), "test")
    st.write_state(np.ones(64, np.int8), 1, 0, 3, 0, hash_=123)
    f = os.path.join(st.path, "state", "hamiltonianstatespace.npy")
    data = open(f, "rb").read()
    open(f, "wb").write(data[: len(data) - 20])
    with pytest.raises(M.MarqovError) as ei:
        CP.Step(path, 0).read_state()
    assert ei.value.status == M._lib.ERR_CHECKSUM


@pytest.mark.gpu
def test_corrupt_state_is_refused(tmp_path):
    """A stored state whose bytes no longer match the stored hash: the next
    Core on the container fails with CHECKSUM and never runs on it; the
    handle-level call leaves the state untouched."""
    import marqov_b200 as M
    cfg = Config(outpath=str(tmp_path) + "/", outname="c", seed=3, warmupsteps=2, gameloopsteps=3, ncluster=0,
                 nmetro=1)
    lat, ham = M.RegularHypercubic(16, 2), M.Ising(-1.0)
    with M.makeCore(lat, cfg, ham, 0.4) as c:
        c.init()
        c.gameloop()
    path = CP.container_path(cfg)
    f = os.path.join(path, "step0", "state", "hamiltonianstatespace.npy")
    st = np.load(f)
    st[5] = -st[5]  # a flipped spin: still a legal state, wrong bytes
    np.save(f, st)
    with pytest.raises(M.MarqovError) as ei:
        M.makeCore(lat, cfg, ham, 0.4)
    assert ei.value.status == M._lib.ERR_CHECKSUM
    with M.makeCore(lat, Config(seed=9), ham, 0.4) as c:
        c.init()
        before, h = c.get_state_checked()
        with pytest.raises(M.MarqovError) as ei:
            c.set_state_checked(st, h)
        assert ei.value.status == M._lib.ERR_CHECKSUM
        assert (c.state == before).all()
        c.set_state_checked(before, h)
