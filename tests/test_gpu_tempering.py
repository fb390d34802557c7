"""Replica exchange between batch members (mqv_batch_tempering) against the
oracle's restatement of the reference scheduler's exchange step: the same
per-EMCS observables, exchange decisions and final states, bit for bit, for
int8 models; for float models the decisions follow the reported energies and
the states equal a plain batch whose states are swapped on the host."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import tempering as T

pytestmark = pytest.mark.gpu


def ladder(M, L, betas, ham, seed0=40):
    return [(M.RegularHypercubic(L, 2), M.Config(seed=seed0 + i, repid=i), ham, b) for i, b in enumerate(betas)]


def oracle_members(orc, b, ms, model, L):
    g = orc.hypercubic(2, L)
    out = []
    for i, (lat, cfg, ham, beta) in enumerate(ms):
        sw, cl = b.member(i).counters
        out.append(dict(model=model, graph=g, state=b.member(i).state.copy(), beta=float(beta), seed=cfg.seed,
                        replica=cfg.repid, sweep=sw, cluster=cl, n=L * L))
    return out


@pytest.mark.parametrize("graph_steps", [1, 8])
def test_ising_ladder_equals_oracle(orc, graph_steps):
    import marqov_b200 as M
    L, betas = 12, [0.35, 0.39, 0.43, 0.47, 0.51, 0.55]
    ms = ladder(M, L, betas, M.Ising(-1.0))
    with M.Batch(ms, graph_steps=graph_steps) as b:
        b.init()
        om = oracle_members(orc, b, ms, O.OrcModel(kind=O.ISING, J=-1.0), L)
        step0, flags_all = 0, []
        for call, (n_steps, k) in enumerate(((8, 2), (5, 3))):
            plan = M.tempering.neighbour_plan(len(ms), n_steps, first=step0)
            obs, acc = b.tempering(n_steps, emcs_per_step=k, ncluster=1, nmetro=1, plan=plan, seed=5)
            oobs, oacc = T.run_int8(orc, om, plan, n_steps, k, 1, 1, 5, step0)
            assert (acc == oacc).all(), f"call {call}: exchange decisions differ"
            assert (obs == oobs).all(), f"call {call}: observables differ"
            for i in range(len(ms)):
                assert (b.member(i).state == om[i]["state"]).all(), f"call {call} member {i}: state differs"
                assert b.member(i).counters == (om[i]["sweep"], om[i]["cluster"])
            step0 += n_steps
            flags_all.append(acc)
        f = np.concatenate([a.reshape(-1) for a in flags_all])
        assert (f == 1).any() and (f == 0).any(), "want both outcomes in the run"


def test_reference_plan_across_chunks(orc):
    """The reference's one-random-pair-per-step plan (self pairs included),
    100 EMCS per step so that exchanges straddle the measurement chunks."""
    import marqov_b200 as M
    L, betas = 8, [0.30, 0.40, 0.45, 0.60]
    ms = ladder(M, L, betas, M.Potts(3, -1.0), seed0=900)
    maxpt = 3
    plan = M.tempering.reference_plan(len(ms), maxpt, seed=123)
    with M.Batch(ms, graph_steps=8) as b:
        b.init()
        om = oracle_members(orc, b, ms, O.OrcModel(kind=O.POTTS, q=3, k=-1.0), L)
        obs, acc = b.tempering(maxpt, emcs_per_step=100, ncluster=1, nmetro=1, plan=plan, seed=77)
        oobs, oacc = T.run_int8(orc, om, plan, maxpt, 100, 1, 1, 77)
        assert (acc == oacc).all()
        assert acc[-1, 0] == -1
        assert (obs == oobs).all()
        for i in range(len(ms)):
            assert (b.member(i).state == om[i]["state"]).all()


def test_heisenberg_ladder_decisions_and_states(orc):
    import marqov_b200 as M
    L, betas, k, n_steps = 6, [0.60, 0.66, 0.72, 0.78], 2, 10
    ham = M.Heisenberg(-1.0, "smallcap", 0.4)
    ms = [(M.RegularHypercubic(L, 3), M.Config(seed=60 + i, repid=i), ham, b) for i, b in enumerate(betas)]
    n = L ** 3
    plan = M.tempering.neighbour_plan(len(ms), n_steps)
    with M.Batch(ms) as b, M.Batch(ms) as twin:
        b.init()
        twin.init()
        obs, acc = b.tempering(n_steps, emcs_per_step=k, ncluster=1, nmetro=1, plan=plan, seed=9)
        for t in range(n_steps):
            o, _ = twin.emcs(k, ncluster=1, nmetro=1)
            np.testing.assert_allclose(o, obs[t * k:(t + 1) * k], rtol=1e-9, atol=1e-12)
            last = obs[(t + 1) * k - 1, :, 0]
            for p, (a, c) in enumerate(plan[t]):
                if a == c:
                    assert acc[t, p] == -1
                    continue
                u = T.uniform(orc, 9, t, p)
                want = T.accepted(T.calcprob(betas[a], last[a] * n, betas[c], last[c] * n), u)
                assert acc[t, p] == int(want), f"step {t} pair {p}"
                if want:
                    sa, sc = twin.member(a).state, twin.member(c).state
                    twin.member(a).state = sc
                    twin.member(c).state = sa
        for i in range(len(ms)):
            assert (b.member(i).state == twin.member(i).state).all()
        assert (acc == 1).any()


def test_plan_rejections_leave_the_batch_untouched():
    import marqov_b200 as M
    L = 8
    ms = ladder(M, L, [0.4, 0.45, 0.5], M.Ising(-1.0))
    ms.append((M.RegularHypercubic(L, 2), M.Config(seed=7, repid=7), M.Ising(-0.5), 0.45))
    ms.append((M.RegularHypercubic(10, 2), M.Config(seed=8, repid=8), M.Ising(-1.0), 0.45))
    with M.Batch(ms) as b:
        b.init()
        before = [b.member(i).state.copy() for i in range(len(ms))]
        cnt = [b.member(i).counters for i in range(len(ms))]
        bad = {
            "shared member": [[[0, 1], [1, 2]]],
            "model differs": [[[0, 3], [1, 1]]],
            "lattice differs": [[[0, 4], [1, 1]]],
            "out of range": [[[0, 5], [1, 1]]],
        }
        for why, plan in bad.items():
            with pytest.raises(M.MarqovError):
                b.tempering(1, emcs_per_step=1, plan=np.array(plan, np.int32))
        for i in range(len(ms)):
            assert (b.member(i).state == before[i]).all()
            assert b.member(i).counters == cnt[i]
        # a plan of self pairs only is plain EMCS
        obs, acc = b.tempering(2, emcs_per_step=1, plan=np.zeros((2, 1, 2), np.int32))
        assert (acc == -1).all()
