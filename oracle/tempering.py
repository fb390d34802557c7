"""Replica exchange between simulations -- TEST INFRASTRUCTURE.

CPU restatement of the reference scheduler's exchange step, used by tests/
only, as the checker of the device exchanges (``mqv_batch_tempering``):

- ``mh_ratio``      calcMHratio (src/libmarqov/marqovscheduler.h:44-57): exp
                    of the action difference, 0 below log(DBL_MIN), DBL_MAX
                    above log(DBL_MAX);
- ``calcprob``      CXX11Scheduler::calcprob (marqovscheduler.h:445-465) with
                    action = beta * total energy (Core::calcAction,
                    src/libmarqov/core.h:1145-1151), the four actions summed
                    left to right as written there;
- ``accepted``      ``rng.real() < min(1, mhratio)`` (marqovscheduler.h:393),
                    real = (64-bit word >> 11) * 2^-53 (rngcache.h:204);
- ``uniform``       the word of the engine's TEMPER stream: Philox4x32-10
                    block (step, pair, 0, 7 << 24) under the key (seed low,
                    seed high), low 64 bits;
- ``run_int8``      a whole exchange run of int8 members on the oracle's own
                    EMCS (Wolff clusters, then sweeps, then a measurement),
                    exchanging states (exchange_statespace,
                    marqovscheduler.h:466-470) after every step.

``calcprob`` and ``mh_ratio`` are pinned against the reference's own
functions compiled in oracle/_ref (tests/test_tempering_oracle.py).
"""
from __future__ import annotations

import math
import sys

import numpy as np

LOG_DBL_MIN = math.log(sys.float_info.min)
LOG_DBL_MAX = math.log(sys.float_info.max)
TEMPER_STREAM = 7


def mh_ratio(en: float) -> float:
    if en > LOG_DBL_MIN:
        return sys.float_info.max if en > LOG_DBL_MAX else math.exp(en)
    return 0.0


def calcprob(beta_a: float, e_a: float, beta_b: float, e_b: float) -> float:
    aa = beta_a * e_a
    bb = beta_b * e_b
    ab = beta_a * e_b
    ba = beta_b * e_a
    return mh_ratio(aa - ab + bb - ba)


def uniform(orc, seed: int, step: int, pair: int) -> float:
    blk = orc.philox([step & 0xFFFFFFFF, pair, 0, TEMPER_STREAM << 24],
                     [seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF])
    word = int(blk[0]) | (int(blk[1]) << 32)
    return (word >> 11) * 2.0 ** -53


def accepted(ratio: float, u: float) -> bool:
    return u < min(1.0, ratio)


def run_int8(orc, members, plan, n_steps, emcs_per_step, ncluster, nmetro, seed, step0=0):
    """members: list of dicts {model, graph, state (int8, reference order),
    beta, seed, replica, sweep, cluster, n}; states and counters are advanced
    in place.  plan: int [n_steps, pairs, 2].  Returns (obs [n_emcs, members,
    4], flags [n_steps, pairs])."""
    nm = len(members)
    obs = np.zeros((n_steps * emcs_per_step, nm, 4))
    flags = np.zeros((n_steps, plan.shape[1]), np.int32)
    last_e = [0.0] * nm
    for t in range(n_steps):
        for k in range(emcs_per_step):
            for i, m in enumerate(members):
                for c in range(ncluster):
                    orc.wolff_int8(m["model"], m["graph"], m["state"], m["beta"], m["seed"], m["replica"],
                                   m["cluster"] + c)
                m["cluster"] += ncluster
                for j in range(nmetro):
                    orc.sweep_int8(m["model"], m["graph"], m["state"], m["beta"], m["seed"], m["replica"],
                                   m["sweep"] + j)
                m["sweep"] += nmetro
                o = orc.measure_int8(m["model"], m["graph"], m["state"])
                obs[t * emcs_per_step + k, i] = o
                last_e[i] = o[0]
        for p in range(plan.shape[1]):
            a, b = int(plan[t, p, 0]), int(plan[t, p, 1])
            if a == b:
                flags[t, p] = -1
                continue
            ma, mb = members[a], members[b]
            ea, eb = last_e[a] * ma["n"], last_e[b] * mb["n"]
            ok = accepted(calcprob(ma["beta"], ea, mb["beta"], eb), uniform(orc, seed, step0 + t, p))
            flags[t, p] = 1 if ok else 0
            if ok:
                ma["state"], mb["state"] = mb["state"], ma["state"]
                last_e[a], last_e[b] = last_e[b], last_e[a]
    return obs, flags
