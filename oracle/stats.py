"""Error bars of correlated Monte Carlo series -- TEST INFRASTRUCTURE.

Batch means for averages, and the jackknife over batches for functions of
averages (susceptibility, Binder cumulant); batches longer than the
autocorrelation time make both autocorrelation-corrected."""
from __future__ import annotations

import numpy as np


def batches(x, nb):
    x = np.asarray(x, np.float64)
    n = len(x) // nb * nb
    return x[:n].reshape(nb, -1)


def mean_err(x, nb=50):
    b = batches(x, nb).mean(1)
    return float(b.mean()), float(b.std(ddof=1) / np.sqrt(nb))


def jackknife(f, series, nb=50):
    """f(*means) and its jackknife error; series: list of equally long arrays."""
    bs = [batches(s, nb) for s in series]
    tot = [b.sum() for b in bs]
    cnt = bs[0].size
    full = f(*[t / cnt for t in tot])
    per = bs[0].shape[1]
    jk = np.array([f(*[(t - b[k].sum()) / (cnt - per) for t, b in zip(tot, bs)]) for k in range(nb)])
    err = np.sqrt((nb - 1) / nb * np.sum((jk - jk.mean()) ** 2))
    return float(full), float(err)


def ising_summary(e, am, N, beta, nb=50):
    """<e>, <|m|>, chi = beta N (<m^2> - <|m|>^2), U4 = 1 - <m^4>/(3 <m^2>^2), each with its error."""
    am = np.asarray(am, np.float64)
    m2, m4 = am ** 2, am ** 4
    return {
        "e": mean_err(e, nb),
        "m": mean_err(am, nb),
        "chi": jackknife(lambda a, b: beta * N * (b - a * a), [am, m2], nb),
        "u4": jackknife(lambda b, c: 1.0 - c / (3.0 * b * b), [m2, m4], nb),
    }
