"""Error bars of correlated Monte Carlo series -- TEST INFRASTRUCTURE.

* tau_int: the integrated autocorrelation time with Sokal's automatic
  window (the smallest W with W >= c tau_int(W), c = 6; A. D. Sokal,
  "Monte Carlo methods in statistical mechanics", 1996); the error of a mean
  is sqrt(2 tau_int var / n).
* Batch means for averages, and the jackknife over batches for functions of
  averages (susceptibility, Binder cumulant); batches longer than the
  autocorrelation time make both autocorrelation-corrected.
* summary(): each quantity with the larger of its batch and tau_int errors."""
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


def tau_int(x, c=6.0):
    """Integrated autocorrelation time (1/2 + sum of normalised autocorrelations
    up to Sokal's window) of a series."""
    x = np.asarray(x, np.float64)
    n = len(x)
    d = x - x.mean()
    var = float(d @ d) / n
    if var == 0.0:
        return 0.5
    f = np.fft.rfft(d, 2 * n)
    acf = np.fft.irfft(f * np.conj(f))[:n] / (n * var)
    tau = 0.5
    for w in range(1, n):
        tau += acf[w]
        if w >= c * tau:
            break
    return float(max(tau, 0.5))


def mean_err_tau(x, c=6.0):
    """Mean and its autocorrelation-corrected error sqrt(2 tau_int var / n)."""
    x = np.asarray(x, np.float64)
    t = tau_int(x, c)
    return float(x.mean()), float(np.sqrt(2.0 * t * x.var() / len(x))), t


def summary(e, am, N, beta, nb=50):
    """<e>, <|m|>, chi = beta N (<m^2> - <|m|>^2), U4 = 1 - <m^4>/(3 <m^2>^2):
    value and error, the error the larger of batch means (jackknife for chi
    and U4) and the tau_int estimate (for chi and U4 the jackknife error
    scaled up where tau_int of m^2 exceeds the batch length / 10)."""
    am = np.asarray(am, np.float64)
    out = ising_summary(e, am, N, beta, nb)
    for k, x in (("e", e), ("m", am)):
        m, err_t, _ = mean_err_tau(x)
        out[k] = (out[k][0], max(out[k][1], err_t))
    blen = len(am) // nb
    t2 = tau_int(am ** 2)
    scale = max(1.0, np.sqrt(10.0 * t2 / blen))
    for k in ("chi", "u4"):
        out[k] = (out[k][0], out[k][1] * scale)
    return out
