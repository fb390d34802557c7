"""FP64 NumPy restatement of the phi^4 gradient estimators -- TEST
INFRASTRUCTURE (the checker of the engine's mqv_phi4_fdt kernel).

Action in the reference's phi^4 form (src/hamiltonian/Phi4.h:84-121, observables
as src/hamiltonian/util/observables.h:331-352 with the Phi4 onsite terms):
    S = -beta sum_<ij> phi_i phi_j + sum_i [mass phi_i^2 + lambda (phi_i^2 - 1)^2]
per-EMCS sums s = (I, M, Q2, Q4), I = sum_i phi_i sum_{j in nbrs(i)} phi_j.

``fdt``: fluctuation-dissipation derivatives d<O>/dtheta = -cov(O, dS/dtheta) +
<dO/dtheta>.  ``reweighted``: single-histogram reweighting of the same samples to
nearby couplings, <O>(theta') = <O' w> / <w>, w = exp(-(S(theta') - S(theta))).
"""
from __future__ import annotations

import numpy as np


def per_sample(s, N, beta, lam, mass):
    I, M, Q2, Q4 = (s[..., k].astype(np.float64) for k in range(4))
    E = (-0.5 * I + (mass / beta) * Q2 + (lam / beta) * Q4) / N
    am = np.abs(M) / N
    m2 = am * am
    return dict(E=E, am=am, m2=m2, m4=m2 * m2, dSb=-0.5 * I, dSl=Q4,
                dEb=-(mass * Q2 + lam * Q4) / (beta * beta) / N, dEl=Q4 / beta / N)


def observables(s, N, beta, lam, mass):
    p = per_sample(s, N, beta, lam, mass)
    m2, m4 = p["m2"].mean(), p["m4"].mean()
    return np.array([p["E"].mean(), p["am"].mean(), 1.0 - m4 / (3.0 * m2 * m2)])


def fdt(s, N, beta, lam, mass):
    """(obs [3], jac [3, 2]) of one chain's samples s [n, 4]."""
    p = per_sample(s, N, beta, lam, mass)
    cov = lambda a, b: np.mean((a - a.mean()) * (b - b.mean()))  # noqa: E731
    d = {}
    for o in ("E", "am", "m2", "m4"):
        d[o] = np.array([-cov(p[o], p["dSb"]), -cov(p[o], p["dSl"])])
    d["E"] += np.array([p["dEb"].mean(), p["dEl"].mean()])
    m2, m4 = p["m2"].mean(), p["m4"].mean()
    du = -d["m4"] / (3 * m2 * m2) + 2 * m4 * d["m2"] / (3 * m2 ** 3)
    return observables(s, N, beta, lam, mass), np.stack([d["E"], d["am"], du])


def reweighted(s, N, beta, lam, mass, beta2, lam2):
    """Observables at (beta2, lam2) reweighted from samples taken at (beta, lam)."""
    I, Q4 = s[:, 0].astype(np.float64), s[:, 3].astype(np.float64)
    dS = -(beta2 - beta) * 0.5 * I + (lam2 - lam) * Q4
    w = np.exp(-(dS - dS.min()))
    p = per_sample(s, N, beta2, lam2, mass)
    avg = lambda x: np.sum(w * x) / np.sum(w)  # noqa: E731
    m2, m4 = avg(p["m2"]), avg(p["m4"])
    return np.array([avg(p["E"]), avg(p["am"]), 1.0 - m4 / (3.0 * m2 * m2)])


def batch_sigma(x, nb=20):
    """Standard error of the mean of a correlated series by batch means."""
    n = len(x) // nb * nb
    b = np.asarray(x[:n]).reshape(nb, -1).mean(1)
    return b.std(ddof=1) / np.sqrt(nb)
