"""Gradients of phi^4 ensemble observables (marqov_b200.autograd): the
engine's fluctuation-dissipation kernel against the FP64 NumPy restatement on
the same device samples, against histogram reweighting of those samples,
against central finite differences with common random numbers, and through
torch.autograd."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def setup_module():
    global torch, A, FDT
    import torch  # noqa: F811
    import marqov_b200.autograd as A  # noqa: F811
    from oracle import fdt as FDT  # noqa: F811


BETAS = [0.36, 0.37, 0.38]
LAM = 1.1


def ens(**kw):
    base = dict(L=4, dim=3, n_therm=300, n_meas=4000, seed=77)
    base.update(kw)
    return A.Phi4Ensemble(**base)


def test_kernel_matches_numpy_on_same_samples():
    e = ens(n_meas=3000)
    b = torch.tensor(BETAS, dtype=torch.float64)
    lm = torch.full((3,), LAM, dtype=torch.float64)
    s = e.samples(b, lm)
    obs, jac, _ = A.phi4_fdt(s, b, lm, e)
    sh = s.cpu().numpy()
    for r in range(3):
        o_ref, j_ref = FDT.fdt(sh[r], e.sites, BETAS[r], LAM, e.mass)
        np.testing.assert_allclose(obs[r].cpu().numpy(), o_ref, rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(jac[r].cpu().numpy(), j_ref, rtol=1e-8, atol=1e-10)


def test_kernel_matches_histogram_reweighting():
    e = ens(n_meas=4000)
    b = torch.tensor([0.37], dtype=torch.float64)
    lm = torch.tensor([LAM], dtype=torch.float64)
    s = e.samples(b, lm)
    _, jac, _ = A.phi4_fdt(s, b, lm, e)
    sh = s.cpu().numpy()[0]
    h = 1e-5
    for t, (db, dl) in enumerate(((h, 0.0), (0.0, h))):
        up = FDT.reweighted(sh, e.sites, 0.37, LAM, e.mass, 0.37 + db, LAM + dl)
        dn = FDT.reweighted(sh, e.sites, 0.37, LAM, e.mass, 0.37 - db, LAM - dl)
        np.testing.assert_allclose(jac[0, :, t].cpu().numpy(), (up - dn) / (2 * h), rtol=1e-4, atol=1e-8)


def test_fdt_agrees_with_finite_differences_common_randoms():
    """FDT gradients of <E>, <|m|> and U4 with respect to beta and lambda, at
    beta = 0.37, lambda = 1.1 on 3D L = 16, all six within 2 sigma of central
    differences with step 1e-3 whose chains reuse the central chain's random
    numbers.  Sigmas: batch means over 20 common batches, the FD one from the
    per-batch differences (so it keeps the correlation of the paired chains)."""
    n, nb, h = 40000, 20, 1e-3
    e = ens(L=16, n_meas=n, n_therm=1000, common_random_numbers=True)
    b0, l0 = 0.37, LAM
    bs = torch.tensor([b0, b0 + h, b0 - h, b0, b0], dtype=torch.float64)
    ls = torch.tensor([l0, l0, l0, l0 + h, l0 - h], dtype=torch.float64)
    s = e.samples(bs, ls).cpu().numpy()
    N = e.sites
    _, jac = FDT.fdt(s[0], N, b0, l0, e.mass)
    _, jc, _ = A.phi4_fdt(torch.from_numpy(s[:1]).cuda(), bs[:1], ls[:1], e)
    np.testing.assert_allclose(jc[0].cpu().numpy(), jac, rtol=1e-8, atol=1e-10)
    split = [np.array_split(s[k], nb) for k in range(5)]
    jac_b = np.stack([FDT.fdt(x, N, b0, l0, e.mass)[1] for x in split[0]])
    sig_fdt = jac_b.std(0, ddof=1) / np.sqrt(nb)
    obs_b = [np.stack([FDT.observables(x, N, float(bs[k]), float(ls[k]), e.mass) for x in split[k]])
             for k in range(5)]
    obs_all = [FDT.observables(s[k], N, float(bs[k]), float(ls[k]), e.mass) for k in range(5)]
    z = np.zeros((3, 2))
    for t, (up, dn) in enumerate(((1, 2), (3, 4))):
        fd = (obs_all[up] - obs_all[dn]) / (2 * h)
        fd_b = (obs_b[up] - obs_b[dn]) / (2 * h)
        sig_fd = fd_b.std(0, ddof=1) / np.sqrt(nb)
        z[:, t] = np.abs(fd - jac[:, t]) / np.hypot(sig_fd, sig_fdt[:, t])
    assert (z < 2.0).all(), f"z-scores (rows E, |m|, U4; columns beta, lambda):\n{z}"


def test_fit_beta_recovers_a_known_coupling():
    """Coupling fitting with the FDT derivative: the beta whose <E> equals the
    <E> measured at beta* = 0.372, found by Newton steps from beta = 0.36."""
    e = ens(L=8, n_meas=20000, n_therm=500, seed=5)
    target = float(A._scalar_obs(0.372, LAM, A.Phi4Ensemble(**{**e.__dict__, "seed": 999}))[0][0])
    beta, hist = A.fit_beta(target, LAM, e, 0.36, which=0, steps=5)
    assert abs(beta - 0.372) < 0.002, (beta, hist)
    assert all(h[2] < 0 for h in hist)  # <E> falls with beta


def test_binder_crossing_locates_the_transition():
    """Critical-point location with the FDT derivative: the crossing of the
    Binder cumulants of L = 6 and L = 10 by Newton steps on U4_6 - U4_10,
    starting at 0.365; it must settle inside the window the configuration
    scans (0.36 .. 0.38) with a residual within 2 sigma of zero."""
    ea = ens(L=6, n_meas=30000, n_therm=1000, seed=21)
    eb = ens(L=10, n_meas=30000, n_therm=1000, seed=41)
    beta, hist = A.binder_crossing(LAM, ea, eb, 0.365, steps=5)
    assert 0.36 < beta < 0.385, (beta, hist)
    # the residual at the final beta, with its batch-means error
    b = torch.tensor([beta], dtype=torch.float64)
    lm = torch.tensor([LAM], dtype=torch.float64)
    u = []
    for e in (A.Phi4Ensemble(**{**ea.__dict__, "seed": 7}), A.Phi4Ensemble(**{**eb.__dict__, "seed": 8})):
        sm = e.samples(b, lm).cpu().numpy()[0]
        ub = np.array([FDT.observables(x, e.sites, beta, LAM, e.mass)[2] for x in np.array_split(sm, 20)])
        u.append((FDT.observables(sm, e.sites, beta, LAM, e.mass)[2], ub.std(ddof=1) / np.sqrt(20)))
    f, sf = u[0][0] - u[1][0], np.hypot(u[0][1], u[1][1])
    assert abs(f) < 2 * sf + 1e-3, (beta, f, sf, hist)


def test_autograd_backward_is_vjp_of_the_kernel_jacobian():
    e = ens(n_meas=2000)
    b = torch.tensor(BETAS, dtype=torch.float64, requires_grad=True)
    lm = torch.full((3,), LAM, dtype=torch.float64, requires_grad=True)
    obs = A.phi4_observables(b, lm, e)
    w = torch.tensor([[1.0, -2.0, 0.5], [0.3, 0.0, 1.0], [-1.0, 1.0, 2.0]], dtype=torch.float64)
    (obs * w).sum().backward()
    s = e.samples(b, lm)  # same seed: the same chains
    _, jac, _ = A.phi4_fdt(s, b, lm, e)
    jac = jac.cpu()
    np.testing.assert_allclose(b.grad.numpy(), (w[:, :, None] * jac).sum(1)[:, 0].numpy(), rtol=1e-10)
    np.testing.assert_allclose(lm.grad.numpy(), (w[:, :, None] * jac).sum(1)[:, 1].numpy(), rtol=1e-10)
    # physics: the energy falls and |m| grows with beta near the transition
    assert (jac[:, 0, 0] < 0).all() and (jac[:, 1, 0] > 0).all()
