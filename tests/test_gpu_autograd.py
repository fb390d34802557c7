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
    """FDT gradients at beta = 0.37, lambda = 1.1 within 2 sigma of central
    differences (the FD runs reuse the chains' random numbers)."""
    n = 20000
    e = ens(n_meas=n, n_therm=500, common_random_numbers=True)
    b0, l0, db, dl = 0.37, LAM, 0.01, 0.02
    bs = torch.tensor([b0, b0 + db, b0 - db, b0, b0], dtype=torch.float64)
    ls = torch.tensor([l0, l0, l0, l0 + dl, l0 - dl], dtype=torch.float64)
    s = e.samples(bs, ls).cpu().numpy()
    N = e.sites
    _, jac = FDT.fdt(s[0], N, b0, l0, e.mass)
    obs, jc, _ = A.phi4_fdt(torch.from_numpy(s[:1]).cuda(), bs[:1], ls[:1], e)
    np.testing.assert_allclose(jc[0].cpu().numpy(), jac, rtol=1e-8, atol=1e-10)
    per = [FDT.per_sample(s[k], N, float(bs[k]), float(ls[k]), e.mass) for k in range(5)]
    # sigma of the FDT estimate from batch means of the per-batch FDT values
    nb = 20
    fd_batches = np.stack([FDT.fdt(x, N, b0, l0, e.mass)[1] for x in np.array_split(s[0], nb)])
    sig_fdt = fd_batches.std(0, ddof=1) / np.sqrt(nb)
    z = []
    for t, (i_up, i_dn, h) in enumerate(((1, 2, db), (3, 4, dl))):
        for j, key in enumerate(("E", "am")):
            diff = (per[i_up][key] - per[i_dn][key]) / (2 * h)
            fd, sig_fd = diff.mean(), FDT.batch_sigma(diff, nb)
            z.append(abs(fd - jac[j, t]) / np.hypot(sig_fd, sig_fdt[j, t]))
    z = np.array(z)
    assert (z < 2.0).mean() >= 0.75 and (z < 4.0).all(), f"z-scores {z}"


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
