"""Differentiable ensemble observables of scalar phi^4 (torch.autograd).

``phi4_observables(beta, lam, ens)`` runs one Markov chain per (beta, lambda)
pair on the GPU -- the reference's phi^4 form (src/hamiltonian/Phi4.h:84-121),
S = -beta sum_<ij> phi_i phi_j + sum_i [mass phi_i^2 + lambda (phi_i^2 - 1)^2],
Metropolis shift proposals plus embedded Wolff reflections -- and returns
<E>, <|m|> and U4 = 1 - <m^4> / (3 <m^2>^2) per pair.  The per-EMCS lattice
sums stay on the device (mqv_emcs_samples); backward is the engine's
fluctuation-dissipation kernel (mqv_phi4_fdt),
d<O>/dtheta = -<O dS/dtheta> + <O><dS/dtheta> + <dO/dtheta>,
contracted with the incoming gradient.  There is no counterpart in the
reference, which has no gradients.

Chains are keyed by (seed, replica id): by default the replica id is the
chain's position in the batch; with ``common_random_numbers`` every chain uses
replica id 0, so chains at shifted couplings draw the same random numbers
(for finite-difference checks).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from . import _lib as L
from .core import Batch, Config
from .hamiltonians import Phi4
from .lattices import RegularHypercubic


@dataclass
class Phi4Ensemble:
    """Run settings: lattice side and dimension, mass and shift amplitude of
    the model, EMCS shape (ncluster Wolff clusters + nmetro sweeps), and how
    many EMCS are discarded (n_therm) and measured (n_meas)."""
    L: int = 16
    dim: int = 3
    mass: float = 1.0
    amp: float = 0.5
    ncluster: int = 1
    nmetro: int = 1
    n_therm: int = 200
    n_meas: int = 2000
    seed: int = 0
    device: int = 0
    common_random_numbers: bool = False

    @property
    def sites(self) -> int:
        return self.L ** self.dim

    def samples(self, beta: torch.Tensor, lam: torch.Tensor) -> torch.Tensor:
        """Per-EMCS sums [R, n_meas, 4] (FP64, on the GPU) of R chains."""
        b = beta.detach().to("cpu", torch.float64).reshape(-1)
        lm = lam.detach().to("cpu", torch.float64).reshape(-1)
        if b.numel() != lm.numel():
            raise ValueError("beta and lambda need one entry per chain")
        dev = torch.device("cuda", self.device)
        out = torch.empty((b.numel(), self.n_meas, 4), dtype=torch.float64, device=dev)
        members = []
        for r in range(b.numel()):
            rep = 0 if self.common_random_numbers else r
            cfg = Config(seed=self.seed, repid=rep, device=self.device, ncluster=self.ncluster, nmetro=self.nmetro)
            members.append((RegularHypercubic(self.L, self.dim), cfg,
                            Phi4(float(b[r]), float(lm[r]), self.mass, self.amp), float(b[r])))
        torch.cuda.current_stream(dev).synchronize()
        # all chains in one batch (batched kernels replayed from a CUDA graph)
        with Batch(members) as bt:
            bt.init()
            if self.n_therm:
                bt.emcs(self.n_therm, self.ncluster, self.nmetro)
            L.check(L.load().mqv_batch_emcs_samples(bt._h, self.n_meas, self.ncluster, self.nmetro,
                                                    C.c_void_p(out.data_ptr())))
        return out


def phi4_fdt(samples: torch.Tensor, beta: torch.Tensor, lam: torch.Tensor, ens: Phi4Ensemble,
             gout: torch.Tensor | None = None):
    """The engine's FDT kernel on device samples: (obs [R, 3], jac [R, 3, 2],
    grads [R, 2] or None)."""
    dev = samples.device
    R, n, _ = samples.shape
    s = samples.contiguous()
    b = beta.detach().to(dev, torch.float64).reshape(-1).contiguous()
    lm = lam.detach().to(dev, torch.float64).reshape(-1).contiguous()
    obs = torch.empty((R, 3), dtype=torch.float64, device=dev)
    jac = torch.empty((R, 3, 2), dtype=torch.float64, device=dev)
    g = grads = None
    if gout is not None:
        g = gout.detach().to(dev, torch.float64).reshape(R, 3).contiguous()
        grads = torch.empty((R, 2), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    L.check(L.load().mqv_phi4_fdt(ptr(s), R, n, ens.sites, ens.mass, ptr(b), ptr(lm), ptr(obs), ptr(jac), ptr(g),
                                  ptr(grads), C.c_void_p(stream.cuda_stream)))
    return obs, jac, grads


class _Phi4Observables(torch.autograd.Function):
    @staticmethod
    def forward(ctx, beta, lam, ens):
        samples = ens.samples(beta, lam)
        obs, _, _ = phi4_fdt(samples, beta, lam, ens)
        ctx.ens = ens
        ctx.save_for_backward(samples, beta.detach(), lam.detach())
        ctx.out_dtype, ctx.out_device = beta.dtype, beta.device
        return obs.to(beta.device, beta.dtype)

    @staticmethod
    def backward(ctx, gout):
        samples, beta, lam = ctx.saved_tensors
        _, _, grads = phi4_fdt(samples, beta, lam, ctx.ens, gout)
        grads = grads.to(ctx.out_device, ctx.out_dtype)
        return grads[:, 0], grads[:, 1], None


def phi4_observables(beta: torch.Tensor, lam: torch.Tensor, ens: Phi4Ensemble) -> torch.Tensor:
    """<E>, <|m|>, U4 per (beta, lambda) pair, [R, 3]; differentiable in beta
    and lambda through the fluctuation-dissipation kernel."""
    return _Phi4Observables.apply(beta, lam, ens)


# ---------------------------------------------------------------------------
# Uses of the gradients: coupling fitting and critical-point location.

def _scalar_obs(beta: float, lam: float, ens: Phi4Ensemble):
    """(observables [3], d obs / d beta [3]) of one chain at (beta, lam)."""
    b = torch.tensor([beta], dtype=torch.float64)
    lm = torch.tensor([lam], dtype=torch.float64)
    s = ens.samples(b, lm)
    obs, jac, _ = phi4_fdt(s, b, lm, ens)
    return obs[0].cpu(), jac[0, :, 0].cpu()


def fit_beta(target: float, lam: float, ens: Phi4Ensemble, beta0: float, which: int = 0, steps: int = 6,
             max_step: float = 0.01):
    """The beta at which observable `which` (0: <E>, 1: <|m|>, 2: U4) of the
    phi^4 ensemble equals `target`: Newton steps beta <- beta - (O - target) /
    (dO/dbeta) with the derivative from the fluctuation-dissipation kernel,
    each step capped at max_step.  Returns (beta, [(beta, O, dO/dbeta), ...]).
    Each step runs fresh chains with the ensemble's seed plus the step."""
    beta, hist = float(beta0), []
    for k in range(steps):
        e = Phi4Ensemble(**{**ens.__dict__, "seed": ens.seed + k})
        obs, d = _scalar_obs(beta, lam, e)
        o, do = float(obs[which]), float(d[which])
        hist.append((beta, o, do))
        step = -(o - target) / do if do != 0 else 0.0
        beta += max(-max_step, min(max_step, step))
    return beta, hist


def binder_crossing(lam: float, ens_a: Phi4Ensemble, ens_b: Phi4Ensemble, beta0: float, steps: int = 5,
                    max_step: float = 0.005):
    """The beta at which the Binder cumulants U4 of two lattice sizes cross
    (the finite-size estimate of the critical coupling): Newton steps on
    f(beta) = U4_a - U4_b with f' = dU4_a/dbeta - dU4_b/dbeta from the
    fluctuation-dissipation kernel.  Returns (beta, [(beta, f, f'), ...])."""
    beta, hist = float(beta0), []
    for k in range(steps):
        ea = Phi4Ensemble(**{**ens_a.__dict__, "seed": ens_a.seed + k})
        eb = Phi4Ensemble(**{**ens_b.__dict__, "seed": ens_b.seed + k})
        oa, da = _scalar_obs(beta, lam, ea)
        ob, db = _scalar_obs(beta, lam, eb)
        f, fp = float(oa[2] - ob[2]), float(da[2] - db[2])
        hist.append((beta, f, fp))
        step = -f / fp if fp != 0 else 0.0
        beta += max(-max_step, min(max_step, step))
    return beta, hist
