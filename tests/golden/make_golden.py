"""Generate the golden fixtures in tests/golden from the reference itself.

Runs the reference's own templates (oracle/_ref/libmarqov_ref.so, built from
the MARQOV sources by oracle/build.py) and stores their outputs as small
.npz files, so the parity tests can check the oracle and the engine on
machines where the reference source is absent.

    python tests/golden/make_golden.py

Fixtures:
  metro_exp.npz   the acceptance known-answer test of
                  testsuite/components/5-metro_exp.cpp (N = 1e5, 500 passes,
                  beta = 0.44): accept counts of the MARQOV rule and of plain
                  exp, and a SHA-256 of the 5e7 individual decisions.
  (philox_curand.npz, cuRAND Philox4_32_10 blocks, is made on a GPU machine
  by make_philox_curand.py.)
  <case>.npz      Metropolis runs through MARQOV::Metropolis<H,L>::move in
                  colour order on the keyed Philox stream: initial state (by
                  the reference initstatespace rule where it has one), final
                  state, per-sweep reference observables (e, |m|, e_obs): e is
                  the energy per site the moves see (the reference's
                  nbrhoodloop / PottsInteraction::diff plus SelfEnergy),
                  e_obs the reference's Energy<H> observable, equal to e
                  except for Potts (its flex energy() is a stub returning 0)
                  and bond lattices (Energy ignores bnds()).
  ref_emcs_*.npz  <e>, <|m|>, chi, U4 and the mean cluster size (each with its
                  autocorrelation-corrected error) of the reference's own EMCS
                  loop -- random-site order, mt19937_64, its Wolff -- for
                  Potts, Heisenberg and phi^4.
  wolff_*.npz     cluster-size statistics of the unmodified reference Wolff
                  updates (sequential draws), for a statistical comparison
                  with the bond-keyed restatement; for the float models also
                  the per-EMCS energy and |m|.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from oracle.build import build_oracle, build_ref  # noqa: E402


def save(name, **arrs):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
    print("wrote", name, {k: getattr(v, "shape", v) for k, v in arrs.items()})


def main():
    build_oracle()
    if build_ref() is None:
        raise SystemExit("reference source tree not found: cannot build oracle/_ref")
    orc = O.Oracle()
    ref = O.RefHarness()

    # -- acceptance KAT (5-metro_exp.cpp at its own sizes)
    N, reps, beta = 100000, 500, 0.44
    acc, dec = ref.metro_exp(N, reps, beta, want_decisions=True)
    plain = ref.metro_exp_plain(N, reps, beta)
    digest = hashlib.sha256(np.packbits(dec).tobytes()).hexdigest()
    save("metro_exp", N=np.int64(N), reps=np.int64(reps), beta=np.float64(beta), accepted=np.int64(acc),
         accepted_plain=np.int64(plain), sha256=np.array(digest))
    # the first words of RNGCache<mt19937_64>{0}, to pin the oracle's MT19937-64
    save("mt19937_64_words", words=ref.mt_words(1024))

    # -- Metropolis cases through the reference templates
    def sublattice(g):
        """Per-site sublattice of a hypercubic graph: its parity colour."""
        sub = np.zeros(g.n, np.uint8)
        sub[g.order[g.colour_ptr[1]:]] = 1
        return sub

    def int_case(name, kind, ref_kind, dim, L, J, D, beta, seed, replica, nsweeps, q=0, bonds=None,
                 init_kind=None, D2=0.0, bipartite=False):
        g = orc.hypercubic(dim, L, bonds)
        if init_kind is not None:
            s0 = ref.init_int(init_kind, g.n, seed, replica)
        else:
            m = O.OrcModel(kind=kind, q=q, J=J, h=D, k=J)
            s0 = orc.init_int8(m, g.n, seed, replica)
        s = s0.copy()
        obs = ref.sweeps_int(ref_kind, g, s, J, D, beta, seed, replica, 0, nsweeps, D2=D2,
                             sub=sublattice(g) if bipartite else None)
        arrs = dict(kind=np.int32(kind), dim=np.int32(dim), L=np.int32(L), J=np.float64(J), D=np.float64(D),
                    D2=np.float64(D2), bipartite=np.int32(bipartite), q=np.int32(q), beta=np.float64(beta),
                    seed=np.uint64(seed), replica=np.uint32(replica), nsweeps=np.int32(nsweeps), init=s0, final=s,
                    obs=obs)
        if bonds is not None:
            arrs["bonds"] = bonds
        save(name, **arrs)

    int_case("ising2d_L16", O.ISING, 1, 2, 16, -1.0, 0.0, 0.44068679, 42, 0, 64, init_kind=1)
    int_case("ising2d_L64", O.ISING, 1, 2, 64, -1.0, 0.0, 0.44068679, 2024, 5, 40, init_kind=1)
    int_case("ising3d_L8", O.ISING, 1, 3, 8, -1.0, 0.0, 0.2216544, 7, 1, 40, init_kind=1)
    int_case("potts2d_L16", O.POTTS, 3, 2, 16, -1.0, 0.0, 1.0050525, 11, 2, 40, q=3, init_kind=3)
    int_case("bc2d_L16", O.BLUME_CAPEL, 4, 2, 16, -1.0, 0.5, 0.6, 13, 0, 40, init_kind=4)
    # BlumeCapelBipartite(J, DA, DB) on SimpleBipartite: DA on sublattice A, DB on B
    int_case("bcbip2d_L16", O.BLUME_CAPEL, 11, 2, 16, -1.0, 0.7, 0.6, 19, 1, 40, init_kind=4, D2=-0.4,
             bipartite=True)
    # Edwards-Anderson +-J on 3D L=8 with symmetric bimodal bonds
    L = 8
    g = orc.hypercubic(3, L)
    rng = np.random.default_rng(5)
    n = g.n
    cols = g.col_idx.reshape(n, 6)
    w = np.where(rng.random((n, 3)) < 0.5, 1, -1).astype(np.int8)
    bonds = np.empty((n, 6), np.int8)
    for j in range(3):
        bonds[:, 2 * j] = w[:, j]
        bonds[:, 2 * j + 1] = w[cols[:, 2 * j + 1], j]
    int_case("ea3d_L8", O.EA, 5, 3, L, -1.0, 0.0, 0.9, 17, 3, 40, bonds=bonds.reshape(-1))

    # -- float cases
    def f32_case(name, ref_kind, dim, L, J, p0, p1, cap, beta, seed, nsweeps, symd, p2=0.0, bipartite=False):
        g = orc.hypercubic(dim, L)
        kind = O.PHI4 if symd == 1 else O.HEISENBERG
        m = O.OrcModel(kind=kind, J=J)
        s0 = orc.init_f32(m, g.n, symd, seed, 0)
        s = s0.copy()
        obs = ref.sweeps_f32(ref_kind, g, s, J, p0, p1, cap, beta, seed, 0, 0, nsweeps, p2=p2,
                             sub=sublattice(g) if bipartite else None)
        save(name, dim=np.int32(dim), L=np.int32(L), J=np.float64(J), p0=np.float64(p0), p1=np.float64(p1),
             p2=np.float64(p2), bipartite=np.int32(bipartite), cap=np.float64(cap), beta=np.float64(beta),
             seed=np.uint64(seed), nsweeps=np.int32(nsweeps), symd=np.int32(symd), ref_kind=np.int32(ref_kind),
             init=s0, final=s, obs=obs)

    f32_case("heis3d_L8_fresh", 6, 3, 8, -1.0, 0, 0, 0.0, 0.6930, 21, 10, 3)
    f32_case("heis3d_L8_cap", 7, 3, 8, -1.0, 0, 0, 0.6, 0.6930, 22, 10, 3)
    f32_case("phi4_3d_L8", 8, 3, 8, -1.0, 1.1, 1.0, 0.5, 0.37, 23, 10, 1)
    # XXZAntiferro(Delta = 0.6, H = 0.35): J = +1, interaction (Delta x, Delta y, z), field on z
    f32_case("xxz3d_L8", 9, 3, 8, 1.0, 0.6, 0.35, 0.0, 0.7, 31, 10, 3)
    # XXZAntiferroSingleAniso(H = 0.25, Delta = 1.4, D = 0.5) on SimpleBipartite
    f32_case("xxzsa3d_L8_bip", 10, 3, 8, 1.0, 1.4, 0.25, 0.0, 0.9, 32, 10, 3, p2=0.5, bipartite=True)

    # -- Wolff statistics: unmodified reference clusters on Ising L=16 and Potts L=16
    for name, kind, okind, beta, q in (("wolff_ising_L16", 1, O.ISING, 0.44068679, 0),
                                        ("wolff_potts_L16", 3, O.POTTS, 1.0050525, 3)):
        g = orc.hypercubic(2, 16)
        m = O.OrcModel(kind=okind, q=q, J=-1.0, k=-1.0)
        s = orc.init_int8(m, g.n, 99, 0)
        for t in range(200):
            orc.sweep_int8(m, g, s, beta, 99, 0, t)
        sizes = []
        for t in range(4000):
            sizes.append(int(ref.wolff_int(kind, g, s, -1.0, beta, 99, 0, t, 1)[0]))
            orc.sweep_int8(m, g, s, beta, 99, 0, 1000 + t)
        sizes = np.array(sizes, np.int32)
        save(name, beta=np.float64(beta), q=np.int32(q), sizes=sizes)

    # -- Wolff statistics of the float models: the reference's generic Wolff
    # with Embedder<Heisenberg> / the scalar Embedder<Phi4>, one cluster then
    # one colour-order Metropolis sweep per EMCS on a 3D L = 8 lattice
    for name, rkind, okind, symd, beta, p0, p1, amp in (
            ("wolff_heis_L8", 6, O.HEISENBERG, 3, 0.6930, 0.0, 0.0, 0.0),
            ("wolff_phi4_L8", 8, O.PHI4, 1, 0.37, 1.1, 1.0, 0.5)):
        g = orc.hypercubic(3, 8)
        m = O.OrcModel(kind=okind, J=-1.0, h=p1 / beta, h2=p0 / beta, cap=amp)
        s = orc.init_f32(m, g.n, symd, 77, 0)
        for t in range(200):
            orc.sweep_f32(m, g, s, symd, beta, 77, 0, t)
        sizes, energies, mags = [], [], []
        for t in range(6000):
            sizes.append(int(ref.wolff_f32(rkind, g, s, -1.0, p0, p1, beta, 77, 0, t, 1)[0]))
            orc.sweep_f32(m, g, s, symd, beta, 77, 0, 1000 + t)
            e, mm, _, _ = orc.measure_f32(m, g, s, symd)
            energies.append(e)
            mags.append(mm)
        save(name, beta=np.float64(beta), p0=np.float64(p0), p1=np.float64(p1), amp=np.float64(amp),
             sizes=np.array(sizes, np.int32), e=np.array(energies), m=np.array(mags))

    # -- long-run statistics of the reference's own EMCS loop (random-site
    # order, mt19937_64, reference Wolff): value and tau_int-corrected error
    # of <e>, <|m|>, chi, U4 and the mean cluster size after 10^3 + 10^4 EMCS
    from oracle import stats as S
    for name, rk, dim, L, beta, ncl, nmet, kw in (
            ("ref_emcs_potts2d_L16", 3, 2, 16, 1.0050525, 1, 1, {}),
            ("ref_emcs_heis3d_L8", 6, 3, 8, 0.6930, 1, 5, {}),
            ("ref_emcs_phi4_3d_L8", 8, 3, 8, 0.37, 1, 2, dict(p0=1.1, p1=1.0, p2=0.5))):
        obs, mc = ref.emcs_generic(rk, L, dim, -1.0, beta, 11, ncl, nmet, 1000, 10000, **kw)
        summ = S.summary(obs[:, 0], obs[:, 1], L ** dim, beta)
        cm, ce = S.mean_err(mc)
        save(name, kind=np.int32(rk), dim=np.int32(dim), L=np.int32(L), beta=np.float64(beta), ncluster=np.int32(ncl),
             nmetro=np.int32(nmet), p0=np.float64(kw.get("p0", 0.0)), p1=np.float64(kw.get("p1", 0.0)),
             p2=np.float64(kw.get("p2", 0.0)), ntherm=np.int32(1000), nmeas=np.int32(10000),
             **{k: np.array(v) for k, v in summ.items()}, cluster=np.array([cm, ce]))


if __name__ == "__main__":
    main()
