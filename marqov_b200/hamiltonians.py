"""Hamiltonians in MARQOV's form, lowered to engine model descriptors.

Each class mirrors a reference Hamiltonian (constructor arguments, ``SymD``,
``name``, sign convention ``dE = J dot(s_new - s_old, sum_nbrs)`` of
src/libmarqov/metropolishelpers.h:598-623) and knows how to describe itself to
the engine (``desc(beta)``).  A model the engine cannot lower raises
``MarqovError(UNSUPPORTED_TERM)`` when the core is created -- there is no CPU
fallback.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L


class Hamiltonian:
    SymD = 1
    name = "Hamiltonian"
    kind = 0
    dtype = np.int8
    # Wolff embedding available (ferromagnetic couplings)
    wolff = True

    def desc(self, beta: float) -> L.ModelDesc:  # pragma: no cover - abstract
        raise NotImplementedError

    def __repr__(self):
        return f"{self.name}({', '.join(f'{k}={v}' for k, v in vars(self).items())})"


class Ising(Hamiltonian):
    """``Ising<SpinType>`` (src/hamiltonian/Ising.h:62-109).

    ``spintype="int"`` (the reference default) selects ``Wolff<Ising<int>>`` with
    the exact -expm1 bond probability (Ising.h:122-169); ``spintype="int8"``
    selects the generic Wolff with the default Embedder that ``Ising<int8_t>``
    instantiates (src/libmarqov/wolff.h:72-126).  Spins are stored as int8 on
    the device either way.
    """

    SymD = 1
    name = "Ising"

    def __init__(self, J: float = -1.0, spintype: str = "int"):
        if spintype not in ("int", "int8"):
            raise ValueError("spintype must be 'int' or 'int8'")
        self.J = float(J)
        self.spintype = spintype

    @property
    def kind(self):
        return L.MODEL_ISING if self.spintype == "int" else L.MODEL_ISING_EMBED

    def desc(self, beta):
        return L.ModelDesc(kind=self.kind, J=self.J)


class EdwardsAndersonIsing(Hamiltonian):
    """``EdwardsAndersonIsing`` (src/hamiltonian/EdwardsAndersonIsing.h:274-331):
    Ising interaction weighted by the lattice's ``bnds``."""

    SymD = 1
    name = "EdwardsAndersonIsing"
    kind = L.MODEL_EA
    wolff = False

    def __init__(self, J: float = -1.0):
        self.J = float(J)

    def desc(self, beta):
        return L.ModelDesc(kind=L.MODEL_EA, J=self.J)


class Potts(Hamiltonian):
    """``Potts<Q>`` (src/hamiltonian/Potts.h:118-158): Dirac-delta flex term with
    prefactor k (``Potts<Q>(J)`` stores J as k; ferromagnetic is k < 0)."""

    SymD = 1
    name = "Potts"
    kind = L.MODEL_POTTS

    def __init__(self, q: int, J: float = -1.0):
        self.q = int(q)
        self.J = float(J)

    def desc(self, beta):
        return L.ModelDesc(kind=L.MODEL_POTTS, q=self.q, k=self.J)


class BlumeCapel(Hamiltonian):
    """``BlumeCapel`` (src/hamiltonian/BlumeCapel.h:46-153): spin-1 states with
    the Spin1 proposal and onsite D s^2.  It has no ``initstatespace``, so its
    initial state is ``Core::init_hot``'s: +-1 (src/libmarqov/core.h:773-782)."""

    SymD = 1
    name = "BlumeCapel"
    kind = L.MODEL_BLUME_CAPEL
    wolff = False

    def __init__(self, J: float = -1.0, D: float = 0.0):
        self.J = float(J)
        self.D = float(D)

    def desc(self, beta):
        return L.ModelDesc(kind=L.MODEL_BLUME_CAPEL, J=self.J, h=self.D)


class BlumeCapelBipartite(Hamiltonian):
    """``BlumeCapelBipartite(J, DA, DB)`` (src/hamiltonian/BlumeCapelBipartite.h:39-86):
    Blume-Capel with two onsite s^2 terms.  On a ``SimpleBipartite`` lattice the
    termselector gives sublattice A the term DA and B the term DB; on any other
    lattice both act on every site, as in the reference."""

    SymD = 1
    name = "BlumeCapelBipartite"
    kind = L.MODEL_BLUME_CAPEL
    wolff = False

    def __init__(self, J: float = -1.0, DA: float = 0.0, DB: float = 0.0):
        self.J = float(J)
        self.DA = float(DA)
        self.DB = float(DB)

    def desc(self, beta):
        return L.ModelDesc(kind=L.MODEL_BLUME_CAPEL, J=self.J, h=self.DA, h2=self.DB)


class Heisenberg(Hamiltonian):
    """``Heisenberg<float>`` (src/hamiltonian/Heisenberg.h:62-105) with the
    plane-reflection embedder (Heisenberg.h:123-186).

    ``proposal="fresh"`` is the reference's fresh uniform direction
    (src/hamiltonian/util/initializers.h:74-80); ``proposal="smallcap"`` draws
    uniformly from the cap of half-angle theta around the old spin, with
    ``cap = cos(theta)``.
    """

    SymD = 3
    name = "Heisenberg"
    kind = L.MODEL_HEISENBERG
    dtype = np.float32

    def __init__(self, J: float = -1.0, proposal: str = "fresh", cap: float = 0.5):
        if proposal not in ("fresh", "smallcap"):
            raise ValueError("proposal must be 'fresh' or 'smallcap'")
        self.J = float(J)
        self.proposal = proposal
        self.cap = float(cap)

    def desc(self, beta):
        return L.ModelDesc(kind=L.MODEL_HEISENBERG, J=self.J,
                           proposal=L.PROPOSAL_SMALL_CAP if self.proposal == "smallcap" else 0,
                           cap=self.cap)


class XXZAntiferro(Hamiltonian):
    """``XXZAntiferro(Delta, H)`` (src/hamiltonian/XXZAntiferro.h:135-205): O(3)
    spins with the interaction ``get(s) = (Delta s_x, Delta s_y, s_z)`` and the
    reference's fixed antiferromagnetic ``J = +1`` (XXZAntiferro.h:141-150),
    plus the field ``H s_z`` (``XXZAntiferro_extfield``, :162-170).

    As in the reference, the Metropolis energy difference is
    ``J dot(s_new - s_old, sum_j get(s_j))`` (linear in Delta) while the
    ``Energy`` observable applies ``get`` to both ends of a bond, so its x and y
    parts carry Delta^2 (src/hamiltonian/util/observables.h:186-217).  No Wolff
    embedding (the reference has none for this model).  ``proposal="smallcap"``
    replaces the fresh-direction proposal by the small-cap one of
    ``Heisenberg``."""

    SymD = 3
    name = "XXZAntiferro"
    kind = L.MODEL_XXZ
    dtype = np.float32
    wolff = False
    J = 1.0

    def __init__(self, Delta: float = 1.0, H: float = 0.0, proposal: str = "fresh", cap: float = 0.5):
        if proposal not in ("fresh", "smallcap"):
            raise ValueError("proposal must be 'fresh' or 'smallcap'")
        self.Delta = float(Delta)
        self.H = float(H)
        self.proposal = proposal
        self.cap = float(cap)

    def _onsite(self):
        return self.H, 0.0

    def desc(self, beta):
        h, h2 = self._onsite()
        return L.ModelDesc(kind=L.MODEL_XXZ, J=self.J, delta=self.Delta, h=h, h2=h2,
                           proposal=L.PROPOSAL_SMALL_CAP if self.proposal == "smallcap" else 0,
                           cap=self.cap)


class XXZAntiferroSingleAniso(XXZAntiferro):
    """``XXZAntiferroSingleAniso(H, Delta, D)`` (src/hamiltonian/XXZAntiferroSingleAniso.h:54-96;
    note the reference's argument order): ``XXZAntiferro`` plus the single-ion
    anisotropy ``D s_z^2`` as onsite term 1.  On a ``SimpleBipartite`` lattice
    the termselector gives sublattice A the field and B the anisotropy."""

    name = "XXZAntiferroSingleAniso"

    def __init__(self, H: float = 0.0, Delta: float = 1.0, D: float = 0.0, proposal: str = "fresh",
                 cap: float = 0.5):
        super().__init__(Delta, H, proposal, cap)
        self.D = float(D)

    def _onsite(self):
        return self.H, self.D


class Phi4(Hamiltonian):
    """Scalar phi^4 in the reference's Phi4 form (src/hamiltonian/Phi4.h:84-121):
    J = -1, onsite (mass/beta) phi^2 + (lambda/beta) (phi^2 - 1)^2, so that
    beta H = -beta sum phi_i phi_j + sum [mass phi^2 + lambda (phi^2 - 1)^2];
    shift proposal old + amp * U(-1, 1) (Phi4_Initializer_Cartesian, Phi4.h:37-58)
    and the reflection embedder (Phi4.h:182-244)."""

    SymD = 1
    name = "Phi4"
    kind = L.MODEL_PHI4
    dtype = np.float32

    def __init__(self, beta: float, lambda_: float, mass: float = 1.0, amp: float = 0.5):
        self.beta = float(beta)
        self.lambda_ = float(lambda_)
        self.mass = float(mass)
        self.amp = float(amp)
        self.J = -1.0

    def desc(self, beta):
        # the onsite prefactors carry the Hamiltonian's own beta, as Phi4.h:110-115
        return L.ModelDesc(kind=L.MODEL_PHI4, J=-1.0, h=self.mass / self.beta,
                           h2=self.lambda_ / self.beta, cap=self.amp)
