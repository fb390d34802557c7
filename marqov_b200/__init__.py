"""marqov_b200 -- MARQOV's Monte Carlo update hot path on NVIDIA B200 (sm_100a).

Metropolis colour sweeps and Wolff embedded clusters run as CUDA kernels
behind a C ABI (include/marqov_b200.h, libmarqov_b200.so in this package);
this package is the host side that mirrors MARQOV's Hamiltonian / lattice /
Core interface.  Importing it loads the engine library; there is no CPU path.
"""
from . import _lib, tempering
from ._lib import MarqovError
from .core import Batch, Config, Core, makeCore, tune_small_cap
from .hamiltonians import (BlumeCapel, BlumeCapelBipartite, EdwardsAndersonIsing, Hamiltonian, Heisenberg, Ising,
                           Phi4, Potts, XXZAntiferro, XXZAntiferroSingleAniso)
from .lattices import (BondedHypercubic, CSRLattice, FixedDimRegularHypercubic, RandomGeometricGraph2D, RegularHypercubic,
                       RegularRandomBond, SimpleBipartite, read_graph_csv, save_geometry)

_lib.load()

__all__ = ["tempering", "Batch", "Config", "Core", "makeCore", "tune_small_cap", "MarqovError", "Hamiltonian", "Ising", "EdwardsAndersonIsing",
           "Potts", "BlumeCapel", "BlumeCapelBipartite", "Heisenberg", "XXZAntiferro", "XXZAntiferroSingleAniso",
           "Phi4", "CSRLattice", "BondedHypercubic", "FixedDimRegularHypercubic", "RegularHypercubic", "SimpleBipartite",
           "RegularRandomBond", "RandomGeometricGraph2D",
           "read_graph_csv", "save_geometry"]
