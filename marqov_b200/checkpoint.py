"""The reference's dump container without HDF5.

MARQOV keeps one HDF5 file per simulation, ``<outpath><outname>.h5``
(Core::setupHDF5Container / dumppresent, src/libmarqov/core.h:635-665).
Every construction of a Core on an existing file adds a step group
``/step<N>`` (createstep, core.h:741-768) and continues from step N-1's
final state and RNG state (setupstatespace, core.h:543-607); a step holds
the environment, the configuration, the observable time series and, at the
end (~Core, core.h:876-902), the final state.  HDF5 is not available to this
package, so the same tree is kept as a directory, one file per data set:

    <outpath><outname>.mqv/
        step<N>/
            environment.json                    (dumpenvtoH5)
            config/marqovconfig.json            beta and Config's parameters
            config/lattice.json                 the lattice's parameters
            config/hamiltonian.json             the Hamiltonian's name and parameters
            state/hamiltonianstatespace.npy     final state, reference site order
            state/hash.json                     FNV-1a 64-bit hash of the state's bytes
            state/RNG.txt                       the generator's name
            state/rngstate.npy                  uint64: seed, replica, sweep, cluster
            observables/<name>.npy              one value per measurement
                                                (e, m, m2, m4, clustersize)

The engine's random numbers are keyed by (seed, replica, sweep, cluster),
so those four words are the whole RNG state.  A step whose state file is
truncated or unreadable, or whose bytes do not match the stored hash, is
refused with MarqovError(CHECKSUM) instead of being continued from.
"""
from __future__ import annotations

import json
import os
import platform
import time

import numpy as np

RNG_NAME = "Philox4x32-10, keyed by (seed, replica, sweep, cluster)"


def container_path(config) -> str:
    """``outpath + outname`` as the reference joins them, with our suffix."""
    return f"{config.outpath}{config.outname}.mqv"


def dump_present(config) -> bool:
    """Core::dumppresent: a container with at least one step exists."""
    return last_step(container_path(config)) >= 0


def last_step(path: str) -> int:
    """findstep (core.h:620-634): the largest N of the step<N> groups, -1 if none."""
    if not os.path.isdir(path):
        return -1
    steps = [int(d[4:]) for d in os.listdir(path) if d.startswith("step") and d[4:].isdigit()]
    return max(steps) if steps else -1


def _params(obj) -> dict:
    out = {}
    for k, v in vars(obj).items():
        if k.startswith("_"):
            continue
        if isinstance(v, (bool, int, float, str)):
            out[k] = v
        elif isinstance(v, np.generic):
            out[k] = v.item()
    return out


def _write_json(path: str, obj) -> None:
    with open(path, "w") as fh:
        json.dump(obj, fh, indent=1, sort_keys=True)


class Step:
    """One step group: created when a Core starts, completed when it ends."""

    def __init__(self, path: str, index: int):
        self.path = os.path.join(path, f"step{index}")
        self.index = index

    def create(self, beta: float, config, lattice, ham, engine_version: str) -> "Step":
        for sub in ("config", "state", "observables"):
            os.makedirs(os.path.join(self.path, sub), exist_ok=True)
        _write_json(os.path.join(self.path, "environment.json"),
                    {"engine": engine_version, "host": platform.node(), "python": platform.python_version(),
                     "created": time.strftime("%Y-%m-%dT%H:%M:%S%z")})
        mc = {k: getattr(config, k) for k in ("id", "repid", "seed", "nsteps", "warmupsteps", "gameloopsteps",
                                              "ncluster", "nmetro")}
        mc["beta"] = float(beta)
        _write_json(os.path.join(self.path, "config", "marqovconfig.json"), mc)
        _write_json(os.path.join(self.path, "config", "lattice.json"),
                    {"name": type(lattice).__name__, "size": int(lattice.size()), **_params(lattice)})
        _write_json(os.path.join(self.path, "config", "hamiltonian.json"),
                    {"name": type(ham).__name__, **_params(ham)})
        return self

    def write_state(self, state: np.ndarray, seed: int, replica: int, sweep: int, cluster: int,
                    hash_: int | None = None) -> None:
        np.save(os.path.join(self.path, "state", "hamiltonianstatespace.npy"), state)
        if hash_ is not None:
            _write_json(os.path.join(self.path, "state", "hash.json"), {"fnv1a64": int(hash_)})
        with open(os.path.join(self.path, "state", "RNG.txt"), "w") as fh:
            fh.write(RNG_NAME + "\n")
        np.save(os.path.join(self.path, "state", "rngstate.npy"),
                np.array([seed & (2 ** 64 - 1), replica, sweep, cluster], np.uint64))

    def write_observables(self, series: dict) -> None:
        for name, values in series.items():
            np.save(os.path.join(self.path, "observables", f"{name}.npy"), np.asarray(values))

    def read_state(self):
        """(state, (seed, replica, sweep, cluster), hash or None) of a completed
        step; a file that cannot be read back whole raises MarqovError(CHECKSUM)."""
        from ._lib import ERR_CHECKSUM, MarqovError
        try:
            st = np.load(os.path.join(self.path, "state", "hamiltonianstatespace.npy"))
            rng = np.load(os.path.join(self.path, "state", "rngstate.npy"))
            if rng.shape != (4,):
                raise ValueError(f"RNG state of shape {rng.shape}")
        except (OSError, ValueError, EOFError) as exc:
            raise MarqovError(ERR_CHECKSUM, f"{self.path}: unreadable state ({exc})") from exc
        h = None
        hp = os.path.join(self.path, "state", "hash.json")
        if os.path.exists(hp):
            with open(hp) as fh:
                h = int(json.load(fh)["fnv1a64"])
        return st, tuple(int(x) for x in rng), h

    def read_observables(self) -> dict:
        d = os.path.join(self.path, "observables")
        return {f[:-4]: np.load(os.path.join(d, f)) for f in sorted(os.listdir(d)) if f.endswith(".npy")}

    @property
    def complete(self) -> bool:
        return os.path.exists(os.path.join(self.path, "state", "rngstate.npy"))
