"""GPU simulation core mirroring ``MARQOV::Core`` (src/libmarqov/core.h:372-1167).

``makeCore(lattice, config, ham, beta)`` plays the part of
``makeCore<L,H>(std::tuple<L&, Config, std::tuple<beta, HArgs...>>)``
(core.h:1223-1246); ``Core`` exposes ``init``, ``wrmploop``, ``gameloop`` and
``elementaryMCstep`` (core.h:829-834, 1001-1050; emcs.h:111-119) over one
engine handle.  The state lives on the GPU; observables come back per EMCS.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .hamiltonians import Hamiltonian
from .lattices import Lattice


def _resident_flag(config) -> int:
    """Run flags of Config.resident: None (engine's choice), True, False."""
    if config.resident is None:
        return 0
    return L.FLAG_RESIDENT if config.resident else L.FLAG_NO_RESIDENT


@dataclass
class Config:
    """``MARQOV::Config`` (core.h:74-192): method parameters."""
    outpath: str = ""   # with outname: the dump container outpath + outname + ".mqv" (none if empty)
    outname: str = ""
    id: int = 0
    repid: int = 0
    seed: int = 0
    nsteps: int = 250
    warmupsteps: int = 100
    gameloopsteps: int = 200
    ncluster: int = 20
    nmetro: int = 10
    device: int = 0
    # force one launch per colour class (no fused two-colour tiles)
    per_colour: bool = False
    # int8 stencil lattices of <= 65536 sites (one CTA) or <= 262144 sites (a
    # thread-block cluster) can run whole chunks of EMCS in shared memory.
    # None: the engine decides (single handles up to 16384 sites; batch
    # members take the batch's graph path); True: wherever the lattice fits;
    # False: never (launch per step).  The results are the same.
    resident: bool | None = None

    def setid(self, i):
        self.id = i
        return self

    def setrepid(self, r):
        self.repid = r
        return self

    def setseed(self, s):
        self.seed = s
        return self

    def setwarmupsteps(self, w):
        self.warmupsteps = w
        return self

    def setgameloopsteps(self, g):
        self.gameloopsteps = g
        return self

    def setncluster(self, n):
        self.ncluster = n
        return self

    def setnmetro(self, n):
        self.nmetro = n
        return self


@dataclass
class TimeSeries:
    e: list = field(default_factory=list)
    m: list = field(default_factory=list)
    m2: list = field(default_factory=list)
    m4: list = field(default_factory=list)
    clustersize: list = field(default_factory=list)

    def arrays(self):
        return {k: np.asarray(v) for k, v in vars(self).items()}


class Core:
    def __init__(self, lattice: Lattice, config: Config, ham: Hamiltonian, beta: float):
        lib = L.load()
        self.lattice = lattice
        self.config = config
        self.ham = ham
        self.beta = float(beta)
        self._lib = lib
        self._h = C.c_void_p()
        self._owner = None
        self._setup(lattice, ham)
        # the dump container (Core's constructor, src/libmarqov/core.h:469-488):
        # a new step, continuing from the previous step's final state and RNG
        seed, replica, restore, prev = int(config.seed), int(config.repid), None, -1
        if config.outpath:
            from . import checkpoint as CP
            path = CP.container_path(config)
            prev = CP.last_step(path)
            if prev >= 0:
                last = CP.Step(path, prev)
                if not last.complete:
                    raise RuntimeError(f"{last.path} holds no final state (its run did not end)")
                restore = last.read_state()
                seed, replica = restore[1][0], restore[1][1]
        md = ham.desc(self.beta)
        ld = lattice.desc()
        rp = L.RunParams(beta=self.beta, seed=seed & (2 ** 64 - 1), replica=replica, device=int(config.device),
                         flags=(L.FLAG_PER_COLOUR if config.per_colour else 0) | _resident_flag(config))
        L.check(lib.mqv_create(C.byref(md), C.byref(ld), C.byref(rp), C.byref(self._h)))
        self._seed, self._replica = seed, replica
        if restore is not None:
            if restore[2] is None:
                self.state = restore[0]
            else:
                self.set_state_checked(restore[0], restore[2])
            self.counters = restore[1][2:]
            self._restored = True
        # the step group exists only for a Core that could be set up
        if config.outpath:
            self._step = CP.Step(path, prev + 1).create(self.beta, config, lattice, ham, L.version())

    def _setup(self, lattice: Lattice, ham: Hamiltonian):
        self._step = None
        self._restored = False
        self.n = int(lattice.size())
        self.symd = ham.SymD
        self.dtype = ham.dtype
        self.obs = TimeSeries()
        self.step = 0

    @classmethod
    def _member(cls, handle: C.c_void_p, owner, lattice: Lattice, config: Config, ham: Hamiltonian,
                beta: float) -> "Core":
        """A view of a handle owned by `owner` (a Batch member)."""
        c = cls.__new__(cls)
        c._lib = L.load()
        c.lattice, c.config, c.ham, c.beta = lattice, config, ham, float(beta)
        c._h = handle
        c._owner = owner
        c._setup(lattice, ham)
        return c

    # -- lifecycle
    def dump(self):
        """Write the step's observable time series and final state (what
        ~Core writes, src/libmarqov/core.h:876-902); close() calls it."""
        if self._step is None or not self._h:
            return
        self._step.write_observables(self.obs.arrays())
        sweep, cluster = self.counters
        st, h = self.get_state_checked()
        self._step.write_state(st, self._seed, self._replica, sweep, cluster, h)

    def close(self):
        if self._h and self._owner is None:
            try:
                self.dump()
            finally:
                self._lib.mqv_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- reference Core API
    def init(self):
        """Random initial state (Core::init -> initstatespace); a Core that
        continues a dump keeps the state it read (core.h:829-834)."""
        if self._restored:
            return
        L.check(self._lib.mqv_init_state(self._h))

    def elementaryMCstep(self) -> float:
        """One EMCS (emcs.h:69-109); returns the mean cluster size."""
        mc = np.zeros(1, np.float64)
        L.check(self._lib.mqv_emcs(self._h, 1, self.config.ncluster, self.config.nmetro, None,
                                   mc.ctypes.data))
        return float(mc[0])

    def wrmploop(self):
        """warmupsteps EMCS without measurements (core.h:1034-1050)."""
        n = 10 * (self.config.warmupsteps // 10)
        self.emcs(n, measure=False)

    def gameloop(self):
        """gameloopsteps EMCS, measuring after each (core.h:1001-1028)."""
        n = 10 * (self.config.gameloopsteps // 10)
        obs, mc = self.emcs(n, measure=True)
        self.obs.e.extend(obs[:, 0].tolist())
        self.obs.m.extend(obs[:, 1].tolist())
        self.obs.m2.extend(obs[:, 2].tolist())
        self.obs.m4.extend(obs[:, 3].tolist())
        self.obs.clustersize.extend(mc.tolist())
        return obs

    # -- engine calls
    def emcs(self, n: int, ncluster: int | None = None, nmetro: int | None = None, measure: bool = True):
        nc = self.config.ncluster if ncluster is None else ncluster
        nm = self.config.nmetro if nmetro is None else nmetro
        obs = np.zeros((n, 4), np.float64) if measure else None
        mc = np.zeros(n, np.float64) if measure else None
        L.check(self._lib.mqv_emcs(self._h, n, nc, nm, None if obs is None else obs.ctypes.data,
                                   None if mc is None else mc.ctypes.data))
        self.step += n
        return obs, mc

    def metropolis(self, nsweeps: int):
        L.check(self._lib.mqv_metropolis(self._h, int(nsweeps)))

    def wolff(self, nclusters: int) -> np.ndarray:
        sizes = np.zeros(nclusters, np.int32)
        L.check(self._lib.mqv_wolff(self._h, int(nclusters), sizes.ctypes.data))
        return sizes

    def set_wolff(self, algorithm: str):
        """Cluster algorithm of this lattice: "auto" (labelling for int8 lattices
        of >= 2^18 sites), "bfs" or "label"; the clusters are the same."""
        code = {"auto": L.WOLFF_AUTO, "bfs": L.WOLFF_BFS, "label": L.WOLFF_LABEL}[algorithm]
        L.check(self._lib.mqv_set_wolff(self._h, code))

    def measure(self) -> tuple[float, float, float, float]:
        o = L.Obs()
        L.check(self._lib.mqv_measure(self._h, C.byref(o)))
        return o.e, o.m, o.m2, o.m4

    def synchronize(self):
        L.check(self._lib.mqv_synchronize(self._h))

    def set_beta(self, beta: float):
        self.beta = float(beta)
        L.check(self._lib.mqv_set_beta(self._h, self.beta))

    def set_model(self, ham: Hamiltonian):
        """Replace the model coefficients (same model kind), e.g. a new
        proposal width."""
        L.check(self._lib.mqv_set_model(self._h, C.byref(ham.desc(self.beta))))
        self.ham = ham

    def set_stream(self, stream_ptr: int):
        L.check(self._lib.mqv_set_stream(self._h, C.c_void_p(stream_ptr)))

    @property
    def state(self) -> np.ndarray:
        out = np.empty(self.n * self.symd, self.dtype)
        L.check(self._lib.mqv_get_state(self._h, out.ctypes.data, out.nbytes))
        return out

    @state.setter
    def state(self, value):
        v = np.ascontiguousarray(value, self.dtype).reshape(-1)
        L.check(self._lib.mqv_set_state(self._h, v.ctypes.data, v.nbytes))

    def get_state_checked(self) -> tuple[np.ndarray, int]:
        """The state and its FNV-1a 64-bit hash (mqv_get_state_checked)."""
        out = np.empty(self.n * self.symd, self.dtype)
        h = C.c_uint64()
        L.check(self._lib.mqv_get_state_checked(self._h, out.ctypes.data, out.nbytes, C.byref(h)))
        return out, int(h.value)

    def set_state_checked(self, value, hash_: int):
        """Set the state if its hash matches (else MarqovError CHECKSUM, state untouched)."""
        v = np.ascontiguousarray(value, self.dtype).reshape(-1)
        L.check(self._lib.mqv_set_state_checked(self._h, v.ctypes.data, v.nbytes, int(hash_) & (2 ** 64 - 1)))

    def state_device_ptr(self) -> tuple[int, int]:
        p = C.c_void_p()
        nb = C.c_size_t()
        L.check(self._lib.mqv_state_device_ptr(self._h, C.byref(p), C.byref(nb)))
        return int(p.value or 0), int(nb.value)

    @property
    def counters(self) -> tuple[int, int]:
        a, b = C.c_uint64(), C.c_uint64()
        L.check(self._lib.mqv_get_counters(self._h, C.byref(a), C.byref(b)))
        return int(a.value), int(b.value)

    @counters.setter
    def counters(self, v):
        L.check(self._lib.mqv_set_counters(self._h, int(v[0]), int(v[1])))

    def describe(self) -> str:
        buf = C.create_string_buffer(256)
        L.check(self._lib.mqv_describe(self._h, buf, len(buf)))
        return buf.value.decode()

    @property
    def launches(self) -> int:
        c = C.c_uint64()
        L.check(self._lib.mqv_launch_count(self._h, C.byref(c)))
        return int(c.value)


def makeCore(lattice: Lattice, config: Config, ham: Hamiltonian, beta: float) -> Core:
    """``MARQOV::makeCore`` (core.h:1223-1246)."""
    return Core(lattice, config, ham, beta)


class Batch:
    """Many independent simulations advanced together on one GPU.

    The farm MARQOV's scheduler runs as one ``Core`` per thread
    (src/libmarqov/marqovscheduler.h:64-494) becomes batched kernels per EMCS
    replayed from a CUDA graph; every member sees exactly the states and
    observables it would have on its own.  ``members`` lists
    ``(lattice, config, hamiltonian, beta)``; int8 models on hypercubic
    lattices.
    """

    def __init__(self, members, graph_steps: int = 8):
        lib = L.load()
        self._lib = lib
        self._h = C.c_void_p()
        specs = (L.SimSpec * len(members))()
        self._members_args = list(members)
        for i, (lat, cfg, ham, beta) in enumerate(members):
            specs[i].model = ham.desc(float(beta))
            specs[i].lattice = lat.desc()
            specs[i].params = L.RunParams(beta=float(beta), seed=int(cfg.seed) & (2 ** 64 - 1),
                                          replica=int(cfg.repid), device=int(cfg.device),
                                          flags=_resident_flag(cfg))
        L.check(lib.mqv_batch_create(specs, len(members), C.byref(self._h)))
        L.check(lib.mqv_batch_set_graph_steps(self._h, int(graph_steps)))
        self.n = len(members)
        self._pt_steps = 0
        self._views = []
        for i, (lat, cfg, ham, beta) in enumerate(members):
            m = C.c_void_p()
            L.check(lib.mqv_batch_member(self._h, i, C.byref(m)))
            self._views.append(Core._member(m, self, lat, cfg, ham, beta))

    def close(self):
        if self._h:
            for v in self._views:
                v._h = C.c_void_p()
            self._lib.mqv_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return self.n

    def member(self, i: int) -> Core:
        return self._views[i]

    def init(self):
        L.check(self._lib.mqv_batch_init_state(self._h))

    def set_wolff(self, algorithm: str):
        """Cluster algorithm, "bfs" (one CTA per member grows its cluster),
        "label" (connected-component labelling of all members) or "auto" (the
        default: the faster of the two, timed on the first run with
        clusters); all give the same clusters."""
        code = {"auto": L.WOLFF_AUTO, "bfs": L.WOLFF_BFS, "label": L.WOLFF_LABEL}[algorithm]
        L.check(self._lib.mqv_batch_set_wolff(self._h, code))

    @property
    def wolff(self) -> str:
        """The cluster algorithm in use ("auto" until it has been timed)."""
        v = C.c_int32()
        L.check(self._lib.mqv_batch_get_wolff(self._h, C.byref(v)))
        return {L.WOLFF_AUTO: "auto", L.WOLFF_BFS: "bfs", L.WOLFF_LABEL: "label"}[v.value]

    def emcs(self, n: int, ncluster: int = 1, nmetro: int = 1):
        """n EMCS of every member; returns (obs [n, members, 4], mean cluster [n, members])."""
        obs = np.zeros((n, self.n, 4), np.float64)
        mc = np.zeros((n, self.n), np.float64)
        L.check(self._lib.mqv_batch_emcs(self._h, int(n), int(ncluster), int(nmetro), obs.ctypes.data, mc.ctypes.data))
        return obs, mc

    def tempering(self, n_steps: int, emcs_per_step: int = 1, ncluster: int = 1, nmetro: int = 1, plan=None,
                  seed: int = 0):
        """Replica exchange: n_steps x (emcs_per_step EMCS of every member,
        then exchange attempts between the step's member pairs).  plan: int
        [n_steps, pairs, 2] (default: alternating neighbours in member order,
        ``tempering.neighbour_plan``).  Returns (obs [n_steps * emcs_per_step,
        members, 4], accepted [n_steps, pairs]: 1 exchanged, 0 rejected, -1
        self pair)."""
        from .tempering import neighbour_plan
        if plan is None:
            plan = neighbour_plan(self.n, n_steps, first=self._pt_steps)
        plan = np.ascontiguousarray(plan, np.int32)
        if plan.ndim != 3 or plan.shape[0] != n_steps or plan.shape[2] != 2:
            raise ValueError("plan must have shape [n_steps, pairs, 2]")
        obs = np.zeros((n_steps * emcs_per_step, self.n, 4), np.float64)
        acc = np.zeros((n_steps, plan.shape[1]), np.int32)
        L.check(self._lib.mqv_batch_tempering(self._h, int(n_steps), int(emcs_per_step), int(ncluster), int(nmetro),
                                              plan.ctypes.data, int(plan.shape[1]), int(seed) & (2 ** 64 - 1),
                                              obs.ctypes.data, acc.ctypes.data))
        self._pt_steps += n_steps
        return obs, acc

    @property
    def launches(self) -> int:
        c = C.c_uint64()
        L.check(self._lib.mqv_batch_launch_count(self._h, C.byref(c)))
        return int(c.value)


def tune_small_cap(core: Core, target: float = 0.5, iters: int = 10, sweeps: int = 1) -> float:
    """Tune the small-cap proposal of an O(3) model to a Metropolis acceptance
    rate near `target` by bisection on cap = cos(half-angle) during
    thermalisation; returns the frozen cap (also set on the core).

    The acceptance rate of a sweep is measured as the fraction of sites whose
    spin changed (an accepted cap move always changes the spin).  This tuning
    has no counterpart in the reference, which draws fresh directions."""
    import copy
    lo, hi = -1.0, 0.9999
    ham = copy.copy(core.ham)
    ham.proposal = "smallcap"
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        ham.cap = mid
        core.set_model(ham)
        before = core.state.reshape(-1, core.symd)
        core.metropolis(sweeps)
        after = core.state.reshape(-1, core.symd)
        acc = float(np.mean(np.any(before != after, axis=1))) ** (1.0 / sweeps)
        if acc < target:
            lo = mid  # too few accepted: narrower cone (larger cap)
        else:
            hi = mid
    ham.cap = 0.5 * (lo + hi)
    core.set_model(ham)
    return ham.cap
