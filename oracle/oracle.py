"""ctypes wrapper of the CPU oracle -- TEST INFRASTRUCTURE.

Loaded only by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline
leg, as the checker.  The engine (package ``marqov_b200``) never imports it.

``Oracle`` wraps the C restatement (oracle/liboracle.so); ``RefHarness`` wraps
the reference's own templates driven by oracle/ref_harness.cpp
(oracle/_ref/libmarqov_ref.so), present where it was built.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

ISING, ISING_EMBED, POTTS, BLUME_CAPEL, EA, HEISENBERG, PHI4, XXZ = range(1, 9)

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")


class OrcModel(C.Structure):
    _fields_ = [("kind", C.c_int), ("q", C.c_int), ("proposal", C.c_int), ("J", C.c_double),
                ("h", C.c_double), ("h2", C.c_double), ("k", C.c_double),
                ("delta", C.c_double), ("cap", C.c_double), ("termsel", C.c_int)]


class OrcLattice(C.Structure):
    _fields_ = [("n", C.c_int32), ("row_ptr", C.c_void_p), ("col_idx", C.c_void_p),
                ("bonds", C.c_void_p), ("ncolours", C.c_int32), ("colour_ptr", C.c_void_p),
                ("order", C.c_void_p)]


class OrcObs(C.Structure):
    _fields_ = [("e", C.c_double), ("m", C.c_double), ("m2", C.c_double), ("m4", C.c_double)]


def _load(path: str) -> C.CDLL:
    if not os.path.exists(path):
        from . import build as _b  # noqa: F401  (package-relative when imported as oracle.oracle)
    return C.CDLL(path)


def load_oracle() -> C.CDLL:
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        import importlib.util
        spec = importlib.util.spec_from_file_location("_oracle_build", os.path.join(HERE, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build_oracle()
    lib = C.CDLL(path)
    lib.orc_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
    lib.orc_draw.restype = C.c_uint64
    lib.orc_draw.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
    lib.orc_draw_c2.restype = C.c_uint64
    lib.orc_draw_c2.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
    lib.orc_accept_word.restype = C.c_uint64
    lib.orc_accept_word.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
    lib.orc_exp2app6.restype = C.c_double
    lib.orc_exp2app6.argtypes = [C.c_double]
    lib.orc_update_accepted.restype = C.c_int
    lib.orc_update_accepted.argtypes = [C.c_int, C.c_double, C.c_double, C.c_uint64]
    lib.orc_accept_threshold.restype = C.c_uint64
    lib.orc_accept_threshold.argtypes = [C.c_int, C.c_double, C.c_double]
    lib.orc_sweep_int8.argtypes = [C.POINTER(OrcModel), C.POINTER(OrcLattice), _i8p, C.c_double,
                                   C.c_uint64, C.c_uint32, C.c_uint32]
    lib.orc_sweep_f32.argtypes = [C.POINTER(OrcModel), C.POINTER(OrcLattice), _f32p, C.c_int,
                                  C.c_double, C.c_uint64, C.c_uint32, C.c_uint32]
    lib.orc_ising2d_sweep.argtypes = [C.c_int32, C.c_double, _i8p, C.c_double, C.c_uint64, C.c_uint32,
                                      C.c_uint32]
    lib.orc_init_int8.argtypes = [C.POINTER(OrcModel), C.c_int32, _i8p, C.c_uint64, C.c_uint32]
    lib.orc_init_f32.argtypes = [C.POINTER(OrcModel), C.c_int32, _f32p, C.c_int, C.c_uint64,
                                 C.c_uint32]
    lib.orc_wolff_int8.restype = C.c_int32
    lib.orc_wolff_int8.argtypes = [C.POINTER(OrcModel), C.POINTER(OrcLattice), _i8p, C.c_double,
                                   C.c_uint64, C.c_uint32, C.c_uint32, _i32p]
    lib.orc_wolff_f32.restype = C.c_int32
    lib.orc_wolff_f32.argtypes = [C.POINTER(OrcModel), C.POINTER(OrcLattice), _f32p, C.c_int,
                                  C.c_double, C.c_uint64, C.c_uint32, C.c_uint32, _i32p]
    lib.orc_measure_int8.argtypes = [C.POINTER(OrcModel), C.POINTER(OrcLattice), _i8p,
                                     C.POINTER(OrcObs)]
    lib.orc_measure_f32.argtypes = [C.POINTER(OrcModel), C.POINTER(OrcLattice), _f32p, C.c_int,
                                    C.POINTER(OrcObs)]
    lib.orc_hypercubic_csr.argtypes = [C.c_int, C.c_int, _i32p, _i32p]
    lib.orc_parity_colours.argtypes = [C.c_int, C.c_int, _i32p, _i32p]
    lib.orc_mt19937_64_words.argtypes = [C.c_uint64, C.c_int64, _u64p]
    lib.orc_metro_exp.restype = C.c_int64
    lib.orc_metro_exp.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_void_p]
    return lib


class Graph:
    """CSR neighbour structure + colour classes, kept alive for ctypes."""

    def __init__(self, row_ptr, col_idx, colour_ptr, order, bonds=None):
        self.row_ptr = np.ascontiguousarray(row_ptr, np.int32)
        self.col_idx = np.ascontiguousarray(col_idx, np.int32)
        self.colour_ptr = np.ascontiguousarray(colour_ptr, np.int32)
        self.order = np.ascontiguousarray(order, np.int32)
        self.bonds = None if bonds is None else np.ascontiguousarray(bonds, np.int8)
        self.n = len(self.row_ptr) - 1
        self.c = OrcLattice(self.n, self.row_ptr.ctypes.data, self.col_idx.ctypes.data,
                            None if self.bonds is None else self.bonds.ctypes.data,
                            len(self.colour_ptr) - 1, self.colour_ptr.ctypes.data,
                            self.order.ctypes.data)


class Oracle:
    def __init__(self):
        self.lib = load_oracle()

    # -- lattices
    def hypercubic(self, dim: int, length: int, bonds=None) -> Graph:
        n = length ** dim
        rp = np.zeros(n + 1, np.int32)
        ci = np.zeros(n * 2 * dim, np.int32)
        self.lib.orc_hypercubic_csr(dim, length, rp, ci)
        cp = np.zeros(3, np.int32)
        order = np.zeros(n, np.int32)
        self.lib.orc_parity_colours(dim, length, cp, order)
        return Graph(rp, ci, cp, order, bonds)

    # -- rng / acceptance
    def philox(self, ctr, key):
        out = np.zeros(4, np.uint32)
        self.lib.orc_philox4x32_10(np.asarray(ctr, np.uint32), np.asarray(key, np.uint32), out)
        return out

    def draw(self, seed, replica, stream, c0, c1, k):
        return self.lib.orc_draw(seed, replica, stream, c0, c1, k)

    def update_accepted(self, pref, dE, beta, word):
        return bool(self.lib.orc_update_accepted(pref, dE, beta, word))

    def accept_word(self, seed, replica, site, sweep):
        return int(self.lib.orc_accept_word(seed, replica, site, sweep))

    def threshold(self, pref, dE, beta):
        return int(self.lib.orc_accept_threshold(pref, dE, beta))

    # -- sweeps
    def sweep_int8(self, model: OrcModel, g: Graph, s, beta, seed, replica, sweep):
        self.lib.orc_sweep_int8(C.byref(model), C.byref(g.c), s, beta, seed, replica, sweep)

    def sweep_f32(self, model: OrcModel, g: Graph, s, symd, beta, seed, replica, sweep):
        self.lib.orc_sweep_f32(C.byref(model), C.byref(g.c), s, symd, beta, seed, replica, sweep)

    def ising2d_sweep(self, L, J, s, beta, seed, replica, sweep):
        self.lib.orc_ising2d_sweep(L, J, s, beta, seed, replica, sweep)

    def init_int8(self, model, n, seed, replica):
        s = np.zeros(n, np.int8)
        self.lib.orc_init_int8(C.byref(model), n, s, seed, replica)
        return s

    def init_f32(self, model, n, symd, seed, replica):
        s = np.zeros(n * symd, np.float32)
        self.lib.orc_init_f32(C.byref(model), n, s, symd, seed, replica)
        return s

    def wolff_int8(self, model, g: Graph, s, beta, seed, replica, serial):
        work = np.zeros(2 * g.n + 8, np.int32)
        return int(self.lib.orc_wolff_int8(C.byref(model), C.byref(g.c), s, beta, seed, replica,
                                           serial, work))

    def wolff_f32(self, model, g: Graph, s, symd, beta, seed, replica, serial):
        work = np.zeros(3 * g.n + 8, np.int32)
        return int(self.lib.orc_wolff_f32(C.byref(model), C.byref(g.c), s, symd, beta, seed,
                                          replica, serial, work))

    def measure_int8(self, model, g: Graph, s):
        o = OrcObs()
        self.lib.orc_measure_int8(C.byref(model), C.byref(g.c), s, C.byref(o))
        return o.e, o.m, o.m2, o.m4

    def measure_f32(self, model, g: Graph, s, symd):
        o = OrcObs()
        self.lib.orc_measure_f32(C.byref(model), C.byref(g.c), s, symd, C.byref(o))
        return o.e, o.m, o.m2, o.m4

    def mt_words(self, seed, n):
        out = np.zeros(n, np.uint64)
        self.lib.orc_mt19937_64_words(seed, n, out)
        return out

    def metro_exp(self, N, reps, beta, want_decisions=False):
        dec = np.zeros(N * reps, np.uint8) if want_decisions else None
        acc = self.lib.orc_metro_exp(N, reps, beta, None if dec is None else dec.ctypes.data)
        return int(acc), dec


# the AVX-512 subsets that -march=x86-64-v4 may use
_V4_FLAGS = {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"}


def host_has_v4() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return _V4_FLAGS <= set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return False


def ref_path() -> str:
    """The reference harness for this host: the x86-64-v4 (AVX-512) build
    where the CPU has it, else the x86-64-v3 one."""
    v4 = os.path.join(HERE, "_ref", "libmarqov_ref_v4.so")
    if host_has_v4() and os.path.exists(v4):
        return v4
    return os.path.join(HERE, "_ref", "libmarqov_ref.so")


def ref_march(path: str | None = None) -> str:
    return "x86-64-v4" if (path or ref_path()).endswith("_v4.so") else "x86-64-v3"


class RefHarness:
    """The reference's own templates (oracle/_ref)."""

    def __init__(self, path: str | None = None):
        path = path or ref_path()
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = C.CDLL(path)
        lib.ref_sweeps_int.restype = C.c_int
        lib.ref_sweeps_int.argtypes = [C.c_int, C.c_int, _i32p, _i32p, C.c_void_p, C.c_void_p, C.c_int, _i32p,
                                       _i32p, _i8p, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_uint64, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p]
        lib.ref_sweeps_f32.restype = C.c_int
        lib.ref_sweeps_f32.argtypes = [C.c_int, C.c_int, _i32p, _i32p, C.c_void_p, C.c_int, _i32p, _i32p, _f32p,
                                       C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_uint64, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p]
        lib.ref_wolff_int.restype = C.c_int
        lib.ref_wolff_int.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _i8p, C.c_double, C.c_double,
                                      C.c_uint64, C.c_uint32, C.c_uint32, C.c_int, _i32p]
        lib.ref_wolff_f32.restype = C.c_int
        lib.ref_wolff_f32.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f32p, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_uint64, C.c_uint32, C.c_uint32, C.c_int, _i32p]
        lib.ref_metro_exp.restype = C.c_longlong
        lib.ref_metro_exp.argtypes = [C.c_int, C.c_int, C.c_double, _f64p, C.c_void_p]
        lib.ref_metro_exp_plain.restype = C.c_longlong
        lib.ref_metro_exp_plain.argtypes = [C.c_int, C.c_int, C.c_double]
        lib.ref_mt_words.argtypes = [C.c_longlong, _u64p]
        lib.ref_update_accepted.restype = C.c_int
        lib.ref_update_accepted.argtypes = [C.c_int, C.c_double, C.c_double, C.c_uint64]
        lib.ref_init_int.restype = C.c_int
        lib.ref_init_int.argtypes = [C.c_int, C.c_int, C.c_uint64, C.c_uint32, _i8p]
        lib.ref_farm_create.restype = C.c_void_p
        lib.ref_farm_create.argtypes = [C.c_int, C.c_double, C.c_int, C.c_uint64]
        lib.ref_farm_step.restype = C.c_double
        lib.ref_farm_step.argtypes = [C.c_void_p, C.c_longlong]
        lib.ref_farm_magnetisation.restype = C.c_longlong
        lib.ref_farm_magnetisation.argtypes = [C.c_void_p, C.c_int]
        lib.ref_farm_destroy.argtypes = [C.c_void_p]
        lib.ref_emcs_ising2d.restype = C.c_int
        lib.ref_emcs_ising2d.argtypes = [C.c_int, C.c_double, C.c_double, C.c_uint64, C.c_int, C.c_int, C.c_int,
                                         C.c_int, _f64p, _f64p]
        lib.ref_emcs_generic.restype = C.c_int
        lib.ref_emcs_generic.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                         C.c_double, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, _f64p, _f64p]
        lib.ref_wolff_ising2d.restype = C.c_int
        lib.ref_wolff_ising2d.argtypes = [C.c_int, C.c_double, C.c_uint64, C.c_int, C.c_int, _f64p, _f64p]
        lib.ref_calc_mh_ratio.restype = C.c_double
        lib.ref_calc_mh_ratio.argtypes = [C.c_double]
        lib.ref_pt_calcprob.restype = C.c_int
        lib.ref_pt_calcprob.argtypes = [C.c_int, _f64p, _f64p, _f64p, _f64p, _f64p]
        lib.ref_save_geometry.restype = C.c_int
        lib.ref_save_geometry.argtypes = [C.c_int, _i32p, _i32p, C.c_int, _f64p, C.c_char_p]
        lib.ref_import_geometry.restype = C.c_int
        lib.ref_import_geometry.argtypes = [C.c_char_p, C.c_int] + [C.POINTER(C.c_int)] * 4 + [C.c_void_p] * 4
        self.lib = lib

    def save_geometry(self, row_ptr, col_idx, coords, path):
        """The reference's save_geometry over CSR arrays and [n, c] coordinates."""
        crd = np.ascontiguousarray(coords, np.float64)
        n = len(row_ptr) - 1
        nc = crd.shape[1] if crd.ndim == 2 else 0
        self.lib.ref_save_geometry(n, np.ascontiguousarray(row_ptr, np.int32), np.ascontiguousarray(col_idx, np.int32),
                                   nc, crd.reshape(-1) if crd.size else np.zeros(1), str(path).encode())

    def import_geometry(self, path, idxoffs=0):
        """GraphFromCSV / import_geometry: (row_ptr, col_idx, per-site coordinate
        lists, ncoords), or None where the reference throws."""
        n, nnz, nv, nc = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        p = str(path).encode()
        if self.lib.ref_import_geometry(p, idxoffs, C.byref(n), C.byref(nnz), C.byref(nv), C.byref(nc),
                                        None, None, None, None):
            return None
        rp = np.zeros(n.value + 1, np.int32)
        ci = np.zeros(max(nnz.value, 1), np.int32)
        cnt = np.zeros(max(n.value, 1), np.int32)
        crd = np.zeros(max(nv.value, 1), np.float64)
        self.lib.ref_import_geometry(p, idxoffs, C.byref(n), C.byref(nnz), C.byref(nv), C.byref(nc),
                                     rp.ctypes.data, ci.ctypes.data, cnt.ctypes.data, crd.ctypes.data)
        lists, o = [], 0
        for k in cnt[:n.value]:
            lists.append(crd[o:o + k].tolist())
            o += k
        return rp, ci[:nnz.value], lists, nc.value

    def calc_mh_ratio(self, en):
        return float(self.lib.ref_calc_mh_ratio(en))

    def pt_calcprob(self, beta_a, e_a, beta_b, e_b):
        """The reference scheduler's calcprob for arrays of (beta, total energy) pairs."""
        arrs = [np.ascontiguousarray(x, np.float64) for x in (beta_a, e_a, beta_b, e_b)]
        out = np.zeros(arrs[0].size, np.float64)
        rc = self.lib.ref_pt_calcprob(out.size, *arrs, out)
        if rc:
            raise RuntimeError(f"ref_pt_calcprob failed ({rc})")
        return out

    @staticmethod
    def _sub(sub):
        if sub is None:
            return None, None
        a = np.ascontiguousarray(sub, np.uint8)
        return a, a.ctypes.data

    def sweeps_int(self, kind, g: Graph, s, J, D, beta, seed, replica, sweep0, nsweeps, want_obs=True, D2=0.0,
                   sub=None):
        """Reference Metropolis sweeps in colour order; per sweep (e, m, e_obs):
        the energy the moves see, the magnetization and Energy<H> (ref_harness.cpp)."""
        obs = np.zeros(3 * nsweeps, np.float64) if want_obs else None
        bonds = None if g.bonds is None else g.bonds.ctypes.data
        keep, subp = self._sub(sub)
        rc = self.lib.ref_sweeps_int(kind, g.n, g.row_ptr, g.col_idx, bonds, subp, len(g.colour_ptr) - 1,
                                     g.colour_ptr, g.order, s, J, D, D2, beta, seed, replica, sweep0,
                                     nsweeps, None if obs is None else obs.ctypes.data)
        assert rc == 0
        return None if obs is None else obs.reshape(nsweeps, 3)

    def sweeps_f32(self, kind, g: Graph, s, J, p0, p1, cap, beta, seed, replica, sweep0, nsweeps,
                   want_obs=True, p2=0.0, sub=None):
        obs = np.zeros(3 * nsweeps, np.float64) if want_obs else None
        keep, subp = self._sub(sub)
        rc = self.lib.ref_sweeps_f32(kind, g.n, g.row_ptr, g.col_idx, subp, len(g.colour_ptr) - 1,
                                     g.colour_ptr, g.order, s, J, p0, p1, p2, cap, beta, seed, replica,
                                     sweep0, nsweeps, None if obs is None else obs.ctypes.data)
        assert rc == 0
        return None if obs is None else obs.reshape(nsweeps, 3)

    def wolff_int(self, kind, g: Graph, s, J, beta, seed, replica, serial0, nclusters):
        sizes = np.zeros(nclusters, np.int32)
        rc = self.lib.ref_wolff_int(kind, g.n, g.row_ptr, g.col_idx, s, J, beta, seed, replica,
                                    serial0, nclusters, sizes)
        assert rc == 0
        return sizes

    def wolff_f32(self, kind, g: Graph, s, J, p0, p1, beta, seed, replica, serial0, nclusters):
        """The reference's generic Wolff with Embedder<Heisenberg> (kind 6) or the
        scalar Embedder<Phi4> (kind 8), sequential draws; s updated in place."""
        sizes = np.zeros(nclusters, np.int32)
        rc = self.lib.ref_wolff_f32(kind, g.n, g.row_ptr, g.col_idx, s, J, p0, p1, beta, seed, replica, serial0,
                                    nclusters, sizes)
        assert rc == 0
        return sizes

    def update_accepted(self, pref, dE, beta, word):
        return bool(self.lib.ref_update_accepted(pref, dE, beta, word))

    def init_int(self, kind, n, seed, replica):
        out = np.zeros(n, np.int8)
        assert self.lib.ref_init_int(kind, n, seed, replica, out) == 0
        return out

    def metro_exp(self, N, reps, beta, want_decisions=False):
        dE = np.zeros(N, np.float64)
        dec = np.zeros(N * reps, np.uint8) if want_decisions else None
        acc = self.lib.ref_metro_exp(N, reps, beta, dE, None if dec is None else dec.ctypes.data)
        return int(acc), dec

    def metro_exp_plain(self, N, reps, beta):
        return int(self.lib.ref_metro_exp_plain(N, reps, beta))

    def mt_words(self, n):
        out = np.zeros(n, np.uint64)
        self.lib.ref_mt_words(n, out)
        return out

    def emcs_ising2d(self, L, J, beta, seed, ncluster, nmetro, ntherm, nmeas):
        """The reference's own EMCS loop (random-site order, mt19937_64):
        per measured EMCS (E, |m|) and mean cluster size."""
        obs = np.zeros(2 * nmeas, np.float64)
        mc = np.zeros(nmeas, np.float64)
        assert self.lib.ref_emcs_ising2d(L, J, beta, seed, ncluster, nmetro, ntherm, nmeas, obs, mc) == 0
        return obs.reshape(nmeas, 2), mc

    def emcs_generic(self, kind, L, dim, J, beta, seed, ncluster, nmetro, ntherm, nmeas, p0=0.0, p1=0.0, p2=0.0):
        """The reference's own EMCS loop for Potts<3> (kind 3), Heisenberg with
        the plane embedder (6) or scalar phi^4 (8): per measured EMCS (e, |m|)
        and the mean cluster size."""
        obs = np.zeros(2 * nmeas, np.float64)
        mc = np.zeros(nmeas, np.float64)
        assert self.lib.ref_emcs_generic(kind, L, dim, J, p0, p1, p2, beta, seed, ncluster, nmetro, ntherm, nmeas,
                                         obs, mc) == 0
        return obs.reshape(nmeas, 2), mc

    def wolff_ising2d_timed(self, L, beta, seed, ntherm, nclusters):
        """The reference's Wolff<Ising<int>> on one core: (seconds, summed
        cluster size) of nclusters clusters after ntherm EMCS."""
        t = np.zeros(1)
        tot = np.zeros(1)
        assert self.lib.ref_wolff_ising2d(L, beta, seed, ntherm, nclusters, t, tot) == 0
        return float(t[0]), float(tot[0])

    def farm(self, length, beta, nthreads, seed=12345):
        return RefFarm(self.lib, length, beta, nthreads, seed)


class RefFarm:
    """nthreads independent 2D Ising replicas stepped by the reference's own
    random-site Metropolis loop (one replica per thread)."""

    def __init__(self, lib, length, beta, nthreads, seed):
        self.lib = lib
        self.nthreads = nthreads
        self.n = length * length
        self.h = lib.ref_farm_create(length, beta, nthreads, seed)

    def step(self, nupdates):
        return float(self.lib.ref_farm_step(self.h, nupdates))

    def magnetisation(self, t=0):
        return int(self.lib.ref_farm_magnetisation(self.h, t))

    def close(self):
        if self.h:
            self.lib.ref_farm_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
