"""ctypes binding of the engine's C ABI (include/marqov_b200.h).

The library is loaded from the package directory (built in-tree by
``marqov_b200/build.py``).  There is no fallback: if the library is missing or
fails to load, importing the engine raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmarqov_b200.so")

# status codes
OK = 0
ERR_INVALID_ARG = 1
ERR_UNSUPPORTED_TERM = 2
ERR_BAD_DESCRIPTOR = 3
ERR_CUDA = 4
ERR_TIMEOUT = 5
ERR_CHECKSUM = 6
ERR_NO_DEVICE = 7
ERR_OUT_OF_MEMORY = 8
ERR_STATE = 9

STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "UNSUPPORTED_TERM", 3: "BAD_DESCRIPTOR", 4: "CUDA",
                5: "TIMEOUT", 6: "CHECKSUM", 7: "NO_DEVICE", 8: "OUT_OF_MEMORY", 9: "STATE"}

MODEL_ISING, MODEL_ISING_EMBED, MODEL_POTTS, MODEL_BLUME_CAPEL, MODEL_EA, MODEL_HEISENBERG, \
    MODEL_PHI4, MODEL_XXZ = range(1, 9)
PROPOSAL_DEFAULT, PROPOSAL_SMALL_CAP = 0, 1
LATTICE_HYPERCUBIC, LATTICE_CSR, LATTICE_BIPARTITE = 1, 2, 3
FLAG_PER_COLOUR = 1
FLAG_NO_RESIDENT = 2
FLAG_RESIDENT = 4
WOLFF_AUTO, WOLFF_BFS, WOLFF_LABEL = 0, 1, 2


class ModelDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("q", C.c_int32), ("proposal", C.c_int32),
                ("reserved", C.c_int32), ("J", C.c_double), ("h", C.c_double),
                ("h2", C.c_double), ("k", C.c_double), ("delta", C.c_double),
                ("cap", C.c_double)]


class LatticeDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("dim", C.c_int32), ("len", C.c_int32), ("n", C.c_int32),
                ("row_ptr", C.c_void_p), ("col_idx", C.c_void_p), ("bonds", C.c_void_p),
                ("colours", C.c_void_p)]


class RunParams(C.Structure):
    _fields_ = [("beta", C.c_double), ("seed", C.c_uint64), ("replica", C.c_uint32),
                ("device", C.c_int32), ("flags", C.c_uint32), ("reserved", C.c_uint32)]


class Obs(C.Structure):
    _fields_ = [("e", C.c_double), ("m", C.c_double), ("m2", C.c_double), ("m4", C.c_double)]


class SimSpec(C.Structure):
    _fields_ = [("model", ModelDesc), ("lattice", LatticeDesc), ("params", RunParams)]


class MarqovError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[marqov_b200] {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


# Every exported symbol with its signature (restype, argtypes).
_vp = C.c_void_p
SIGNATURES = {
    "mqv_version": (C.c_char_p, []),
    "mqv_device_count": (C.c_int32, [C.POINTER(C.c_int32)]),
    "mqv_last_error": (C.c_int32, [C.c_char_p, C.c_size_t]),
    "mqv_create": (C.c_int32, [C.POINTER(ModelDesc), C.POINTER(LatticeDesc), C.POINTER(RunParams),
                               C.POINTER(_vp)]),
    "mqv_destroy": (C.c_int32, [_vp]),
    "mqv_set_wolff": (C.c_int32, [_vp, C.c_int32]),
    "mqv_get_state_checked": (C.c_int32, [_vp, _vp, C.c_size_t, C.POINTER(C.c_uint64)]),
    "mqv_set_state_checked": (C.c_int32, [_vp, _vp, C.c_size_t, C.c_uint64]),
    "mqv_selftest_inject_timeout": (C.c_int32, [_vp, C.c_int32, C.c_uint64]),
    "mqv_set_stream": (C.c_int32, [_vp, _vp]),
    "mqv_get_stream": (C.c_int32, [_vp, C.POINTER(_vp)]),
    "mqv_set_beta": (C.c_int32, [_vp, C.c_double]),
    "mqv_set_model": (C.c_int32, [_vp, C.POINTER(ModelDesc)]),
    "mqv_init_state": (C.c_int32, [_vp]),
    "mqv_get_state": (C.c_int32, [_vp, _vp, C.c_size_t]),
    "mqv_set_state": (C.c_int32, [_vp, _vp, C.c_size_t]),
    "mqv_state_device_ptr": (C.c_int32, [_vp, C.POINTER(_vp), C.POINTER(C.c_size_t)]),
    "mqv_state_bytes": (C.c_int32, [_vp, C.POINTER(C.c_size_t)]),
    "mqv_get_counters": (C.c_int32, [_vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "mqv_set_counters": (C.c_int32, [_vp, C.c_uint64, C.c_uint64]),
    "mqv_metropolis": (C.c_int32, [_vp, C.c_int32]),
    "mqv_wolff": (C.c_int32, [_vp, C.c_int32, _vp]),
    "mqv_wolff_noalloc": (C.c_int32, [_vp, C.c_int32, _vp]),
    "mqv_emcs": (C.c_int32, [_vp, C.c_int32, C.c_int32, C.c_int32, _vp, _vp]),
    "mqv_measure": (C.c_int32, [_vp, C.POINTER(Obs)]),
    "mqv_emcs_samples": (C.c_int32, [_vp, C.c_int32, C.c_int32, C.c_int32, _vp]),
    "mqv_phi4_fdt": (C.c_int32, [_vp, C.c_int32, C.c_int32, C.c_int64, C.c_double, _vp, _vp, _vp, _vp, _vp, _vp,
                                 _vp]),
    "mqv_synchronize": (C.c_int32, [_vp]),
    "mqv_launch_count": (C.c_int32, [_vp, C.POINTER(C.c_uint64)]),
    "mqv_describe": (C.c_int32, [_vp, C.c_char_p, C.c_size_t]),
    "mqv_batch_create": (C.c_int32, [C.POINTER(SimSpec), C.c_int32, C.POINTER(_vp)]),
    "mqv_batch_destroy": (C.c_int32, [_vp]),
    "mqv_batch_member": (C.c_int32, [_vp, C.c_int32, C.POINTER(_vp)]),
    "mqv_batch_init_state": (C.c_int32, [_vp]),
    "mqv_batch_set_graph_steps": (C.c_int32, [_vp, C.c_int32]),
    "mqv_batch_set_wolff": (C.c_int32, [_vp, C.c_int32]),
    "mqv_batch_get_wolff": (C.c_int32, [_vp, C.POINTER(C.c_int32)]),
    "mqv_batch_emcs": (C.c_int32, [_vp, C.c_int32, C.c_int32, C.c_int32, _vp, _vp]),
    "mqv_batch_emcs_samples": (C.c_int32, [_vp, C.c_int32, C.c_int32, C.c_int32, _vp]),
    "mqv_batch_tempering": (C.c_int32, [_vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _vp, C.c_int32,
                                        C.c_uint64, _vp, _vp]),
    "mqv_batch_launch_count": (C.c_int32, [_vp, C.POINTER(C.c_uint64)]),
    "mqv_selftest_accept_cut": (C.c_int32, [C.c_int32, C.c_int32, _vp, _vp, _vp]),
    "mqv_selftest_philox": (C.c_int32, [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32,
                                        _vp, _vp]),
}

_lib = None


def load() -> C.CDLL:
    """Load (once) the engine library; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"marqov_b200 engine library not built: {LIB_PATH} "
                          "(run `python marqov_b200/build.py` or __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def version() -> str:
    return load().mqv_version().decode()


def device_count() -> int:
    n = C.c_int32(0)
    load().mqv_device_count(C.byref(n))
    return int(n.value)


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().mqv_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != OK:
        raise MarqovError(status, last_error())
