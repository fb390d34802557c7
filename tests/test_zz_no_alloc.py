"""mqv_wolff_noalloc: the Wolff update on static device scratch.

Collected last, so it also runs after every other GPU test has used the
engine on the same device.  The entry point must grow the same clusters as
mqv_wolff on the same state and counters, call after call, and leave its
static visited bitmap clean for the next call.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _engine():
    import marqov_b200 as M
    if M._lib.device_count() < 1:
        pytest.skip("no CUDA device")
    return M


CASES = [
    ("ising", 64, 2),        # Wolff<Ising<int>>, fused split-row layout
    ("ising8", 16, 3),       # generic Wolff + Embedder (Ising<int8_t>)
    ("potts", 32, 2),        # Wolff<Potts<3>>
]


def _ham(M, name):
    if name == "ising":
        return M.Ising(-1.0, "int")
    if name == "ising8":
        return M.Ising(-1.0, "int8")
    return M.Potts(3, -1.0)


@pytest.mark.parametrize("name,L,dim", CASES)
def test_noalloc_equals_wolff_two_calls(name, L, dim):
    M = _engine()
    lib = M._lib.load()
    beta = 0.44068679 if name != "potts" else 1.005
    mk = lambda: M.makeCore(M.RegularHypercubic(L, dim), M.Config(seed=31337, repid=2), _ham(M, name), beta)
    with mk() as a, mk() as b:
        a.init()
        b.init()
        assert (a.state == b.state).all()
        for call in range(2):
            n = 9
            ref = a.wolff(n)
            got = np.zeros(n, np.int32)
            M._lib.check(lib.mqv_wolff_noalloc(b.handle, n, got.ctypes.data))
            assert (got == ref).all(), f"call {call}: cluster sizes differ"
            assert (b.state == a.state).all(), f"call {call}: states differ"
            assert a.counters == b.counters


def test_noalloc_without_sizes_then_with_sizes():
    M = _engine()
    lib = M._lib.load()
    mk = lambda: M.makeCore(M.RegularHypercubic(32, 2), M.Config(seed=5, repid=0), M.Ising(-1.0), 0.44068679)
    with mk() as a, mk() as b:
        a.init()
        b.init()
        a.wolff(4)
        M._lib.check(lib.mqv_wolff_noalloc(b.handle, 4, None))
        ref = a.wolff(3)
        got = np.zeros(3, np.int32)
        M._lib.check(lib.mqv_wolff_noalloc(b.handle, 3, got.ctypes.data))
        assert (got == ref).all()
        assert (b.state == a.state).all()


def test_noalloc_rejects_lattice_above_limit():
    M = _engine()
    lib = M._lib.load()
    # 1026^2 = 1,052,676 sites > 2^20
    with M.makeCore(M.RegularHypercubic(1026, 2), M.Config(seed=1), M.Ising(-1.0), 0.44068679) as c:
        c.init()
        st = lib.mqv_wolff_noalloc(c.handle, 1, None)
        assert st == M._lib.ERR_INVALID_ARG
        assert "1048576" in M._lib.last_error()


def test_noalloc_rejects_float_models():
    M = _engine()
    lib = M._lib.load()
    with M.makeCore(M.RegularHypercubic(8, 3), M.Config(seed=1), M.Heisenberg(-1.0), 0.693) as c:
        c.init()
        assert lib.mqv_wolff_noalloc(c.handle, 1, None) == M._lib.ERR_UNSUPPORTED_TERM
