"""C-ABI library and host logic, without a GPU: the library loads, exports
every entry point include/marqov_b200.h declares, and the host-side lattice
lowering matches the reference's neighbour conventions."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "marqov_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"MQV_API\s+[\w\s\*]+?\b(mqv_\w+)\s*\(", txt)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for must in ("mqv_create", "mqv_destroy", "mqv_metropolis", "mqv_wolff", "mqv_emcs", "mqv_measure",
                 "mqv_get_state", "mqv_set_state", "mqv_last_error"):
        assert must in syms


def test_library_exports_every_declared_symbol():
    from marqov_b200 import _lib
    lib = _lib.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (mqv_\w+)", out))
    assert set(declared_symbols()) <= exported
    # nothing but the C ABI is exported from the engine's own code
    assert all(s.startswith("mqv_") for s in exported)


def test_version_and_errors():
    from marqov_b200 import _lib
    lib = _lib.load()
    assert b"marqov_b200" in lib.mqv_version()
    assert lib.mqv_destroy(None) == 0
    assert lib.mqv_create(None, None, None, None) == _lib.ERR_INVALID_ARG
    assert "null" in _lib.last_error()


def test_create_without_device_reports_no_device():
    from marqov_b200 import _lib
    if _lib.device_count() > 0:
        pytest.skip("a GPU is present")
    lib = _lib.load()
    md = _lib.ModelDesc(kind=_lib.MODEL_ISING, J=-1.0)
    ld = _lib.LatticeDesc(kind=_lib.LATTICE_HYPERCUBIC, dim=2, len=16)
    rp = _lib.RunParams(beta=0.44, seed=1, replica=0, device=0)
    h = C.c_void_p()
    assert lib.mqv_create(C.byref(md), C.byref(ld), C.byref(rp), C.byref(h)) == _lib.ERR_NO_DEVICE
    assert not h.value


def test_hypercubic_neighbours_match_oracle(orc):
    from marqov_b200 import RegularHypercubic
    for dim, L in ((1, 6), (2, 4), (3, 4), (4, 4)):
        lat = RegularHypercubic(L, dim)
        g = orc.hypercubic(dim, L)
        csr = lat.to_csr()
        assert (csr.row_ptr == g.row_ptr).all() and (csr.col_idx == g.col_idx).all()
        for i in (0, 1, L - 1, lat.size() - 1):
            assert lat.nbrs(0, i) == g.col_idx[g.row_ptr[i]:g.row_ptr[i + 1]].tolist()
        # parity colouring is proper
        for i in range(lat.size()):
            for j in lat.nbrs(0, i):
                assert csr.colours[i] != csr.colours[j]


def test_hypercubic_crds():
    """RegularLattice::crds (src/lattice/util/regular_lattice.h:36-48)."""
    from marqov_b200 import RegularHypercubic
    lat = RegularHypercubic(16, 3)
    for k in (0, 5, 17, 4000):
        ref = []
        kk = k
        for i in range(3):
            idx = (kk // 16 ** i) % 16
            kk -= idx * 16 ** i
            ref.append(idx / 16 + 0.5 / 16)
        assert np.allclose(lat.crds(k), ref)


def _symmetric(csr):
    pairs = {}
    for i in range(csr.n):
        for p in range(csr.row_ptr[i], csr.row_ptr[i + 1]):
            pairs[(i, int(csr.col_idx[p]))] = None if csr.bonds is None else int(csr.bonds[p])
    return all((j, i) in pairs and pairs[(j, i)] == w for (i, j), w in pairs.items())


def test_random_bond_lattice_symmetric():
    from marqov_b200 import RegularRandomBond
    lat = RegularRandomBond(6, 3, p=0.5, seed=3)
    assert _symmetric(lat.to_csr())
    for i in range(lat.size()):
        assert lat.bnds(0, i) == lat.to_csr().bnds(0, i)
    assert set(np.unique(lat.bonds)) <= {-1, 1}
    frac = (lat.bonds == 1).mean()
    assert 0.35 < frac < 0.65


def test_random_geometric_graph():
    from marqov_b200 import RandomGeometricGraph2D
    g = RandomGeometricGraph2D(20000, 8.0, seed=1)
    deg = np.diff(g.row_ptr)
    assert abs(deg.mean() - 8.0) < 0.3
    assert _symmetric(g)
    assert (g.col_idx != np.repeat(np.arange(g.n), deg)).all()
    col = g.greedy_colours()
    for i in range(0, g.n, 97):
        for j in g.nbrs(0, i):
            assert col[i] != col[j]


def test_graph_csv_roundtrip(tmp_path):
    from marqov_b200 import read_graph_csv
    p = tmp_path / "g.csv"
    p.write_text("2\nx y neighbours\n0.1\t0.2\t1\t2\n0.3\t0.4\t0\n0.5\t0.6\t0\n")
    g = read_graph_csv(str(p))
    assert g.n == 3 and g.nbrs(0, 0) == [1, 2] and g.nbrs(0, 2) == [0]
