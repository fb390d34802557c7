"""Geometry files: read_graph_csv (GraphFromCSV) and save_geometry against the
reference's own io.h compiled into oracle/_ref, on files with the format's
corners (header line, ragged rows, empty rows, trailing tab, CRLF, no final
newline, 1-based ids) and on the lattices the engine builds."""
import os

import numpy as np
import pytest

import marqov_b200 as M


@pytest.fixture(scope="module")
def ref():
    from oracle.oracle import RefHarness, ref_path
    if not os.path.exists(ref_path()):
        pytest.skip("reference harness not built")
    return RefHarness()


CASES = {
    "plain": "2\nx\ty\tnbrs\n0.1\t0.2\t1\t2\n0.3\t0.4\t0\n0.5\t0.6\t0\t1\n",
    "no_final_newline": "2\n\n0.1\t0.2\t1\n0.3\t0.4\t0",
    "empty_row": "1\nh\n0.5\t1\n\n0.25\t0\n",
    "trailing_tab": "1\nh\n0.5\t1\t\n0.25\t0\t\n",
    "crlf": "2\r\nheader\r\n1.0\t2.0\t1\r\n3.0\t4.0\t0\r\n",
    "ragged": "2\nh\n1e-3\t-2.5E2\t1\t2\t3\n7\n0.5\t0.5\t0\n1\t1\t0\n",
    "no_coords": "0\nh\n1\t2\n0\n0\n",
    "numbers_with_tails": "2 coords\nh\n 0.5x\t+1.5\t 2\t1\n.5\t-0\t0\n-inf\tnan\t0\n",
}


def read_both(ref, path, idxoffs=0):
    mine = M.read_graph_csv(str(path), idxoffs=idxoffs)
    theirs = ref.import_geometry(path, idxoffs)
    return mine, theirs


@pytest.mark.parametrize("name", sorted(CASES))
def test_reader_equals_graph_from_csv(ref, tmp_path, name):
    p = tmp_path / f"{name}.csv"
    p.write_bytes(CASES[name].encode())
    mine, theirs = read_both(ref, p)
    rp, ci, crd, nc = theirs
    assert (mine.row_ptr == rp).all() and (mine.col_idx == ci).all()
    got = [mine.crds(i) for i in range(mine.n)]
    assert len(got) == len(crd)
    for a, b in zip(got, crd):
        np.testing.assert_array_equal(np.array(a), np.array(b))


def test_reader_one_based_ids(ref, tmp_path):
    p = tmp_path / "one.csv"
    p.write_text("1\nh\n0.1\t2\t3\n0.2\t1\n0.3\t1\n")
    mine, (rp, ci, _, _) = read_both(ref, p, idxoffs=1)
    assert (mine.col_idx == ci).all() and list(ci) == [1, 2, 0, 0]


def test_reader_rejects_what_the_reference_throws_on(ref, tmp_path):
    p = tmp_path / "bad.csv"
    p.write_text("1\nh\n0.1\t\t2\n")
    assert ref.import_geometry(p) is None
    with pytest.raises(ValueError):
        M.read_graph_csv(str(p))


@pytest.mark.parametrize("which", ["rgg", "hypercubic", "csr_without_coords"])
def test_save_geometry_equals_reference(ref, tmp_path, which):
    if which == "rgg":
        lat = M.RandomGeometricGraph2D(300, 6.0, seed=5)
        crd = np.array([lat.crds(i) for i in range(lat.size())])
        rp, ci = lat.row_ptr, lat.col_idx
    elif which == "hypercubic":
        lat = M.RegularHypercubic(6, 3)
        crd = np.array([lat.crds(i) for i in range(lat.size())])
        c = M.CSRLattice.from_nbrs(lat)
        rp, ci = c.row_ptr, c.col_idx
    else:
        lat = M.CSRLattice.from_nbrs(M.RegularHypercubic(4, 2))
        crd = np.zeros((lat.size(), 0))
        rp, ci = lat.row_ptr, lat.col_idx
    a, b = tmp_path / "mine.dat", tmp_path / "ref.dat"
    M.save_geometry(lat, str(a))
    ref.save_geometry(rp, ci, crd, b)
    assert a.read_bytes() == b.read_bytes()


def test_saved_geometry_reads_back_with_a_header(tmp_path):
    """save_geometry's rows behind the two header lines GraphFromCSV expects
    (the saved count column then reads as the first coordinate)."""
    lat = M.RandomGeometricGraph2D(200, 5.0, seed=2)
    p = tmp_path / "g.dat"
    M.save_geometry(lat, str(p))
    q = tmp_path / "g.csv"
    q.write_text("3\nsaved\n" + p.read_text())
    g = M.read_graph_csv(str(q))
    assert (g.row_ptr == lat.row_ptr).all() and (g.col_idx == lat.col_idx).all()
    np.testing.assert_allclose(np.array([g.crds(i)[1:] for i in range(g.n)]), lat.coords, atol=1e-15)
