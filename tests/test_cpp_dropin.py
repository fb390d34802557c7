"""The header-only C++ layer (include/marqov_b200_core.hpp with the MARQOV
lowerings of include/marqov_b200_marqov.hpp) used the way a MARQOV program
uses makeCore: tests/cpp/dropin_demo.cpp is compiled against the reference's
own Hamiltonian and lattice headers.  Without a GPU it must build and report
the missing device; on a GPU its results must equal the Python API's."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "cpp"))


def demo_binary(build: bool):
    import build as B
    path = B.build_demo() if build else (B.OUT if os.path.exists(B.OUT) else None)
    if path is None:
        pytest.skip("C++ drop-in program not built (reference headers absent)")
    return path


def test_dropin_builds_and_runs_without_a_device():
    import marqov_b200 as M
    path = demo_binary(build=True)
    if M._lib.device_count() > 0:
        pytest.skip("a GPU is present: see the gpu test")
    out = subprocess.run([path], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.startswith("no device:")


@pytest.mark.gpu
def test_dropin_equals_python_api():
    import marqov_b200 as M
    path = demo_binary(build=False)
    out = subprocess.run([path], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [l.split() for l in out.stdout.strip().splitlines()]
    core = np.array([[float(a), float(b)] for t, a, b in (l for l in lines if l[0] == "core")])
    farm = {int(l[1]): (float(l[2]), float(l[3])) for l in lines if l[0] == "farm"}
    ea = [l for l in lines if l[0] == "ea"]
    # the same runs through the Python API
    cfg = M.Config(seed=17, repid=0, ncluster=1, nmetro=1)
    with M.makeCore(M.RegularHypercubic(32, 2), cfg, M.Ising(-1.0), 0.44068679) as c:
        c.init()
        c.emcs(50, measure=False)
        obs, _ = c.emcs(5)
    np.testing.assert_array_equal(core, obs[:, :2])
    ms = [(M.RegularHypercubic(L, 2), M.Config(seed=5, repid=i), M.Potts(3, -1.0), 1.0 + 0.05 * i)
          for i, L in enumerate((16, 24, 32))]
    with M.Batch(ms) as b:
        b.init()
        b.emcs(20, 1, 2)
        fo, _ = b.emcs(4, 1, 2)
    for i in range(3):
        assert farm[i] == (fo[3, i, 0], fo[3, i, 1])
    assert len(ea) == 1 and np.isfinite([float(ea[0][1]), float(ea[0][2])]).all()
    # parallel tempering: GPUScheduler(maxptsteps=6, ptseed=3) vs Batch.tempering
    pt = {int(l[1]): (float(l[2]), float(l[3])) for l in lines if l[0] == "pt"}
    ptacc = [float(l[1]) for l in lines if l[0] == "ptacc"]
    ms = [(M.RegularHypercubic(12, 2), M.Config(seed=21 + i, repid=i), M.Ising(-1.0), 0.38 + 0.04 * i)
          for i in range(4)]
    with M.Batch(ms) as b:
        b.init()
        b.emcs(10, 1, 1)
        po, acc = b.tempering(6, emcs_per_step=3, ncluster=1, nmetro=1,
                              plan=M.tempering.reference_plan(4, 6, seed=3), seed=3)
    for i in range(4):
        assert pt[i] == (po[-1, i, 0], po[-1, i, 1])
    assert ptacc == [float((acc == 1).sum()) / 6.0]
    # XXZAntiferroSingleAniso(H=0.3, Delta=1.2, D=0.5) on SimpleBipartite(6, 3) at beta 0.8
    xxz = np.array([[float(a), float(b)] for t, a, b in (l for l in lines if l[0] == "xxz")])
    cfg = M.Config(seed=33, repid=0, ncluster=0, nmetro=1)
    with M.makeCore(M.SimpleBipartite(6, 3), cfg, M.XXZAntiferroSingleAniso(0.3, 1.2, 0.5), 0.8) as c:
        c.init()
        c.emcs(4, ncluster=0, nmetro=1, measure=False)
        xo, _ = c.emcs(3, ncluster=0, nmetro=1)
    np.testing.assert_array_equal(xxz, xo[:, :2])
    # user term-API classes: MyIsing lowers to the generic-Wolff Ising, MyXXZ
    # to XXZ (Delta = 0.6, H = 0.25), a component-mixing interaction is refused
    mi = np.array([[float(a), float(b)] for t, a, b in (l for l in lines if l[0] == "myising")])
    cfg = M.Config(seed=44, repid=0, ncluster=1, nmetro=1)
    with M.makeCore(M.RegularHypercubic(16, 2), cfg, M.Ising(-1.0, "int8"), 0.44) as c:
        c.init()
        c.emcs(5, measure=False)
        o, _ = c.emcs(4)
    np.testing.assert_array_equal(mi, o[:, :2])
    mx = np.array([[float(a), float(b)] for t, a, b in (l for l in lines if l[0] == "myxxz")])
    cfg = M.Config(seed=45, repid=0, ncluster=0, nmetro=1)
    with M.makeCore(M.RegularHypercubic(6, 3), cfg, M.XXZAntiferro(0.6, 0.25), 0.7) as c:
        c.init()
        c.emcs(3, ncluster=0, nmetro=1, measure=False)
        o, _ = c.emcs(3, ncluster=0, nmetro=1)
    np.testing.assert_array_equal(mx, o[:, :2])
    assert [l for l in lines if l[0] == "unsupported"] == [["unsupported", str(M._lib.ERR_UNSUPPORTED_TERM)]]
