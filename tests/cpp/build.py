"""Build recipe of the C++ drop-in test program (tests/cpp/dropin_demo.cpp).

Compiles against the reference's own headers where the reference source tree
is present (MARQOV_REF_SRC, else reference/src beside this checkout) and links the engine
library; the binary (tests/cpp/_build/dropin_demo, git-ignored) finds the
library through its rpath.  Returns None where the reference is absent.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
# the reference's source tree: MARQOV_REF_SRC, else a checkout of it beside this one
REF_SRC_DEFAULT = os.path.join(ROOT, "..", "reference", "src")
OUT = os.path.join(HERE, "_build", "dropin_demo")


def build_demo(force: bool = False) -> str | None:
    src_root = os.environ.get("MARQOV_REF_SRC", REF_SRC_DEFAULT)
    if not os.path.isdir(os.path.join(src_root, "hamiltonian")):
        return OUT if os.path.exists(OUT) else None
    src = os.path.join(HERE, "dropin_demo.cpp")
    deps = [src] + [os.path.join(ROOT, "include", f) for f in
                    ("marqov_b200.h", "marqov_b200_core.hpp", "marqov_b200_marqov.hpp")]
    lib = os.path.join(ROOT, "marqov_b200", "libmarqov_b200.so")
    if not force and os.path.exists(OUT) and all(os.path.getmtime(d) <= os.path.getmtime(OUT) for d in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-w", "-I", os.path.join(ROOT, "include"), "-I", src_root, "-o", OUT, src,
           lib, "-Wl,-rpath,$ORIGIN/../../../marqov_b200"]
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build_demo("--force" in sys.argv))
