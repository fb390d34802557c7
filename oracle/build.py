"""Build recipe for the CPU oracle -- TEST INFRASTRUCTURE.

* ``oracle/liboracle.so``        -- the C restatement (oracle.c), always built.
* ``oracle/_ref/libmarqov_ref.so`` -- ref_harness.cpp compiled against the
  reference's own headers, built only where the reference source tree exists
  (``MARQOV_REF_SRC`` or ``reference/src`` beside the checkout).  The output stays out of git but
  travels with the working tree, so machines without the source can still load it.
  (The reference tree is ``MARQOV_REF_SRC``, else ``../reference/src`` beside
  this checkout.)

Both use ``-march=x86-64-v3`` so the binaries run on any AVX2 host, not only
the build machine, and ``-ffp-contract=off`` so every FP64 operation of the
acceptance rule is rounded as written (the engine does the same on host and
device).  The reference harness is also built for ``-march=x86-64-v4``
(AVX-512) as ``libmarqov_ref_v4.so``; ``oracle.oracle.ref_path`` loads that
one on hosts whose CPU has the AVX-512 subsets of x86-64-v4, which is the
closest a binary built on one machine gets to ``-march=native`` on another.
Neither flag changes a result: without contraction or fast-math every FP
operation is the same IEEE operation in either build.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference's source tree: MARQOV_REF_SRC, else a checkout of it beside this one
REF_SRC_DEFAULT = os.path.join(os.path.dirname(HERE), "..", "reference", "src")
ARCH = ["-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fPIC", "-shared"]


def _newer(out: str, srcs: list[str]) -> bool:
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(s) <= t for s in srcs)


def build_oracle(force: bool = False) -> str:
    out = os.path.join(HERE, "liboracle.so")
    srcs = [os.path.join(HERE, "oracle.c"), os.path.join(HERE, "oracle.h")]
    if force or not _newer(out, srcs):
        cmd = ["gcc", "-std=gnu11", *ARCH, "-o", out, srcs[0], "-lm"]
        subprocess.check_call(cmd)
    return out


def build_ref(force: bool = False) -> str | None:
    src_root = os.environ.get("MARQOV_REF_SRC", REF_SRC_DEFAULT)
    out_dir = os.path.join(HERE, "_ref")
    out = os.path.join(out_dir, "libmarqov_ref.so")
    if not os.path.isdir(os.path.join(src_root, "libmarqov")):
        return out if os.path.exists(out) else None
    os.makedirs(out_dir, exist_ok=True)
    srcs = [os.path.join(HERE, "ref_harness.cpp"), os.path.join(HERE, "oracle.c"),
            os.path.join(HERE, "ref_scheduler.cpp"), os.path.join(HERE, "ref_io.cpp")]
    for march, lib in (("x86-64-v3", out), ("x86-64-v4", os.path.join(out_dir, "libmarqov_ref_v4.so"))):
        if force or not _newer(lib, srcs):
            obj = os.path.join(out_dir, f"oracle_c_{march}.o")
            subprocess.check_call(["gcc", "-std=gnu11", "-O3", f"-march={march}", "-ffp-contract=off", "-fPIC", "-c",
                                   "-o", obj, srcs[1]])
            cmd = ["g++", "-std=gnu++14", "-O3", f"-march={march}", "-ffp-contract=off", "-fPIC", "-shared", "-w",
                   "-I", src_root, "-o", lib, srcs[0], srcs[2], srcs[3], obj, "-lm", "-lpthread"]
            subprocess.check_call(cmd)
    return out


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build_oracle(force))
    print(build_ref(force))
