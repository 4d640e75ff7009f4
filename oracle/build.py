"""Build recipe for the oracle's C code (TEST INFRASTRUCTURE ONLY).

``python -m oracle.build`` compiles oracle/dft.c with gcc/OpenMP into
oracle/_build/liboracle_dft.so, and -- when the reference sources are present
in this container -- the reference library itself into oracle/_ref/ via
oracle/Makefile.ref.  Both outputs are git-ignored; they travel to GPU boxes
with the working tree.  The reference source tree is taken from the
CURIG_REFERENCE environment variable (default: the read-only checkout this
recipe was written against).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_SRC = os.environ.get("CURIG_REFERENCE", "/root/reference")


def build_dft(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, "liboracle_dft.so")
    src = os.path.join(HERE, "dft.c")
    if force or not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=gnu11",
                               src, "-o", out, "-lm"])
    return out


def build_ref(force: bool = False) -> str | None:
    """Reference libcurafft.so for sm_100a from its own sources (GPU-only code)."""
    if not os.path.isdir(REF_SRC):
        return None
    out = os.path.join(HERE, "_ref", "libcurafft_ref.so")
    if os.path.exists(out) and not force:
        return out
    subprocess.check_call(["make", "-f", os.path.join(HERE, "Makefile.ref"),
                           "REF=" + REF_SRC, "OUT=" + os.path.join(HERE, "_ref")])
    return out


if __name__ == "__main__":
    print(build_dft(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
