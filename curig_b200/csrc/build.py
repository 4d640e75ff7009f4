"""Build libcurafft.so (the B200 gridder) in-tree with nvcc for sm_100a.

    python curig_b200/csrc/build.py [--force] [-v] [--check]

Objects go to curig_b200/csrc/_build/, the shared library to
curig_b200/libcurafft.so (next to the Python package, as the reference's
package_data, setup.py:24).  --check builds the bounds-checked variant
curig_b200/libcurafft_check.so (objects in _build_check/, -DCURIG_BOUNDS_CHECK:
the kernels check their buffer indices, skip an access that would leave its
buffer and report it as an error status); select it with CURIG_LIB.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(PKG, "libcurafft.so")
OBJ_CHECK = os.path.join(HERE, "_build_check")
LIB_CHECK = os.path.join(PKG, "libcurafft_check.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I" + HERE, "-I" + os.path.join(ROOT, "include")]
SOURCES = ["params.cpp", "kernels.cu", "plan.cu", "abi.cu", "learned.cu", "nufft3.cu"]
HEADERS = ["curig_internal.h", "kernels.cuh", "plan.h"]


def _newer(src_paths, out):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in src_paths)


def _compile(src, force, verbose, check=False):
    path = os.path.join(HERE, src)
    out = os.path.join(OBJ_CHECK if check else OBJ, os.path.splitext(src)[0] + ".o")
    deps = [path] + [os.path.join(HERE, h) for h in HEADERS] + [
        os.path.join(ROOT, "include", "curig.h"), os.path.join(ROOT, "include", "cugridder.h")]
    if not force and not _newer(deps, out):
        return out
    lang = ["-x", "cu"] if src.endswith(".cu") else ["-x", "c++"]
    cmd = [NVCC, *ARCH, *FLAGS, *(["-DCURIG_BOUNDS_CHECK"] if check else []), *lang, "-c", path, "-o", out]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return out


def build(force: bool = False, verbose: bool = False, check: bool = False) -> str:
    obj_dir, lib = (OBJ_CHECK, LIB_CHECK) if check else (OBJ, LIB)
    os.makedirs(obj_dir, exist_ok=True)
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(HERE, s))]
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose, check), srcs))
    if force or _newer(objs, lib):
        subprocess.check_call([NVCC, *ARCH, "-shared", *objs, "-o", lib, "-lcufft"])
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv, check="--check" in sys.argv))
