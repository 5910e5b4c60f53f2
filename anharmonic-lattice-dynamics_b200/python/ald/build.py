"""Build libald.so in-tree for sm_100a with nvcc (no JIT cache, no pip install).

The shared library lands in anharmonic-lattice-dynamics_b200/lib/libald.so
so it travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
OBJDIR = os.path.join(PKG, "lib", "obj")
LIB = os.path.join(LIBDIR, "libald.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]

SOURCES = {
    "ald_host.cpp": [],
    "ald_pool.cpp": [],
    "ald_capi.cpp": [],
    "ald_pipeline.cpp": [],
    "ald_tune.cpp": [],
    "ald_phonon.cu": [],
    "ald_heev.cu": [],
    "ald_v3.cu": [],
    "ald_v3_pair.cu": [],
    "ald_v3_tc.cu": [],
    "ald_v3_dense.cu": [],
    "ald_v3_dense_tc.cu": [],
    # weight_tet's FP32/FP64 arithmetic must not be contracted into FMAs
    "ald_tetra.cu": ["-fmad=false", "--expt-relaxed-constexpr"],
    "ald_iso.cu": ["-fmad=false", "--expt-relaxed-constexpr"],
    "ald_bte.cu": [],
    "ald_util.cu": [],
    "ald_cg_static.cu": [],
    "ald_writers.cpp": [],
    # the self terms follow the reference's operation order: no contraction
    "ald_self.cu": ["-fmad=false"],
    "ald_self.cpp": [],
}


def _compile(src: str, extra) -> str:
    obj = os.path.join(OBJDIR, src + ".o")
    path = os.path.join(CSRC, src)
    # the compiler writes the object's header dependencies beside it (obj.d)
    dep = ["-MD", "-MF", obj + ".d"]
    if src.endswith(".cu"):
        cmd = [NVCC] + ARCH + COMMON + extra + dep + ["-c", path, "-o", obj]
    else:
        cmd = [os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-fPIC", "-Wall", "-I/usr/local/cuda/include",
               "-c", path, "-o", obj] + dep + extra
    subprocess.run(cmd, check=True)
    return obj


def _deps(obj: str, src: str):
    """The source and every header the compiler read for obj (from obj.d),
    system headers included; without a dependency file, every header of the
    package and include/."""
    d = obj + ".d"
    if os.path.exists(d):
        text = open(d).read().replace("\\\n", " ")
        files = text.split(":", 1)[1].split() if ":" in text else []
        return [os.path.join(CSRC, src)] + files
    hdr = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    return [os.path.join(CSRC, src), os.path.join(os.path.dirname(PKG), "include", "ald.h")] + hdr


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in _deps(obj, src) if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    todo = [s for s in srcs if force or _stale(os.path.join(OBJDIR, s + ".o"), s)]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            list(ex.map(lambda s: _compile(s, SOURCES[s]), todo))
    objs = [os.path.join(OBJDIR, s + ".o") for s in srcs]
    if force or todo or not os.path.exists(LIB):
        subprocess.run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"], check=True)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
