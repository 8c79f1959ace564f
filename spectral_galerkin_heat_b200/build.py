"""Build ``libsgh_b200.so`` in-tree with nvcc for sm_100a.

``python -m spectral_galerkin_heat_b200.build`` (or ``build()``). The library is
rebuilt when any source under ``csrc/`` or ``include/`` is newer than it.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libsgh_b200.so")
SOURCES = [os.path.join(CSRC, "sgh_b200.cu"), os.path.join(CSRC, "sgh_batch.cu"),
           os.path.join(CSRC, "sgh_mixed.cu"), os.path.join(CSRC, "sgh_outputs.cu")]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(d, f) for d in (CSRC, INCLUDE) for f in os.listdir(d)]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library if needed (translation units in parallel); return its path."""
    if not force and not _stale():
        return LIB
    objs, procs = [], []
    for src in SOURCES:
        obj = os.path.join(CSRC, os.path.basename(src) + ".o")
        cmd = [_nvcc(), *NVCC_FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append(subprocess.Popen(cmd))
        objs.append(obj)
    if any(p.wait() != 0 for p in procs):
        raise RuntimeError("nvcc failed")
    link = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs,
            "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
    os.replace(LIB + ".tmp", LIB)
    for obj in objs:
        os.remove(obj)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
