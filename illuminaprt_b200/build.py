"""Build the sm_100a shared library (libilg.so) in-tree with nvcc.

The library is the product: every query of the package goes through it. It is
compiled for sm_100a only (B200); there is no other code path.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libilg.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fvisibility=hidden: only the entry points include/ilg.h marks ILG_API are
# exported; the library's C++ internals stay private to it
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    if not force and not _stale():
        return LIB
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, "-dc" if False else "-c", src, "-o", obj]
        if ptxas_v:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


PLUGIN_DIR = os.path.join(PKG, "plugin")
PLUGIN = os.path.join(PLUGIN_DIR, "libilg_gpuspace.so")
# the engine's Core tree: $ILLUMINA_CORE, else a checkout named "reference"
# beside this repository
REF_CORE = os.environ.get("ILLUMINA_CORE", os.path.join(os.path.dirname(ROOT), "reference", "Core"))


def build_plugin() -> str | None:
    """Build the GpuSpace engine plug-in (plugin/libilg_gpuspace.so) against the
    engine's headers in REF_CORE; returns its path, or None when the headers
    are not on this machine (a plug-in built elsewhere is used as it is)."""
    if not os.path.isdir(os.path.join(REF_CORE, "Space")):
        return PLUGIN if os.path.exists(PLUGIN) else None
    build()
    subprocess.run(["make", "-s", "-C", PLUGIN_DIR, f"REF={REF_CORE}"], check=True)
    return PLUGIN


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_v="--ptxas-v" in sys.argv)
    build_plugin()
