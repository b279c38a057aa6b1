"""Build libhm_erosion.so in-tree with nvcc for sm_100a.

``python -m highmap_b200.build`` (or ``build()`` of the repository's entry
module) compiles every source of ``highmap_b200/csrc`` into
``highmap_b200/lib/libhm_erosion.so``.  The library links the CUDA runtime
statically, so it depends only on the driver.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
OBJDIR = os.path.join(PKG, "lib", "obj")
LIB = os.path.join(LIBDIR, "libhm_erosion.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
          "-I", CSRC]
CUFLAGS = ARCH + COMMON + ["--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(ROOT, "include", "*.h")))


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
    flags = list(CUFLAGS)
    if verbose_ptxas and src.endswith(".cu"):
        flags += ["-Xptxas", "-v"]
    cmd = [NVCC, *flags, "-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, *COMMON, "-x", "cu", *ARCH, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s\n%s\n%s" % (src, r.stdout, r.stderr))
    if verbose_ptxas and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = _sources()
    newest_dep = max(os.path.getmtime(p) for p in srcs + _headers() + [__file__])
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest_dep:
        return LIB
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed\n%s\n%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv))
