"""Build recipe for the test oracle (TEST INFRASTRUCTURE ONLY).

* ``oracle/libhm_oracle.so``: the C restatement (hm_oracle.c), gcc -O2,
  -ffp-contract=off so each float operation rounds once, OpenMP.
* ``oracle/_ref/libhm_ref.so``: the reference's own kernel text
  (HighMap/src/gpu_opencl/kernels/_common_index.cl, thermal.cl,
  hydraulic_vpipes.cl, thermal_ridge.cl, thermal_scree.cl, thermal_schott.cl,
  thermal_olsen.cl, thermal_flatten.cl, thermal_inflate.cl, thermal_rib.cl,
  shallow_viscous_flow.cl, and the helper functions they call from
  _common_math.cl and _common_rand.cl) compiled for the CPU behind
  ``ref_shim.h``, linked
  with the host-driver restatement ``ref_harness.cpp``.  Built only where
  the reference tree is present (``HM_REFERENCE_ROOT``, default: a
  ``reference`` directory beside the repository); the kernel files are read in place and streamed to the
  compiler, nothing of them is written anywhere but the object in _ref/.

Run: ``python oracle/build_oracle.py`` (``build()`` in the repository's
entry module calls the same functions).
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(HERE, "libhm_oracle.so")
REF_SO = os.path.join(REF_DIR, "libhm_ref.so")
KERNEL_FILES = ("_common_index.cl", "thermal.cl", "hydraulic_vpipes.cl", "thermal_ridge.cl", "thermal_scree.cl",
                "thermal_schott.cl", "thermal_olsen.cl", "thermal_flatten.cl", "thermal_inflate.cl", "thermal_rib.cl",
                "shallow_viscous_flow.cl")
# helpers the sibling talus kernels call, taken function by function from
# the shared kernel files (the rest of those files is not needed)
HELPER_FUNCTIONS = (("_common_math.cl", ("almost_unit_identity", "smoothstep3")), ("_common_rand.cl", ("hash21u",)))
CFLAGS = ["-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-march=x86-64-v2"]


def reference_root() -> str:
    """The HighMap checkout: HM_REFERENCE_ROOT, else a directory named
    ``reference`` beside the repository's root."""
    env = os.environ.get("HM_REFERENCE_ROOT")
    if env:
        return env
    return os.path.normpath(os.path.join(HERE, "..", "..", "reference"))


def _run(cmd, **kw):
    r = subprocess.run(cmd, capture_output=True, text=True, **kw)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def _stale(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build_oracle(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("hm_oracle.c", "hm_oracle_body.inc", "hm_oracle.h")]
    if force or _stale(ORACLE_SO, srcs):
        _run(["gcc", "-std=c11", *CFLAGS, "-shared", "-o", ORACLE_SO, srcs[0], "-lm"])
    return ORACLE_SO


def _kernel_text(path: str) -> str:
    """The OpenCL C of one kernel file: its R""( ... )"" wrapper lines are
    dropped and the two vector-literal spellings are rewritten (see
    ref_shim.h)."""
    with open(path) as f:
        lines = f.read().splitlines()
    if not lines or lines[0].strip() != 'R""(' or lines[-1].strip() != ')""':
        raise RuntimeError("unexpected framing in %s" % path)
    body = "\n".join(lines[1:-1]) + "\n"
    return body.replace("(int2)(", "HM_INT2(").replace("(float2)(", "HM_FLOAT2(")


def _function_text(path: str, name: str) -> str:
    """The definition of one function of a kernel file: from the line that
    declares it to its closing brace."""
    text = _kernel_text(path)
    m = re.search(r"^[A-Za-z_][\w ]*\b%s\s*\(" % re.escape(name), text, re.M)
    if not m:
        raise RuntimeError("%s not found in %s" % (name, path))
    start = text.index("{", m.end())
    depth = 0
    for k in range(start, len(text)):
        depth += {"{": 1, "}": -1}.get(text[k], 0)
        if depth == 0:
            return text[m.start():k + 1] + "\n"
    raise RuntimeError("unbalanced braces after %s in %s" % (name, path))


def build_ref(force: bool = False) -> str | None:
    """Compile the reference's kernel text into oracle/_ref/libhm_ref.so.
    Returns the path, or None when the reference tree is absent (the GPU
    box uses the library built here)."""
    kdir = os.path.join(reference_root(), "HighMap", "src", "gpu_opencl", "kernels")
    kfiles = [os.path.join(kdir, f) for f in KERNEL_FILES]
    hfiles = [os.path.join(kdir, f) for f, _ in HELPER_FUNCTIONS]
    if not all(os.path.exists(k) for k in kfiles + hfiles):
        return REF_SO if os.path.exists(REF_SO) else None
    own = [os.path.join(HERE, f) for f in ("ref_shim.h", "ref_harness.cpp", "hm_oracle.h")]
    if not (force or _stale(REF_SO, kfiles + hfiles + own)):
        return REF_SO
    os.makedirs(REF_DIR, exist_ok=True)
    unit = '#include "ref_shim.h"\nnamespace hmref {\n'
    for (f, names), path in zip(HELPER_FUNCTIONS, hfiles):
        for name in names:
            unit += '#line 1 "%s"\n' % path + _function_text(path, name)
    for k in kfiles:
        unit += '#line 2 "%s"\n' % k + _kernel_text(k)
    unit += "}\n"
    kobj = os.path.join(REF_DIR, "ref_kernels.o")
    _run(["g++", "-std=c++17", *CFLAGS, "-w", "-I", HERE, "-x", "c++", "-c", "-", "-o", kobj], input=unit)
    hobj = os.path.join(REF_DIR, "ref_harness.o")
    _run(["g++", "-std=c++17", *CFLAGS, "-I", HERE, "-c", os.path.join(HERE, "ref_harness.cpp"), "-o", hobj])
    _run(["g++", *CFLAGS, "-shared", "-o", REF_SO, kobj, hobj, "-lm"])
    return REF_SO


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
