"""Compiles the OpenMM adapter (gluedmd_b200/openmm/B200GluedKernels.cpp) with
the test harness (fake_openmm.cpp) against the stub headers in include/, linked
with the product library, into _build/libadapter_harness.so (git-ignored).

Test infrastructure: with OpenMM installed, the same adapter source compiles
against OpenMM's own headers and GLUED's openmmapi headers instead."""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
ADAPTER = os.path.join(ROOT, "gluedmd_b200", "openmm")
LIBDIR = os.path.join(ROOT, "gluedmd_b200", "_lib")
OUT = os.path.join(HERE, "_build", "libadapter_harness.so")


def _cuda_include():
    for d in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if d and os.path.exists(os.path.join(d, "include", "cuda.h")):
            return os.path.join(d, "include")
    raise RuntimeError("cuda.h not found (CUDA toolkit headers)")


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, "fake_openmm.cpp"), os.path.join(ADAPTER, "B200GluedKernels.cpp")]
    deps = srcs + [os.path.join(ADAPTER, "B200GluedKernels.h"), os.path.join(LIBDIR, "libglued_b200.so")]
    for root, _, files in os.walk(os.path.join(HERE, "include")):
        deps += [os.path.join(root, f) for f in files]
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= max(os.path.getmtime(d) for d in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    tmp = OUT + f".tmp{os.getpid()}"
    cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall",
           "-I" + os.path.join(HERE, "include"), "-I" + ADAPTER, "-I" + os.path.join(ROOT, "include"),
           "-I" + _cuda_include(), *srcs, "-o", tmp, "-L" + LIBDIR, "-lglued_b200",
           "-Wl,-rpath,$ORIGIN/../../../gluedmd_b200/_lib"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("adapter build failed:\n" + r.stdout + r.stderr)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force=True))
