"""Build recipe for oracle/_ref: the reference's own hot-path kernel source
compiled for the host CPU.

GLUED keeps its kernels as C-like source strings inside
``platforms/common/src/CommonGluedKernels.cpp`` (runtime-compiled by OpenMM).
This script reads that file from the reference tree, pulls out the kernel
strings of the hot path, prefixes a small shim header that maps the OpenMM
kernel dialect (KERNEL, GLOBAL, real4, GLOBAL_ID, atomicAdd, ...) onto serial
host C++, and compiles it twice into ``oracle/_ref/``:

  libglued_ref_f32.so   real = float   (the reference's single/mixed precision)
  libglued_ref_f64.so   real = double

The extracted text is written only under ``oracle/_ref/`` (git-ignored). Nothing
here is vendored into the repository. Usage:

    python oracle/build_ref.py [--reference /root/reference]
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
DEFAULT_REF = os.environ.get("GLUED_REFERENCE", "/root/reference")

# Kernel strings of the hot path, in the order they are concatenated.
KERNELS = [
    "kDistanceKernelSrc", "kAngleKernelSrc", "kDihedralKernelSrc", "kCOMDistanceKernelSrc",
    "kGyrationKernelSrc", "kPathKernelSrc", "kRMSDKernelSrc", "kCoordinationKernelSrc",
    "kContactMapKernelSrc", "kPCAKernelSrc", "kScatterKernelSrc", "kHarmonicKernelSrc",
    "kOPESKernelSrc", "kMetaDKernelSrc", "kPBMetaDKernelSrc",
]

SHIM = r"""
// Shim: OpenMM common-compute kernel dialect -> serial host C++.
#include <cmath>
#include <algorithm>
#include <cstdint>
using std::floor; using std::sqrt; using std::exp; using std::log; using std::pow;
using std::fabs; using std::atan2; using std::acos; using std::round; using std::log1p;
using std::max; using std::min;
typedef REAL real;
struct real4 { real x, y, z, w; };
struct real3 { real x, y, z; };
static inline real3 make_real3(real x, real y, real z) { real3 r = {x, y, z}; return r; }
typedef long long mm_long;
typedef unsigned long long mm_ulong;
#define KERNEL extern "C"
#define GLOBAL
#define RESTRICT
#define DEVICE static
#define GLOBAL_ID 0
#define GLOBAL_SIZE 1
static inline int atomicAdd(int* p, int v) { int o = *p; *p += v; return o; }
static inline mm_ulong atomicAdd(mm_ulong* p, mm_ulong v) { mm_ulong o = *p; *p += v; return o; }
static inline double atomicAdd(double* p, double v) { double o = *p; *p += v; return o; }
"""

_RAW = re.compile(r'extern const string (k\w+)\s*=\s*(?:(k\w+)\s*\+\s*)?R"\((.*?)\)";', re.S)


def extract(reference: str) -> str:
    src_path = os.path.join(reference, "platforms", "common", "src", "CommonGluedKernels.cpp")
    with open(src_path, encoding="utf-8") as fh:
        text = fh.read()
    raw = {}
    for name, _prefix, body in _RAW.findall(text):
        raw[name] = body
    missing = [k for k in ["kGeometryFunctions"] + KERNELS if k not in raw]
    if missing:
        raise SystemExit(f"build_ref: kernel strings not found: {missing}")
    parts = ["// Extracted from " + src_path + " at build time. Not part of the repository.",
             SHIM, raw["kGeometryFunctions"]]
    for k in KERNELS:
        parts.append(f"// ---- {k}\n" + raw[k])
    return "\n".join(parts)


def build(reference: str = DEFAULT_REF, quiet: bool = False) -> bool:
    if not os.path.isdir(reference):
        if not quiet:
            print(f"build_ref: reference tree {reference} not present; skipping", file=sys.stderr)
        return False
    os.makedirs(OUT, exist_ok=True)
    src = os.path.join(OUT, "glued_ref_kernels.cpp")
    with open(src, "w", encoding="utf-8") as fh:
        fh.write(extract(reference))
    for tag, real in (("f32", "float"), ("f64", "double")):
        out = os.path.join(OUT, f"libglued_ref_{tag}.so")
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
               "-w", f"-DREAL={real}", src, "-o", out]
        subprocess.check_call(cmd)
    return True


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REF)
    a = ap.parse_args()
    ok = build(a.reference)
    print("built oracle/_ref" if ok else "reference absent; nothing built")
