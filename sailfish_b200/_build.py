"""
Builds libcbdiso_b200.so in-tree from sailfish_b200/csrc with nvcc for sm_100a.

    python -m sailfish_b200._build [--verbose] [--ptxas]

Translation units whose arithmetic must match the reference operation for
operation (the EXACT stage kernel and the zone-wise kernels) are compiled with
-fmad=false; the others allow FMA contraction.
"""

import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_objs")
LIB = os.path.join(HERE, "libcbdiso_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE, "--expt-relaxed-constexpr"]
NO_FMA = {"stage_exact.cu", "elementwise.cu", "stepper.cu", "batched_exact.cu", "adjoint.cu", "gam.cu"}
SOURCES = ["capi.cu", "elementwise.cu", "stage_exact.cu", "stage_fma.cu", "stage_fast.cu", "noalloc.cu",
           "stepper.cu", "batched_exact.cu", "batched.cu", "adjoint.cu", "gam.cu", "fp64_peak.cu"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _digest(paths, extra):
    h = hashlib.sha256()
    for p in sorted(paths):
        with open(p, "rb") as f:
            h.update(f.read())
    h.update(" ".join(extra).encode())
    return h.hexdigest()


def build(verbose=False, ptxas=False, force=False):
    """Compile every CUDA source and link the shared library. Returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, "cbdiso_b200.h")]
    stamp_path = os.path.join(BUILD, "stamp")
    digest = _digest(deps, ARCH + COMMON + (["ptxas"] if ptxas else []))
    if not force and os.path.exists(LIB) and os.path.exists(stamp_path):
        with open(stamp_path) as f:
            if f.read() == digest:
                return LIB
    cc = nvcc()
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        flags = ARCH + COMMON + (["-fmad=false"] if src in NO_FMA else [])
        if ptxas:
            flags = flags + ["-Xptxas", "-v"]
        cmd = [cc, "-c", os.path.join(CSRC, src), "-o", obj] + flags
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if out and (verbose or ptxas or p.returncode):
            print(f"--- {src}\n{out}", file=sys.stderr)
        failed |= p.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed")
    cmd = [cc, "-shared", "-o", LIB] + objs + ARCH + ["-Xcompiler", "-fPIC"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    with open(stamp_path, "w") as f:
        f.write(digest)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, ptxas="--ptxas" in sys.argv, force="--force" in sys.argv))
