"""
Builds the CPU oracle (test infrastructure only): the C restatement of the
reference kernels into oracle/_build/liboracle_cbdiso.so, and, where the
reference tree is present, the reference kernels themselves into oracle/_ref
(oracle/build_ref.sh).
"""

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build_oracle(verbose=False):
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    src = os.path.join(HERE, "cbdiso_2d_oracle.c")
    out = os.path.join(out_dir, "liboracle_cbdiso.so")
    if os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    cmd = ["/usr/bin/gcc", "-O2", "-fwrapv", "-fPIC", "-shared", "-fopenmp", "-std=c99", src, "-o", out, "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return out


def build_reference(verbose=False):
    script = os.path.join(HERE, "build_ref.sh")
    subprocess.run(["bash", script], check=True, capture_output=not verbose)


if __name__ == "__main__":
    print(build_oracle(verbose=True))
    build_reference(verbose=True)
