"""
Builds the CPU oracle (test infrastructure only): the C restatements of the
reference kernels into oracle/_build/liboracle_cbdiso.so and
liboracle_cbdgam.so, and, where the
reference tree is present, the reference kernels themselves into oracle/_ref
(oracle/build_ref.sh).
"""

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def _compile(src_name, lib_name, verbose):
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    src = os.path.join(HERE, src_name)
    out = os.path.join(out_dir, lib_name)
    if os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    cmd = ["/usr/bin/gcc", "-O2", "-fwrapv", "-fPIC", "-shared", "-fopenmp", "-std=c99", src, "-o", out, "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return out


def build_oracle(verbose=False):
    """The isothermal oracle (returned) and the gamma-law one."""
    _compile("cbdgam_2d_oracle.c", "liboracle_cbdgam.so", verbose)
    return _compile("cbdiso_2d_oracle.c", "liboracle_cbdiso.so", verbose)


def build_reference(verbose=False):
    script = os.path.join(HERE, "build_ref.sh")
    subprocess.run(["bash", script], check=True, capture_output=not verbose)


if __name__ == "__main__":
    print(build_oracle(verbose=True))
    build_reference(verbose=True)
