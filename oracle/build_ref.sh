#!/usr/bin/env bash
# Builds the reference's own cbdiso_2d kernels (sailfish/solvers/cbdiso_2d.c,
# read in place from the reference tree) into oracle/_ref/ as shared
# libraries, for use as a test-only checker and as the timed CPU baseline.
#
#   libref_t18_cpu.so  theta = 1.8 (the source as written), serial
#   libref_t18_omp.so  theta = 1.8, OpenMP
#   libref_t15_cpu.so  theta = 1.5 (line `#define PLM_THETA 1.8` rewritten
#   libref_t15_omp.so  on the fly, as a solver option would), serial / OpenMP
#   libref_gam_cpu.so  the gamma-law kernels (sailfish/solvers/cbdgam_2d.c,
#   libref_gam_omp.so  theta 1.5 as written), serial / OpenMP
#
# Flags mirror what cffi uses for sailfish's JIT build (-O2 -fwrapv, plus
# -fopenmp -std=c99 in omp mode; sailfish/kernel/system.py:78-81). The
# reference source is never copied into the repository.
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
ref_root="${REFERENCE_ROOT:-/root/reference}"
src="$ref_root/sailfish/solvers/cbdiso_2d.c"
out="$here/_ref"
if [[ ! -f "$src" ]]; then
    echo "build_ref.sh: reference source not found at $src; skipping" >&2
    exit 0
fi
mkdir -p "$out"
cc=/usr/bin/gcc
for theta in 1.8 1.5; do
    tag="t${theta/./}"
    for mode in cpu omp; do
        if [[ $mode == omp ]]; then flags="-DEXEC_MODE=1 -fopenmp -std=c99"; else flags="-DEXEC_MODE=0"; fi
        sed "s/^#define PLM_THETA 1\.8\$/#define PLM_THETA $theta/" "$src" \
            | $cc -O2 -fwrapv -fPIC -shared $flags -include "$here/ref_macros.h" -x c - \
                  -o "$out/libref_${tag}_${mode}.so" -lm
    done
done
grep -q "^#define PLM_THETA 1\.8$" "$src" || { echo "build_ref.sh: PLM_THETA line not found" >&2; exit 1; }
# the gamma-law kernels (sailfish/solvers/cbdgam_2d.c, theta 1.5 as written)
gsrc="$ref_root/sailfish/solvers/cbdgam_2d.c"
if [[ -f "$gsrc" ]]; then
    for mode in cpu omp; do
        if [[ $mode == omp ]]; then flags="-DEXEC_MODE=1 -fopenmp -std=c99"; else flags="-DEXEC_MODE=0"; fi
        $cc -O2 -fwrapv -fPIC -shared $flags -include "$here/ref_macros.h" -x c "$gsrc" \
            -o "$out/libref_gam_${mode}.so" -lm
    done
fi
echo "built reference kernels into $out"
