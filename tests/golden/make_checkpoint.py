"""
Generates checkpoint fixtures by running the reference driver itself
(sailfish.driver.simulate, CPU mode, its own cffi-built kernels):

  * chkpt_cbd_n24.pk / chkpt_cbd_n24_continued.npz: an isothermal
    circumbinary disk at 24^2 (theta = 1.8 as shipped), eccentric unequal
    binary, checkpoint event every 0.05 time units, fold 3, CFL 0.3;
  * chkpt_gam_n24.pk / chkpt_gam_n24_continued.npz: the gamma-law disk
    (cbdgam_2d) at 24^2 with alpha viscosity and cooling, the same binary
    and events, CFL 0.1;
  * for each, the reference's write_checkpoint output for its second
    checkpoint, copied here verbatim, and the state after the reference
    driver continues from that point for six more iterations (the dt rule
    of driver.py:508-510, dt recomputed every iteration), for the restart
    tests.

Usage (needs the reference tree, by default at /root/reference, or set
REFERENCE_ROOT); existing fixtures are kept unless --force is given:

    python tests/golden/make_checkpoint.py [--force]
"""

import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("REFERENCE_ROOT", "/root/reference")
CASES = {
    "cbd_n24": dict(params=dict(domain_radius=6.0, mach_number=10.0, mass_ratio=0.5, eccentricity=0.2, nu=0.001),
                    cfl=0.3, solver_options=dict(rk_order=2)),
    "gam_n24": dict(params=dict(eos="gamma-law", domain_radius=6.0, mass_ratio=0.5, eccentricity=0.2, alpha=0.1,
                                cooling_coefficient=1.0),
                    cfl=0.1, solver_options=dict()),
}


def make(tag, case, tmp):
    from sailfish.driver import DriverArgs, simulate, write_checkpoint
    from sailfish.event import LINEAR, Recurrence

    driver = DriverArgs(setup_name="circumbinary-disk", model_parameters=dict(case["params"]), resolution=24,
                        end_time=1.0, execution_mode="cpu", fold=3, cfl_number=case["cfl"],
                        events=dict(checkpoint=Recurrence(LINEAR, 0.05)),
                        solver_options=dict(case["solver_options"]))
    outdir = os.path.join(tmp, "out_" + tag)
    written = 0
    for name, number, state in simulate(driver):
        if name == "checkpoint":
            write_checkpoint(number, outdir, state)
            written += 1
            if written == 2:
                break
    src = os.path.join(outdir, f"chkpt.{number:04d}.pk")
    shutil.copyfile(src, os.path.join(HERE, f"chkpt_{tag}.pk"))
    # continue the same solver for six iterations with the driver's dt rule
    solver, mesh = state.solver, state.mesh
    dts = []
    for _ in range(6):
        dt = mesh.min_spacing(solver.time) / solver.maximum_wavespeed() * state.cfl_number
        solver.advance(dt)
        dts.append(dt)
    np.savez_compressed(os.path.join(HERE, f"chkpt_{tag}_continued.npz"), solution=solver.solution,
                        time=np.float64(solver.time), dts=np.array(dts), iteration=np.int64(state.iteration))
    print(f"wrote chkpt_{tag}.pk and chkpt_{tag}_continued.npz, iteration", state.iteration)


def main():
    force = "--force" in sys.argv
    tmp = tempfile.mkdtemp(prefix="sailfish_ref_")
    try:
        shutil.copytree(os.path.join(REF, "sailfish"), os.path.join(tmp, "sailfish"))
        sys.path.insert(0, tmp)
        os.environ.setdefault("CC", "/usr/bin/gcc")
        import sailfish.setups  # noqa: F401  (registers the setup classes)

        for tag, case in CASES.items():
            if force or not os.path.exists(os.path.join(HERE, f"chkpt_{tag}.pk")):
                make(tag, case, tmp)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main()
