"""
Generates tests/golden/chkpt_cbd_n24.pk and chkpt_cbd_n24_continued.npz by
running the reference driver itself (sailfish.driver.simulate, CPU mode,
its own cffi-built kernels):

  * a circumbinary disk at 24^2 (theta = 1.8 as shipped), eccentric unequal
    binary, checkpoint event every 0.05 time units, fold 3;
  * the reference's write_checkpoint output for its second checkpoint,
    copied here verbatim;
  * the state after the reference driver continues from that point for six
    more iterations (the dt rule of driver.py:508-510, dt recomputed every
    iteration), for the restart test.

Usage (needs the reference tree, by default at /root/reference, or set
REFERENCE_ROOT):

    python tests/golden/make_checkpoint.py
"""

import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("REFERENCE_ROOT", "/root/reference")
PARAMS = dict(domain_radius=6.0, mach_number=10.0, mass_ratio=0.5, eccentricity=0.2, nu=0.001)


def main():
    tmp = tempfile.mkdtemp(prefix="sailfish_ref_")
    try:
        shutil.copytree(os.path.join(REF, "sailfish"), os.path.join(tmp, "sailfish"))
        sys.path.insert(0, tmp)
        os.environ.setdefault("CC", "/usr/bin/gcc")
        import sailfish.setups  # noqa: F401  (registers the setup classes)
        from sailfish.driver import DriverArgs, simulate, write_checkpoint
        from sailfish.event import LINEAR, Recurrence

        driver = DriverArgs(setup_name="circumbinary-disk", model_parameters=dict(PARAMS), resolution=24,
                            end_time=1.0, execution_mode="cpu", fold=3, cfl_number=0.3,
                            events=dict(checkpoint=Recurrence(LINEAR, 0.05)), solver_options=dict(rk_order=2))
        outdir = os.path.join(tmp, "out")
        written = 0
        for name, number, state in simulate(driver):
            if name == "checkpoint":
                write_checkpoint(number, outdir, state)
                written += 1
                if written == 2:
                    break
        src = os.path.join(outdir, f"chkpt.{number:04d}.pk")
        shutil.copyfile(src, os.path.join(HERE, "chkpt_cbd_n24.pk"))
        # continue the same solver for six iterations with the driver's dt rule
        solver, mesh = state.solver, state.mesh
        dts = []
        for _ in range(6):
            dt = mesh.min_spacing(solver.time) / solver.maximum_wavespeed() * state.cfl_number
            solver.advance(dt)
            dts.append(dt)
        np.savez_compressed(os.path.join(HERE, "chkpt_cbd_n24_continued.npz"), solution=solver.solution,
                            time=np.float64(solver.time), dts=np.array(dts), iteration=np.int64(state.iteration))
        print("wrote chkpt_cbd_n24.pk and chkpt_cbd_n24_continued.npz, iteration", state.iteration)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main()
