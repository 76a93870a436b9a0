"""
Generates the golden fixtures in this directory by running the reference
sailfish cbdiso_2d and cbdgam_2d solvers themselves (CPU mode, their own
cffi-built kernels).

Usage (needs the reference tree, by default at /root/reference, or set
REFERENCE_ROOT):

    python tests/golden/make_golden.py            # all cases
    python tests/golden/make_golden.py CASE ...   # selected cases

The reference package is copied to a temporary directory first, because its
kernel loader writes build products next to its own sources, and so that the
PLM limiter parameter can be set: the reference fixes it at compile time
(`#define PLM_THETA 1.8`, sailfish/solvers/cbdiso_2d.c:11), so the copy's line
is rewritten for the theta = 1.5 cases. Each case runs in a fresh interpreter.

Each fixture holds: the setup-generated initial primitive state (before the
seeded noise), the noise seed, the time step sequence chosen by the driver's
CFL rule (driver.py:508-510), the state after the first and after the last
step, the wavespeed maximum after the last step, and the reductions time
series (cbdiso_2d.py:370-503) after every step.

The long cases (`LONG_CASES`: the plain-solver throughput configuration at
1024^2, 2048^2 and 4096^2, 1000 RK2 steps each) run the reference's kernels
in its OpenMP mode (`mode="omp"`, one zone per loop iteration, so the results
are the serial build's bit for bit) and store, instead of whole states, the
full dt and reductions series, a 1-in-16 subsample of the states after the
first and the last step, and per-row (fixed i) maximum magnitudes and sums of
each field of the last state. They take about 5 min, 15 min and an hour on
8 cores, and run only when named:

    python tests/golden/make_golden.py config1_t15_n1024 config1_t15_n2048 config1_t15_n4096
"""

import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("REFERENCE_ROOT", "/root/reference")

KITP_DIAG = [
    dict(quantity="time"),
    dict(quantity="mdot", which_mass=1, accretion=True),
    dict(quantity="mdot", which_mass=2, accretion=True),
    dict(quantity="torque", which_mass="both", gravity=True),
    dict(quantity="torque", which_mass="both", gravity=True, radial_cut=(1.0, 8.0)),
    dict(quantity="sigma_m1"),
    dict(quantity="eccentricity_vector", radial_cut=(1.0, 6.0)),
]
FORCE_DIAG = [
    dict(quantity="time"),
    dict(quantity="mdot", which_mass=1, accretion=True),
    dict(quantity="fx", which_mass=1, gravity=True),
    dict(quantity="fy", which_mass=2, gravity=True),
    dict(quantity="fx", which_mass=2, accretion=True),
    dict(quantity="angular_momentum", radial_cut=(0.5, 4.0)),
    dict(quantity="mass"),
    dict(quantity="power", which_mass=1, gravity=True),
    dict(quantity="power", which_mass=2, gravity=True),
]
GAM_DIAG = [
    dict(quantity="time"),
    dict(quantity="mdot", which_mass=1, accretion=True),
    dict(quantity="mdot", which_mass=2, accretion=True),
    dict(quantity="torque", which_mass="both", gravity=True),
    dict(quantity="torque", which_mass=1, gravity=True, radial_cut=(1.0, 4.0)),
    dict(quantity="sigma_m1"),
    dict(quantity="eccentricity_vector", radial_cut=(1.0, 4.0)),
]
CBD_DIAG = [
    dict(quantity="time"),
    dict(quantity="mdot", which_mass=1, accretion=True),
    dict(quantity="mdot", which_mass=2, accretion=True),
    dict(quantity="torque", which_mass="both", gravity=True),
]

# name -> case description
CASES = {
    # config-0 physics at 64^2, theta = 1.5 (patched), torque-free sinks
    "cbd_t15_n64": dict(
        setup="circumbinary-disk", theta=1.5, resolution=64, steps=20, seed=1, patches=1, rk=2,
        params=dict(domain_radius=8.0, mach_number=10.0, mass_ratio=1.0, eccentricity=0.0, sink_rate=10.0,
                    sink_radius=0.05, softening_length=0.05, nu=0.001),
        diagnostics=CBD_DIAG),
    # same at theta = 1.8 with three patches (exercises the reference's guard exchange)
    "cbd_t18_n64_p3": dict(
        setup="circumbinary-disk", theta=1.8, resolution=64, steps=20, seed=2, patches=3, rk=2,
        params=dict(domain_radius=8.0, mach_number=10.0, mass_ratio=1.0, eccentricity=0.0, sink_rate=10.0,
                    sink_radius=0.05, softening_length=0.05, nu=0.001),
        diagnostics=CBD_DIAG),
    # eccentric, unequal binary; acceleration-free sinks; RK3; two patches; kitp diagnostics
    # (no added noise: the kitp cavity density is 1e-5, below the noise amplitude)
    "kitp_t18_n64_rk3_p2": dict(
        setup="kitp-code-comparison", theta=1.8, resolution=64, steps=15, seed=None, patches=2, rk=3,
        params=dict(eccentricity=0.3, mass_ratio=0.5, nu=0.001, sink_model="acceleration_free"),
        diagnostics=KITP_DIAG),
    # non-square mesh (48 x 40 zones on [-8, 8] x [-6, 6]), eccentric binary, torque-free sinks
    "cbd_t18_48x40_ecc": dict(
        setup="circumbinary-disk", theta=1.8, mesh=(-8.0, -6.0, 8.0, 6.0, 48, 40), steps=15, seed=7,
        patches=1, rk=2,
        params=dict(domain_radius=8.0, eccentricity=0.3, mass_ratio=0.5, nu=0.001),
        diagnostics=KITP_DIAG),
    # force-free sinks, no viscosity, buffer off, RK1, force / power diagnostics
    "kitp_t15_n56_rk1_forcefree": dict(
        setup="kitp-code-comparison", theta=1.5, resolution=56, steps=15, seed=None, patches=1, rk=1,
        params=dict(eccentricity=0.1, mass_ratio=0.7, nu=0.0, sink_model="force_free", buffer_is_enabled=False),
        diagnostics=FORCE_DIAG),
    # inactive sinks on a circumbinary disk, Mach 20, theta = 1.8
    "cbd_t18_n48_inactive": dict(
        setup="circumbinary-disk", theta=1.8, resolution=48, steps=12, seed=5, patches=1, rk=2,
        params=dict(domain_radius=6.0, mach_number=20.0, mass_ratio=0.4, eccentricity=0.2, sink_model="inactive",
                    nu=0.0005),
        diagnostics=CBD_DIAG),
    # globally isothermal EOS (eos_type 1) with a binary in a wind
    "bondi_t18_64x32": dict(
        setup="binary-bondi", theta=1.8, resolution=32, steps=12, seed=6, patches=1, rk=2,
        params=dict(aspect=2, height=1.0, sound_speed=1.0, wind_vel=1.0, bh_sep=0.25, sink_rate=100.0,
                    sink_model="acceleration_free"),
        diagnostics=[dict(quantity="time"), dict(quantity="mdot", which_mass=1, accretion=True),
                     dict(quantity="mdot", which_mass=2, accretion=True)]),
    # no point masses at all (eos 1, zero-mass branch of the potential)
    "explosion_t15_n40": dict(
        setup="cylindrical-explosion", theta=1.5, resolution=40, steps=10, seed=None, patches=1, rk=2,
        params=dict(), diagnostics=[dict(quantity="time"), dict(quantity="mass")]),
    # gamma-law (cbdgam_2d, theta 1.5 as the reference fixes it): alpha viscosity, constant softening
    "gam_n64": dict(
        setup="circumbinary-disk", solver="cbdgam_2d", noise="relative", theta=1.5, resolution=64, steps=20, seed=11, patches=1,
        cfl=0.1, params=dict(eos="gamma-law", domain_radius=8.0, mass_ratio=1.0, eccentricity=0.0, alpha=0.1),
        diagnostics=CBD_DIAG),
    # eccentric, unequal, cooling, acceleration-free sinks, two patches, all four gamma-law diagnostics
    "gam_n48_cool_p2": dict(
        setup="circumbinary-disk", solver="cbdgam_2d", noise="relative", theta=1.5, resolution=48, steps=15, seed=12, patches=2,
        cfl=0.1, params=dict(eos="gamma-law", domain_radius=6.0, mass_ratio=0.5, eccentricity=0.3, alpha=0.05,
                             cooling_coefficient=10.0, sink_model="acceleration_free"),
        diagnostics=GAM_DIAG),
    # softening that follows the disk height, force-free sinks, inviscid, no buffer
    "gam_n40_soft_inviscid": dict(
        setup="circumbinary-disk", solver="cbdgam_2d", noise="relative", theta=1.5, resolution=40, steps=12, seed=13, patches=1,
        cfl=0.1, params=dict(eos="gamma-law", domain_radius=4.0, mass_ratio=0.8, eccentricity=0.1, alpha=0.0,
                             constant_softening=False, sink_model="force_free", buffer_is_enabled=False),
        diagnostics=GAM_DIAG),
    # 256^2, 60 steps (state stored subsampled)
    "gam_n256": dict(
        setup="circumbinary-disk", solver="cbdgam_2d", noise="relative", theta=1.5, resolution=256, steps=60, seed=14, patches=1,
        cfl=0.1, params=dict(eos="gamma-law", domain_radius=8.0, mass_ratio=1.0, eccentricity=0.0, alpha=0.1),
        diagnostics=CBD_DIAG, store="subsample8"),
    # config 0 as stated: 256^2, theta = 1.5, 100 steps (state stored subsampled, see `store`)
    "config0_t15_n256": dict(
        setup="circumbinary-disk", theta=1.5, resolution=256, steps=100, seed=0, patches=1, rk=2,
        params=dict(domain_radius=8.0, mach_number=10.0, mass_ratio=1.0, eccentricity=0.0, sink_rate=10.0,
                    sink_radius=0.05, softening_length=0.05, nu=0.001),
        diagnostics=CBD_DIAG, store="subsample8"),
}

# the plain-solver throughput configuration: config-0 physics, 1000 steps (see the module docstring)
CONFIG1_PARAMS = dict(domain_radius=8.0, mach_number=10.0, mass_ratio=1.0, eccentricity=0.0, sink_rate=10.0,
                      sink_radius=0.05, softening_length=0.05, nu=0.001)
LONG_CASES = {
    f"config1_t15_n{n}": dict(
        setup="circumbinary-disk", theta=1.5, resolution=n, steps=1000, seed=0, patches=1, rk=2,
        params=CONFIG1_PARAMS, diagnostics=CBD_DIAG, store="long16", mode="omp")
    for n in (1024, 2048, 4096)
}
CASES.update(LONG_CASES)


def run_case(name, out_path):
    import numpy as np

    case = CASES[name]
    tmp = tempfile.mkdtemp(prefix="sailfish_ref_")
    try:
        shutil.copytree(os.path.join(REF, "sailfish"), os.path.join(tmp, "sailfish"))
        src = os.path.join(tmp, "sailfish", "solvers", "cbdiso_2d.c")
        text = open(src).read()
        line = "#define PLM_THETA 1.8\n"
        assert line in text
        text = text.replace(line, f"#define PLM_THETA {case['theta']}\n")
        open(src, "w").write(text)
        sys.path.insert(0, tmp)
        os.environ.setdefault("CC", "/usr/bin/gcc")
        # the system compiler links OpenMP (the interpreter's default LDSHARED may not)
        os.environ.setdefault("LDSHARED", "/usr/bin/gcc -shared")
        mode = case.get("mode", "cpu")
        if mode == "omp":
            from sailfish.kernel.system import configure_build

            configure_build(enable_openmp=True, execution_mode="omp")
        from sailfish.setup_base import SetupBase
        import sailfish.setups  # noqa: F401  (registers the setup classes)
        from sailfish.mesh import PlanarCartesian2DMesh
        from sailfish.solvers import make_solver

        setup = SetupBase.find_setup_class(case["setup"])(**case["params"])
        if "mesh" in case:
            mesh = PlanarCartesian2DMesh(*case["mesh"])
        else:
            mesh = setup.mesh(case["resolution"])
        ni, nj = mesh.shape
        solver_name = case.get("solver", "cbdiso_2d")
        nq = 4 if solver_name == "cbdgam_2d" else 3
        ic = np.zeros((ni, nj, nq))
        for i in range(ni):
            for j in range(nj):
                setup.primitive(0.0, mesh.cell_coordinates(i, j), ic[i, j])
        prim = ic.copy()
        if case["seed"] is not None:
            rng = np.random.default_rng(case["seed"])
            noise = 1e-3 * rng.uniform(-1.0, 1.0, size=(ni, nj))
            if case.get("noise") == "relative":
                # the gamma-law disk's cavity density (~1e-4) is below the absolute amplitude
                prim[..., 0] *= 1.0 + noise
            else:
                prim[..., 0] += noise
        physics = setup.physics
        physics["diagnostics"] = case["diagnostics"]
        options = dict(rk_order=case["rk"]) if solver_name == "cbdiso_2d" else dict()
        solver = make_solver(
            solver_name, physics, options, setup=setup, mesh=mesh, time=0.0, solution=prim,
            num_patches=case["patches"], mode=mode)
        cfl = case.get("cfl", 0.3)
        dts, series, first = [], [], None
        for n in range(case["steps"]):
            dt = mesh.min_spacing(0.0) / solver.maximum_wavespeed() * cfl
            solver.advance(dt)
            dts.append(dt)
            series.append([complex(v) for v in solver.reductions()])
            if n == 0:
                first = solver.solution
            if case.get("store") == "long16" and (n + 1) % 50 == 0:
                print(f"{name}: step {n + 1} t={solver.time:.6f} dt={dt:.6e}", file=sys.stderr, flush=True)
        last = solver.solution
        ws = solver.maximum_wavespeed()
        meta = dict(case, name=name, mesh=list(mesh), cfl=cfl, rk=case.get("rk", 2))
        out = dict(meta=json.dumps(meta), ic=ic, dts=np.array(dts), series=np.array(series, dtype=complex),
                   max_wavespeed=np.float64(ws), time=np.float64(solver.time))
        if case.get("store") == "subsample8":
            out.update(first_sub=first[::8, ::8], last_sub=last[::8, ::8],
                       last_sums=np.array([last[..., q].sum() for q in range(nq)]),
                       ic=ic[::8, ::8])
        elif case.get("store") == "long16":
            out.update(first_sub=first[::16, ::16], last_sub=last[::16, ::16],
                       last_row_max=np.abs(last).max(axis=1), last_row_sum=last.sum(axis=1),
                       last_row_abs=np.abs(last).sum(axis=1),
                       last_sums=np.array([last[..., q].sum() for q in range(nq)]),
                       ic=ic[::16, ::16])
        else:
            out.update(first=first, last=last)
        np.savez_compressed(out_path, **out)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def main(argv):
    if len(argv) >= 2 and argv[0] == "--one":
        run_case(argv[1], argv[2])
        return
    names = argv or [n for n in CASES if n not in LONG_CASES]
    for name in names:
        out = os.path.join(HERE, f"{name}.npz")
        subprocess.run([sys.executable, __file__, "--one", name, out], check=True)
        print(f"wrote {out} ({os.path.getsize(out) // 1024} KiB)")


if __name__ == "__main__":
    main(sys.argv[1:])
