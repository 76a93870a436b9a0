"""
Parity at the plain-solver throughput configuration: the circumbinary disk of
config 0 (theta 1.5, RK2, CFL 0.3, seeded noise, per-step mdot / torque
reductions) at 1024^2, 2048^2 and 4096^2, 1000 steps, against fixtures the
reference's own solver wrote (tests/golden/make_golden.py, LONG_CASES: its
cbdiso_2d kernels in OpenMP mode, driven by its solver adapter with the
driver's dt rule, cbdiso_2d.c:385-604, cbdiso_2d.py:536-551,
driver.py:508-511).

Both loops are held to the bar (1e-12 per step, 1e-10 after 1000 steps):
  * `Solver.run`, the device-resident loop the benchmark times (dt and the
    Kepler orbit on the device, CUDA graphs, face cache on, EXACT);
  * the host-driven loop of the reference's driver (`maximum_wavespeed`,
    `advance`, `reductions` every step).
Compared: the dt and reductions series (each column against its largest
magnitude over the run), the state after the first step and after the last
(1-in-16 subsample, each field against its maximum magnitude), and per-row
maximum magnitudes and sums of each field of the last state (a sum against
the row's sum of magnitudes).

Also here: batched disks at the corners of the many-disk workload's
parameter box (q 0.1 / 1, e 0.5 / 0, Mach 40 / 10, nu 1e-2 / 1e-4; 128^2 and
1024^2) against the CPU oracle for 50 steps.
"""

import os

import numpy as np
import pytest

from cases import GOLDEN, diagnostics, load, oracle_config
from oracle import host as oh

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sailfish_b200 import make_solver  # noqa: E402
from sailfish_b200.cbdiso_2d import initial_condition  # noqa: E402
from sailfish_b200.setups import CircumbinaryDisk  # noqa: E402

STEP_TOL = 1e-12
RUN_TOL = 1e-10


def _fixture(n):
    name = f"config1_t15_n{n}"
    if not os.path.exists(os.path.join(GOLDEN, name + ".npz")):
        pytest.skip(f"fixture {name} not generated")
    return load(name)


def _solver(d):
    meta = d["meta"]
    n = meta["resolution"]
    setup = CircumbinaryDisk(**meta["params"])
    mesh = setup.mesh(n)
    physics = setup.physics
    physics["diagnostics"] = diagnostics(meta)
    prim = initial_condition(setup, mesh, 0.0)
    stride = prim.shape[0] // d["ic"].shape[0]
    assert np.array_equal(prim[::stride, ::stride], d["ic"])
    prim[..., 0] += oh.seeded_noise(n, n, meta["seed"])
    return make_solver("cbdiso_2d", physics, dict(rk_order=2, plm_theta=meta["theta"]), setup=setup, mesh=mesh,
                       solution=prim), mesh


def _field_error(a, b):
    return max(float(np.abs(a[..., q] - b[..., q]).max() / np.abs(b[..., q]).max()) for q in range(3))


def _check_series(dts, series, d):
    want_dt = d["dts"]
    assert np.abs(np.array(dts) - want_dt).max() <= RUN_TOL * want_dt.max()
    want = d["series"].real  # time, mdot1, mdot2, torque
    got = np.array(series, dtype=float)
    assert got.shape == want.shape
    for c in range(want.shape[1]):
        scale = np.abs(want[:, c]).max()
        err = np.abs(got[:, c] - want[:, c]).max() / scale
        assert err <= RUN_TOL, (c, err)
    # the first step's values at the per-step bar
    for c in range(want.shape[1]):
        assert abs(got[0, c] - want[0, c]) <= STEP_TOL * np.abs(want[:, c]).max(), c


def _check_last(last, d):
    assert _field_error(last[::16, ::16], d["last_sub"]) <= RUN_TOL
    row_max = np.abs(last).max(axis=1)
    for q in range(3):
        assert np.abs(row_max[:, q] - d["last_row_max"][:, q]).max() <= RUN_TOL * d["last_row_max"][:, q].max()
    row_sum = last.sum(axis=1)
    assert np.all(np.abs(row_sum - d["last_row_sum"]) <= RUN_TOL * d["last_row_abs"])


@pytest.mark.slow
@pytest.mark.parametrize("n", [1024, 2048, 4096])
def test_device_loop_against_reference_1000_steps(n):
    d = _fixture(n)
    steps = d["meta"]["steps"]
    s, _ = _solver(d)
    rows = s.run(1, cfl=0.3)
    assert _field_error(s.solution[::16, ::16], d["first_sub"]) <= STEP_TOL
    rows += s.run(steps - 1, cfl=0.3)
    assert len(rows) == steps
    _check_series([r[-1] for r in rows], [r[:-1] for r in rows], d)
    assert s.time == pytest.approx(float(d["time"]), rel=RUN_TOL)
    _check_last(s.solution, d)
    assert s.maximum_wavespeed() == pytest.approx(float(d["max_wavespeed"]), rel=RUN_TOL)


@pytest.mark.slow
@pytest.mark.parametrize("n", [1024, 2048, 4096])
def test_host_loop_against_reference_1000_steps(n):
    d = _fixture(n)
    steps = d["meta"]["steps"]
    s, mesh = _solver(d)
    dts, series = [], []
    for k in range(steps):
        dt = mesh.min_spacing() / s.maximum_wavespeed() * 0.3
        s.advance(dt)
        dts.append(dt)
        series.append(s.reductions())
        if k == 0:
            assert _field_error(s.solution[::16, ::16], d["first_sub"]) <= STEP_TOL
    _check_series(dts, series, d)
    _check_last(s.solution, d)


# ---------------------------------------------------------------------------
# batched disks at the corners of the many-disk parameter box
# ---------------------------------------------------------------------------

CORNERS = [  # (size, q, e, Mach, nu)
    (128, 0.1, 0.5, 40.0, 1e-2),
    (1024, 0.1, 0.5, 40.0, 1e-2),
    (128, 1.0, 0.0, 10.0, 1e-4),
    (1024, 0.1, 0.5, 10.0, 1e-4),
]
BATCH_DIAGS = [dict(quantity="time"), dict(quantity="mdot", which_mass=1, accretion=True),
               dict(quantity="mdot", which_mass=2, accretion=True),
               dict(quantity="torque", which_mass="both", gravity=True)]


@pytest.mark.slow
def test_batched_extreme_disks_against_oracle():
    from sailfish_b200.batched import BatchedSolver, Disk

    steps = 50
    disks, metas = [], []
    rng = np.random.default_rng(77)
    for n, q, e, mach, nu in CORNERS:
        params = dict(domain_radius=8.0, mach_number=mach, mass_ratio=q, eccentricity=e, nu=nu)
        setup = CircumbinaryDisk(**params)
        mesh = setup.mesh(n)
        prim = initial_condition(setup, mesh, 0.0)
        prim[..., 0] += 1e-3 * rng.uniform(-1.0, 1.0, size=(n, n))
        disks.append(Disk(setup, mesh, prim))
        metas.append(dict(setup="circumbinary-disk", mesh=[-8.0, -8.0, 8.0, 8.0, n, n], rk=2, theta=1.5,
                          params=params))
    b = BatchedSolver(disks, diagnostics=BATCH_DIAGS)
    got_series = b.run(steps, cfl=0.3, graph=True, steps_per_graph=10)
    for i, (disk, meta) in enumerate(zip(disks, metas)):
        cfg = oracle_config(meta)
        o = oh.OracleSolver(cfg, disk.solution, 0.0, oh.Kernels("oracle", 1.5, threads="omp"))
        dts, want = oh.run(o, steps, cfl=0.3, diagnostics=BATCH_DIAGS)
        got = np.array(got_series[i], dtype=float)
        np.testing.assert_allclose(got[:, -1], dts, rtol=RUN_TOL, atol=0)
        want = np.array(want).real
        for c in range(want.shape[1]):
            scale = np.abs(want[:, c]).max()
            assert np.abs(got[:, c] - want[:, c]).max() <= RUN_TOL * scale, (i, c)
        err = _field_error(b.solution(i), o.solution)
        assert err <= RUN_TOL, (i, err)
