"""
Restart compatibility with the reference driver's checkpoints: the fixture
chkpt_cbd_n24.pk was written by the reference's own write_checkpoint
(tests/golden/make_checkpoint.py), chkpt_cbd_n24_continued.npz holds the
state after the reference driver continued that run for six iterations.
"""

import os
import pickletools
import types

import numpy as np
import pytest

from cases import oh
from sailfish_b200.checkpoint import (DriverArgs, Recurrence, RecurringEvent, checkpoint_dict, load_checkpoint,
                                      write_checkpoint)
from sailfish_b200.mesh import PlanarCartesian2DMesh
from sailfish_b200.physics import PointMass, SinkModel
from sailfish_b200.setups import CircumbinaryDisk, find_setup_class

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CHKPT = os.path.join(GOLDEN, "chkpt_cbd_n24.pk")


def _continued():
    return np.load(os.path.join(GOLDEN, "chkpt_cbd_n24_continued.npz"))


def test_reference_checkpoint_loads_without_the_reference():
    c = load_checkpoint(CHKPT)
    assert c["setup_name"] == "circumbinary-disk" and c["solver"] == "cbdiso_2d"
    assert isinstance(c["mesh"], PlanarCartesian2DMesh) and c["mesh"].shape == (24, 24)
    assert c["solution"].shape == (24, 24, 3) and c["primitive"] is None
    assert isinstance(c["driver"], DriverArgs) and c["driver"].resolution == 24
    assert c["driver"].events["checkpoint"] == Recurrence(0, 0.05)
    assert isinstance(c["event_states"]["checkpoint"], RecurringEvent)
    assert all(isinstance(m, PointMass) and m.sink_model is SinkModel.TORQUE_FREE for m in c["point_masses"])
    assert c["iteration"] == int(_continued()["iteration"])
    setup = find_setup_class(c["setup_name"])(**c["model_parameters"])
    assert setup.model_parameter_dict() == c["model_parameters"]
    assert setup.dash_case_class_name() == c["setup_name"]
    # the stored point masses are the setup's at the stored time
    assert list(setup.point_masses(c["time"])) == list(c["point_masses"])


def _oracle_from_checkpoint(c):
    p = c["model_parameters"]
    m = c["mesh"]
    cfg = oh.Config(x0=m.x0, x1=m.x1, y0=m.y0, y1=m.y1, ni=m.ni, nj=m.nj, rk_order=c["solver_options"]["rk_order"],
                    plm_theta=1.8, eos_type=2, mach_number=p["mach_number"], nu=p["nu"],
                    buffer_is_enabled=p["buffer_is_enabled"], buffer_driving_rate=100.0, buffer_onset_width=1.0,
                    buffer_surface_density=p["initial_sigma"],
                    masses=oh.binary_masses(1.0, 1.0, p["mass_ratio"], p["eccentricity"], p["softening_length"],
                                            p["sink_model"], p["sink_rate"], p["sink_radius"]))
    return oh.OracleSolver(cfg, np.array(c["solution"]), time=c["time"])


def test_restarted_oracle_continues_like_the_reference_driver():
    """The checkpoint's time, solution and parameters, taken as restart()
    takes them, continue bit for bit like the reference run did."""
    c = load_checkpoint(CHKPT)
    ref = _continued()
    s = _oracle_from_checkpoint(c)
    for n in range(6):
        dt = c["mesh"].min_spacing() / s.maximum_wavespeed() * c["cfl_number"]
        assert dt == ref["dts"][n]
        s.advance(dt)
    assert s.time == float(ref["time"])
    np.testing.assert_array_equal(s.solution, ref["solution"])


def test_written_checkpoint_uses_the_reference_class_names_and_reads_back(tmp_path):
    c = load_checkpoint(CHKPT)
    setup = CircumbinaryDisk(**c["model_parameters"])
    solver = types.SimpleNamespace(time=c["time"], solution=c["solution"], primitive=None,
                                   options=dict(c["solver_options"], plm_theta=1.5, precision="fast"))
    name = write_checkpoint(7, str(tmp_path), solver, setup, c["mesh"], c["iteration"], c["timestep_dt"],
                            c["cfl_number"], c["timeseries"], c["event_states"], c["driver"])
    assert os.path.basename(name) == "chkpt.0007.pk"
    data = open(name, "rb").read()
    strings = [arg for op, arg, _ in pickletools.genops(data) if isinstance(arg, str)]
    assert "sailfish_b200" not in " ".join(strings) and "sailfish_b200.mesh" not in strings
    for module in ("sailfish.mesh", "sailfish.event", "sailfish.driver", "sailfish.physics.circumbinary"):
        assert module in strings
    back = load_checkpoint(name)
    want = checkpoint_dict(solver, setup, c["mesh"], c["iteration"], c["timestep_dt"], c["cfl_number"],
                           c["timeseries"], c["event_states"], c["driver"])
    assert set(back) == set(c) | {"b200_solver_options"} == set(want)
    assert back["solver_options"] == c["solver_options"]
    assert back["b200_solver_options"] == dict(plm_theta=1.5, precision="fast")
    for k in want:
        if isinstance(want[k], np.ndarray):
            np.testing.assert_array_equal(back[k], want[k])
        else:
            assert back[k] == want[k], k


@pytest.mark.gpu
def test_restart_continues_like_the_reference_driver():
    """restart() builds the B200 solver from the reference checkpoint; six
    more iterations with the driver's dt rule match the reference's own
    continuation (EXACT precision: identical up to the sign of zeros)."""
    from sailfish_b200.checkpoint import restart

    ref = _continued()
    solver, state = restart(CHKPT, solver_options=dict(plm_theta=1.8))
    assert state.iteration == int(ref["iteration"])
    for n in range(6):
        dt = state.mesh.min_spacing() / solver.maximum_wavespeed() * state.cfl_number
        assert dt == ref["dts"][n]
        solver.advance(dt)
    assert solver.time == float(ref["time"])
    np.testing.assert_array_equal(solver.solution, ref["solution"])


# ---------------------------------------------------------------------------
# the gamma-law solver's checkpoints (chkpt_gam_n24.pk, written by the
# reference driver running cbdgam_2d with alpha viscosity and cooling)
# ---------------------------------------------------------------------------

GAM_CHKPT = os.path.join(GOLDEN, "chkpt_gam_n24.pk")


def _gam_continued():
    return np.load(os.path.join(GOLDEN, "chkpt_gam_n24_continued.npz"))


def test_reference_gamma_checkpoint_loads():
    c = load_checkpoint(GAM_CHKPT)
    assert c["solver"] == "cbdgam_2d" and c["solution"].shape == (24, 24, 4)
    assert set(c["solver_options"]) == {"pressure_floor", "density_floor", "velocity_ceiling", "mach_ceiling"}
    setup = find_setup_class(c["setup_name"])(**c["model_parameters"])
    assert setup.solver == "cbdgam_2d" and setup.model_parameter_dict() == c["model_parameters"]
    assert list(setup.point_masses(c["time"])) == list(c["point_masses"])


def _gam_oracle_from_checkpoint(c):
    from oracle import host_gam as og

    p = c["model_parameters"]
    m = c["mesh"]
    setup = CircumbinaryDisk(**p)
    onset = [0.0] * 4
    setup.primitive(c["time"], [m.x1 - 0.1, 0.0], onset)
    o = c["solver_options"]
    cfg = og.GamConfig(m.x0, m.x1, m.y0, m.y1, m.ni, m.nj, gamma_law_index=p["gamma_law_index"], alpha=p["alpha"],
                       cooling_coefficient=p["cooling_coefficient"], constant_softening=p["constant_softening"],
                       buffer_is_enabled=p["buffer_is_enabled"], buffer_surface_density=onset[0],
                       buffer_surface_pressure=onset[3], pressure_floor=o["pressure_floor"],
                       density_floor=o["density_floor"], velocity_ceiling=o["velocity_ceiling"],
                       mach_ceiling=o["mach_ceiling"],
                       masses=oh.binary_masses(1.0, 1.0, p["mass_ratio"], p["eccentricity"], p["softening_length"],
                                               p["sink_model"], p["sink_rate"], p["sink_radius"]))
    return og.GamOracleSolver(cfg, np.array(c["solution"]), time=c["time"])


def test_restarted_gamma_oracle_continues_like_the_reference_driver():
    c = load_checkpoint(GAM_CHKPT)
    ref = _gam_continued()
    s = _gam_oracle_from_checkpoint(c)
    for n in range(6):
        dt = c["mesh"].min_spacing() / s.maximum_wavespeed() * c["cfl_number"]
        assert dt == ref["dts"][n]
        s.advance(dt)
    assert s.time == float(ref["time"])
    np.testing.assert_array_equal(s.solution, ref["solution"])


def test_written_gamma_checkpoint_keeps_the_gamma_options_apart(tmp_path):
    c = load_checkpoint(GAM_CHKPT)
    setup = CircumbinaryDisk(**c["model_parameters"])
    solver = types.SimpleNamespace(time=c["time"], solution=c["solution"], primitive=None,
                                   options=dict(c["solver_options"], plm_theta=1.5))
    name = write_checkpoint(3, str(tmp_path), solver, setup, c["mesh"], c["iteration"], c["timestep_dt"],
                            c["cfl_number"], c["timeseries"], c["event_states"], c["driver"])
    back = load_checkpoint(name)
    assert back["solver"] == "cbdgam_2d"
    assert back["solver_options"] == c["solver_options"]
    assert back["b200_solver_options"] == dict(plm_theta=1.5)
    np.testing.assert_array_equal(back["solution"], c["solution"])


@pytest.mark.gpu
def test_gamma_restart_continues_like_the_reference_driver():
    """restart() builds the gamma-law B200 solver from the reference's
    checkpoint; six more iterations with the driver's dt rule match the
    reference's own continuation."""
    from sailfish_b200.checkpoint import restart

    ref = _gam_continued()
    solver, state = restart(GAM_CHKPT)
    assert type(solver).__module__ == "sailfish_b200.cbdgam_2d"
    for n in range(6):
        dt = state.mesh.min_spacing() / solver.maximum_wavespeed() * state.cfl_number
        assert dt == pytest.approx(ref["dts"][n], rel=1e-14)
        solver.advance(dt)
    assert solver.time == pytest.approx(float(ref["time"]), rel=1e-15)
    got, want = solver.solution, ref["solution"]
    for q in range(4):
        assert np.abs(got[..., q] - want[..., q]).max() <= 1e-13 * np.abs(want[..., q]).max()
