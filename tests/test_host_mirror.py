"""
Host-side mirror of the reference's solver interface (no GPU needed): Kepler
orbits, physics point masses, mesh, setups and initial data, the solver
registry and the constructor's validation errors.
"""

import math

import numpy as np
import pytest

from cases import load
from oracle import host as oh
from sailfish_b200 import SolverInitializationError, make_solver
from sailfish_b200.cbdiso_2d import RK_WEIGHTS, initial_condition
from sailfish_b200.kepler import OrbitalElements
from sailfish_b200.mesh import PlanarCartesian2DMesh
from sailfish_b200.physics import EquationOfState, Physics, PointMass, SinkModel, ViscosityModel
from sailfish_b200.setups import BinaryBondi, CircumbinaryDisk, KitpCodeComparison, SetupError


@pytest.mark.parametrize("q,e", [(1.0, 0.0), (0.5, 0.1), (0.3, 0.5), (0.9, 0.3)])
def test_kepler_state_matches_oracle_bitwise(q, e):
    orb = OrbitalElements(1.0, 1.0, q, e)
    for t in np.linspace(0.0, 40.0, 97):
        a, b = orb.orbital_state(float(t))
        c, d = oh.kepler_state(float(t), 1.0, 1.0, q, e)
        assert (a.mass, a.position_x, a.position_y, a.velocity_x, a.velocity_y) == tuple(c)
        assert (b.mass, b.position_x, b.position_y, b.velocity_x, b.velocity_y) == tuple(d)


def test_kepler_newton_error_behaviour():
    with pytest.raises(ValueError):
        OrbitalElements(1.0, 1.0, 1.0, 1.5).orbital_state(1.0)


def test_point_masses_normalisation():
    assert Physics().point_masses(0.0) == (PointMass(), PointMass())
    one = PointMass(mass=1.0)
    assert Physics(point_mass_function=lambda t: one).point_masses(0.0) == (one, PointMass())
    assert Physics(point_mass_function=lambda t: [one]).point_masses(0.0) == (one, PointMass())
    with pytest.raises(ValueError):
        Physics(point_mass_function=lambda t: [one, one, one]).point_masses(0.0)


def test_mesh():
    m = PlanarCartesian2DMesh.centered_square(8.0, 256)
    assert m.shape == (256, 256) and m.dx == 16.0 / 256 and m.min_spacing() == m.dx
    assert m.cell_coordinates(0, 0) == (-8.0 + 0.5 * m.dx, -8.0 + 0.5 * m.dy)
    r = PlanarCartesian2DMesh.centered_rectangle(1.0, 32, 2)
    assert r.shape == (64, 32)


@pytest.mark.parametrize("name", ["cbd_t15_n64", "cbd_t18_48x40_ecc", "bondi_t18_64x32"])
def test_vectorised_initial_condition_is_bitwise_the_per_zone_loop(name):
    d = load(name)
    meta = d["meta"]
    x0, y0, x1, y1, ni, nj = meta["mesh"]
    mesh = PlanarCartesian2DMesh(x0, y0, x1, y1, ni, nj)
    if meta["setup"] == "binary-bondi":
        setup = BinaryBondi(**meta["params"])
    else:
        setup = CircumbinaryDisk(**meta["params"])
    ic = initial_condition(setup, mesh, 0.0)
    assert np.array_equal(ic, d["ic"])


def test_kitp_initial_condition_per_zone_matches_reference():
    d = load("kitp_t18_n64_rk3_p2")
    setup = KitpCodeComparison(**d["meta"]["params"])
    assert not hasattr(setup, "primitive_array")
    mesh = setup.mesh(64)
    assert np.array_equal(initial_condition(setup, mesh, 0.0), d["ic"])


def test_setup_parameter_types_are_checked():
    with pytest.raises(SetupError):
        CircumbinaryDisk(mass_ratio=1)
    with pytest.raises(SetupError):
        CircumbinaryDisk(not_a_parameter=1.0)


def test_rk_stage_times_follow_the_reference_update():
    """cbdiso_2d.py:239: time = time0 * a + (time + dt) * (1 - a) per stage."""
    t0, dt = 0.123456789, 0.0041
    t = t0
    for a in RK_WEIGHTS[2]:
        t = t0 * a + (t + dt) * (1.0 - a)
    assert t == t0 * 0.5 + ((t0 + dt) + dt) * 0.5


def _cbd(**kw):
    setup = CircumbinaryDisk(domain_radius=8.0)
    physics = setup.physics
    physics.update(kw)
    return setup, physics


@pytest.mark.parametrize("change,msg", [
    (dict(viscosity_model=ViscosityModel.CONSTANT_ALPHA), "constant-nu"),
    (dict(eos_type=EquationOfState.GAMMA_LAW), "isothermal"),
    (dict(cooling_coefficient=1.0), "cooling"),
    (dict(constant_softening=False), "softening"),
])
def test_constructor_validation_errors(change, msg):
    setup, physics = _cbd(**change)
    with pytest.raises(SolverInitializationError, match=msg):
        make_solver("cbdiso_2d", physics, {}, setup=setup, mesh=setup.mesh(16))


def test_constructor_rejects_non_cartesian_mesh_and_unknown_option():
    setup, physics = _cbd()
    with pytest.raises(SolverInitializationError, match="cartesian"):
        make_solver("cbdiso_2d", physics, {}, setup=setup, mesh=(16, 16))
    with pytest.raises(SolverInitializationError):
        make_solver("cbdiso_2d", physics, dict(no_such_option=1), setup=setup, mesh=setup.mesh(16))
    with pytest.raises(SolverInitializationError, match="rk_order"):
        make_solver("cbdiso_2d", physics, dict(rk_order=4), setup=setup, mesh=setup.mesh(16))


def test_sink_model_enum_values_match_kernel_codes():
    assert [m.value for m in SinkModel] == [0, 1, 2, 3]
    assert oh.SINK_MODELS == dict(inactive=0, acceleration_free=1, torque_free=2, force_free=3)
