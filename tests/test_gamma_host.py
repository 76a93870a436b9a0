"""
Host side of the gamma-law path, without a GPU: the gamma-law branch of the
circumbinary setup against the oracle's restatement, the solver's
validation (the reference's errors, raised before any device work), and the
argument checks of the gamma-law C-ABI entry points (which return before
touching the device).
"""

import ctypes

import numpy as np
import pytest

from oracle import host_gam as og
from sailfish_b200 import SolverInitializationError, _capi, make_solver
from sailfish_b200.mesh import PlanarCartesian2DMesh
from sailfish_b200.physics import EquationOfState, ViscosityModel
from sailfish_b200.setups import CircumbinaryDisk, SetupError


def test_gamma_setup_primitive_matches_restatement():
    setup = CircumbinaryDisk(eos="gamma-law")
    out = [0.0] * 4
    for x, y in ((0.3, -1.2), (0.0, 0.0), (7.9, 7.9), (-0.05, 0.02), (1.0, 0.0)):
        setup.primitive(0.0, (x, y), out)
        assert tuple(out) == og.gamma_disk_primitive(x, y)


def test_gamma_setup_primitive_array_equals_zone_wise():
    """The vectorised initial data equals the per-zone setup formula (the
    reference's initial_condition loop) bit for bit, on random points, the
    origin and a 96^2 mesh."""
    setup = CircumbinaryDisk(eos="gamma-law", initial_pressure=3e-3, softening_length=0.1)
    rng = np.random.default_rng(5)
    x, y = rng.uniform(-8, 8, (2, 400, 7))
    x[0, 0] = y[0, 0] = 0.0
    arr = setup.primitive_array(0.0, x, y)
    assert arr.shape == (400, 7, 4)
    out = [0.0] * 4
    for i in range(400):
        for j in range(7):
            setup.primitive(0.0, (x[i, j], y[i, j]), out)
            assert tuple(arr[i, j]) == tuple(out), (i, j)
    from sailfish_b200.cbdgam_2d import initial_condition

    mesh = setup.mesh(96)
    fast = initial_condition(setup, mesh, 0.0)
    for i in (0, 17, 47, 48, 95):
        for j in (0, 5, 48, 95):
            setup.primitive(0.0, mesh.cell_coordinates(i, j), out)
            assert tuple(fast[i, j]) == tuple(out)


def test_gamma_setup_physics_and_solver():
    setup = CircumbinaryDisk(eos="gamma-law", alpha=0.0, cooling_coefficient=2.0)
    p = setup.physics
    assert p["eos_type"] == EquationOfState.GAMMA_LAW
    assert p["viscosity_model"] == ViscosityModel.NONE
    assert p["buffer_driving_rate"] == 1000.0 and p["buffer_onset_width"] == 0.1
    assert p["cooling_coefficient"] == 2.0 and p["gamma_law_index"] == 5.0 / 3.0
    assert setup.solver == "cbdgam_2d"
    assert CircumbinaryDisk(eos="gamma-law").physics["viscosity_model"] == ViscosityModel.CONSTANT_ALPHA
    assert CircumbinaryDisk().solver == "cbdiso_2d"
    with pytest.raises(SetupError):
        CircumbinaryDisk(eos="polytropic")


def _solver(physics_update=None, setup=None, mesh=None):
    setup = setup or CircumbinaryDisk(eos="gamma-law")
    physics = setup.physics
    physics.update(physics_update or {})
    mesh = mesh or PlanarCartesian2DMesh(-4.0, -4.0, 4.0, 4.0, 8, 8)
    return make_solver("cbdgam_2d", physics, dict(), setup=setup, mesh=mesh)


@pytest.mark.parametrize("update,message", [
    (dict(eos_type=EquationOfState.LOCALLY_ISOTHERMAL), "equation of states"),
    (dict(viscosity_model=ViscosityModel.CONSTANT_NU), "constant-alpha"),
])
def test_gamma_solver_rejects_what_the_reference_rejects(update, message):
    with pytest.raises(SolverInitializationError, match=message):
        _solver(update)


def test_gamma_solver_rejects_other_meshes_and_boundaries():
    class Mesh:
        shape = (8, 8)

    with pytest.raises(SolverInitializationError, match="cartesian mesh"):
        _solver(mesh=Mesh())

    class Periodic(CircumbinaryDisk):
        @property
        def boundary_condition(self):
            return "periodic"

    with pytest.raises(SolverInitializationError, match="outflow"):
        _solver(setup=Periodic(eos="gamma-law"))


def _grid(ni=8, nj=8):
    g = _capi.GamGrid()
    g.ni, g.nj = ni, nj
    g.xl, g.xr, g.yl, g.yr = -1.0, 1.0, -1.0, 1.0
    g.plm_theta, g.gamma_law_index = 1.5, 5.0 / 3.0
    return g


def test_gamma_capi_argument_checks():
    lib = _capi.lib()
    V = ctypes.c_void_p
    a, b = V(0x1000), V(0x2000)
    g, st = _grid(), _capi.GamStage()
    assert lib.cbdgam_b200_set_plm_theta(0.5) == 1 and lib.cbdgam_b200_set_plm_theta(2.5) == 1
    assert lib.cbdgam_b200_set_plm_theta(1.5) == 0
    # null grid / stage / arrays, and writing over the state being read
    assert lib.cbdgam_b200_advance_stage(None, ctypes.byref(st), a, None, b, None, None) == 1
    assert lib.cbdgam_b200_advance_stage(ctypes.byref(g), None, a, None, b, None, None) == 1
    assert lib.cbdgam_b200_advance_stage(ctypes.byref(g), ctypes.byref(st), a, None, a, None, None) == 1
    st.a = 0.5  # a later stage needs u_n's primitives
    assert lib.cbdgam_b200_advance_stage(ctypes.byref(g), ctypes.byref(st), a, None, b, None, None) == 1
    bad = _grid(ni=0)
    assert lib.cbdgam_b200_advance_stage(ctypes.byref(bad), ctypes.byref(st), a, a, b, None, None) == 1
    assert lib.cbdgam_b200_fill_guards(ctypes.byref(bad), a, None) == 1
    assert lib.cbdgam_b200_scratch_bytes(ctypes.byref(bad)) == 0
    iso = _grid()
    iso.gamma_law_index = 1.0  # the energy equation needs gamma != 1
    assert lib.cbdgam_b200_fill_guards(ctypes.byref(iso), a, None) == 1
    # reductions: at most four sums, known quantities, rates need a term
    masses = (_capi.Mass * 2)()
    diags = (_capi.Diag * 5)()
    for d in diags:
        d.quantity, d.which_mass, d.accretion = _capi.QUANTITY["mdot"], 1, 1
    assert lib.cbdgam_b200_scratch_bytes(ctypes.byref(g)) > 0
    assert lib.cbdgam_b200_reduce(ctypes.byref(g), masses, diags, 5, a, a, a, None) == 1
    diags[0].quantity = _capi.QUANTITY["power"]
    assert lib.cbdgam_b200_reduce(ctypes.byref(g), masses, diags, 1, a, a, a, None) == 1
    diags[0].quantity, diags[0].accretion, diags[0].gravity = _capi.QUANTITY["torque"], 0, 0
    assert lib.cbdgam_b200_reduce(ctypes.byref(g), masses, diags, 1, a, a, a, None) == 1
    # the drop-in kernels' own checks
    assert lib.cbdgam_2d_wavespeed(0, 8, a, b, 5.0 / 3.0) == 1
    assert lib.cbdgam_2d_primitive_to_conserved(8, 8, None, b, 5.0 / 3.0) == 1
    m9 = [0.0] * 8 + [0]
    assert lib.cbdgam_2d_point_mass_source_term(8, 8, -1.0, 1.0, -1.0, 1.0, *m9, *m9, 3, a, b, 1,
                                                5.0 / 3.0) == 1


def test_mass_cache_calls_the_physics_once_per_time():
    from sailfish_b200.physics import MassCache, Physics

    calls = []

    def masses(t):
        calls.append(t)
        return CircumbinaryDisk().point_masses(t)

    cache = MassCache(Physics(point_mass_function=masses), size=2)
    a = cache(0.5)
    assert cache(0.5) is a and calls == [0.5]
    cache(0.75)
    cache(1.0)  # 0.5 drops out
    cache(0.5)
    assert calls == [0.5, 0.75, 1.0, 0.5]
    assert tuple(a) == tuple(CircumbinaryDisk().point_masses(0.5))
