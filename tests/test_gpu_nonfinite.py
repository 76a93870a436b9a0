"""
Non-finite detection. The reference's driver takes dt = min spacing / max
wavespeed * cfl with no check (sailfish/driver.py:508-510) and runs on with a
NaN time step. Here:
  * the wavespeed maximum keeps a NaN zone value, as numpy's max over the
    reference's wavespeed array does (cbdiso_2d.py:174), and
    `maximum_wavespeed()` raises CbdError with CBD_ERR_NONFINITE for it;
  * the device stepper (Solver.run) sets CBD_ERR_NONFINITE when a step's dt
    is not finite and positive, marks that step's stage records halted, so
    the stages of that and every later captured step leave the state as it
    was, and `run` raises.
The NaN is put into the initial state on the host; nothing on the GPU traps
or faults: the kernels only read it.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from oracle import host as oh  # noqa: E402
from sailfish_b200 import _capi, make_solver  # noqa: E402
from sailfish_b200.cbdiso_2d import initial_condition  # noqa: E402
from sailfish_b200.setups import CircumbinaryDisk  # noqa: E402

NONFINITE = 3


def _solver(n=96, poison=None):
    setup = CircumbinaryDisk(domain_radius=8.0, nu=1e-3)
    mesh = setup.mesh(n)
    physics = setup.physics
    physics["diagnostics"] = [dict(quantity="time"), dict(quantity="mdot", which_mass=1, accretion=True)]
    prim = initial_condition(setup, mesh, 0.0)
    prim[..., 0] += oh.seeded_noise(n, n, 3)
    if poison is not None:
        i, j, value = poison
        prim[i, j, 1] = value
        prim[i, j, 2] = value
    s = make_solver("cbdiso_2d", physics, dict(rk_order=2, plm_theta=1.5), setup=setup, mesh=mesh, solution=prim)
    return s, prim


@pytest.mark.parametrize("where", [(0, 0), (40, 57), (95, 95)])
def test_nan_velocity_makes_maximum_wavespeed_raise(where):
    s, _ = _solver(poison=(*where, np.nan))
    with pytest.raises(_capi.CbdError) as e:
        s.maximum_wavespeed()
    assert e.value.status == NONFINITE


def test_infinite_velocity_makes_the_device_stepper_stop():
    """An infinite velocity gives an infinite wavespeed and dt = 0: the first
    step stops the stepper, the graph's 16 steps leave the state as it was."""
    s, prim = _solver(poison=(30, 31, np.inf))
    before = s.solution
    with pytest.raises(_capi.CbdError) as e:
        s.run(16, graph=True, steps_per_graph=16)
    assert e.value.status == NONFINITE
    assert np.array_equal(s.solution, before, equal_nan=True)
    assert s.time == 0.0


@pytest.mark.parametrize("graph", [False, True])
def test_nan_wavespeed_stops_the_device_stepper(graph):
    s, _ = _solver(poison=(12, 80, np.nan))
    before = s.solution
    with pytest.raises(_capi.CbdError) as e:
        s.run(16, graph=graph, steps_per_graph=16)
    assert e.value.status == NONFINITE
    assert np.array_equal(s.solution, before, equal_nan=True)


@pytest.mark.parametrize("bad", [np.nan, np.inf, 0.0])
def test_bad_dt_halts_a_captured_run_where_it_occurs(bad):
    """A frozen dt sequence whose 6th entry is bad: the captured 16-step run
    stops there, and the state is the one after the first 5 steps."""
    s, _ = _solver()
    ref, _ = _solver()
    dts = np.full(16, 1e-3)
    dts[5] = bad
    seq = torch.from_numpy(dts).cuda()
    with pytest.raises(_capi.CbdError) as e:
        s.run(16, graph=True, steps_per_graph=16, dt_sequence=seq)
    assert e.value.status == NONFINITE
    ref.run(5, graph=False, dt_sequence=seq[:5].clone())
    assert np.array_equal(s.solution, ref.solution)


def test_advance_rejects_a_non_finite_time_step():
    s, _ = _solver()
    with pytest.raises(_capi.CbdError) as e:
        s.advance(float("nan"))
    assert e.value.status == NONFINITE


def test_gamma_law_maximum_wavespeed_raises_on_nan():
    from sailfish_b200.cbdgam_2d import initial_condition as gam_ic

    setup = CircumbinaryDisk(eos="gamma-law", domain_radius=8.0)
    mesh = setup.mesh(64)
    prim = gam_ic(setup, mesh, 0.0)
    prim[20, 20, 1] = prim[20, 20, 2] = np.nan
    s = make_solver("cbdgam_2d", setup.physics, {}, setup=setup, mesh=mesh, solution=prim)
    with pytest.raises(_capi.CbdError) as e:
        s.maximum_wavespeed()
    assert e.value.status == NONFINITE
