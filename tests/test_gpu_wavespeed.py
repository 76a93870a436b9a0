"""
The stage-2 epilogue kernel computes the next step's CFL wavespeed maximum
(cbdiso_2d.c:340-350 per zone, numpy's max over the zones,
cbdiso_2d.py:174) over the new state, tile by tile in its own launch. It must
be the same double as the maximum the standalone reduction kernel computes
zone by zone on the same state: compared bit for bit on a noisy disk at
three sizes, on columns that are mirror images of themselves (exact ties
between zones), on a uniform isothermal state (every zone tied), after a
NaN in the input state (which the stage's velocity ceiling clamps) and on
explicit tiles of many and few rows.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from oracle import host as oh  # noqa: E402
from sailfish_b200 import make_solver  # noqa: E402
from sailfish_b200.cbdiso_2d import initial_condition  # noqa: E402
from sailfish_b200.mesh import PlanarCartesian2DMesh  # noqa: E402
from sailfish_b200.physics import EquationOfState  # noqa: E402
from sailfish_b200.setups import CircumbinaryDisk  # noqa: E402


class _Uniform:
    boundary_condition = "outflow"
    reference_time_scale = 1.0
    physics = dict(eos_type=EquationOfState.GLOBALLY_ISOTHERMAL, sound_speed=1.0)


def _epilogue_and_per_zone(s, dt, steps=1):
    """The wavespeed maximum from the last stage's epilogue, then the one
    the reduction kernel computes zone by zone on the same state."""
    for _ in range(steps):
        s.advance(dt)
    fused = float(s._read_result()[0])
    s._reduce_now(True, [])
    per_zone = float(s._read_result()[0])
    return fused, per_zone


def _same(a, b):
    return np.array(a).view(np.int64) == np.array(b).view(np.int64)


@pytest.mark.parametrize("n", [96, 256, 1000])
def test_noisy_disk(n):
    setup = CircumbinaryDisk(domain_radius=8.0, nu=1e-3)
    mesh = setup.mesh(n)
    prim = initial_condition(setup, mesh, 0.0)
    prim[..., 0] += oh.seeded_noise(n, n, 11)
    s = make_solver("cbdiso_2d", setup.physics, dict(rk_order=2, plm_theta=1.5), setup=setup, mesh=mesh,
                    solution=prim)
    fused, per_zone = _epilogue_and_per_zone(s, 1e-4, steps=3)
    assert np.isfinite(fused) and _same(fused, per_zone)


@pytest.mark.parametrize("n", [64, 200])
def test_mirror_symmetric_columns(n):
    """Equal masses on the x axis and a fluid at rest: every column's
    wavespeeds are mirror images about the middle row, so the tiles across
    the middle hold ties (kept through a short step)."""
    setup = CircumbinaryDisk(domain_radius=8.0, nu=0.0)
    mesh = setup.mesh(n)
    prim = np.zeros((n, n, 3))
    prim[..., 0] = 1.0
    s = make_solver("cbdiso_2d", setup.physics, dict(rk_order=2, plm_theta=1.5), setup=setup, mesh=mesh,
                    solution=prim)
    fused, per_zone = _epilogue_and_per_zone(s, 1e-9)
    assert np.isfinite(fused) and _same(fused, per_zone)


@pytest.mark.parametrize("n", [48, 300])
def test_uniform_isothermal_state(n):
    """No masses, constant sound speed, a fluid at rest: every zone has the
    same wavespeed."""
    mesh = PlanarCartesian2DMesh(-1.0, -1.0, 1.0, 1.0, n, n)
    prim = np.zeros((n, n, 3))
    prim[..., 0] = 1.0
    setup = _Uniform()
    s = make_solver("cbdiso_2d", dict(setup.physics), dict(rk_order=2, plm_theta=1.5), setup=setup, mesh=mesh,
                    solution=prim)
    fused, per_zone = _epilogue_and_per_zone(s, 1e-3)
    assert fused == 1.0 and _same(fused, per_zone)


def test_nan_zone():
    """A NaN velocity in the input state: the stage's floors clamp it to the
    velocity ceiling, and both maxima see the same clamped zone."""
    n = 96
    setup = CircumbinaryDisk(domain_radius=8.0, nu=1e-3)
    mesh = setup.mesh(n)
    prim = initial_condition(setup, mesh, 0.0)
    prim[40, 57, 1] = np.nan
    s = make_solver("cbdiso_2d", setup.physics, dict(rk_order=2, plm_theta=1.5), setup=setup, mesh=mesh,
                    solution=prim)
    fused, per_zone = _epilogue_and_per_zone(s, 1e-4)
    assert _same(fused, per_zone) or (np.isnan(fused) and np.isnan(per_zone))


@pytest.mark.parametrize("tile", [(128, 70), (256, 45), (64, 5)])
def test_explicit_tiles(tile):
    """Tiles of many rows (a thread's column of 70 zones), 256-column strips
    and short 64-column tiles: the maximum is the same double either way."""
    n = 300
    setup = CircumbinaryDisk(domain_radius=8.0, nu=1e-3)
    mesh = setup.mesh(n)
    prim = initial_condition(setup, mesh, 0.0)
    prim[..., 0] += oh.seeded_noise(n, n, 5)
    s = make_solver("cbdiso_2d", setup.physics, dict(rk_order=2, plm_theta=1.5, tile=tile), setup=setup,
                    mesh=mesh, solution=prim)
    fused, per_zone = _epilogue_and_per_zone(s, 1e-4, steps=2)
    assert np.isfinite(fused) and _same(fused, per_zone)
