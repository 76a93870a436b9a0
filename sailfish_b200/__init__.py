"""
sailfish_b200: sailfish's 2D isothermal circumbinary-disk solver (cbdiso_2d)
rebuilt for one NVIDIA B200, behind sailfish's own solver plugin API.

    from sailfish_b200 import make_solver
    from sailfish_b200.setups import CircumbinaryDisk

    setup = CircumbinaryDisk(domain_radius=8.0, nu=1e-3)
    mesh = setup.mesh(1024)
    solver = make_solver("cbdiso_2d", setup.physics, dict(rk_order=2), setup=setup, mesh=mesh)
    dt = mesh.min_spacing() / solver.maximum_wavespeed() * 0.3
    solver.advance(dt)

Host states go to the device fastest from pinned memory: `pinned_empty(shape)`
gives such an array, and `solution` returns one.

The compute path is libcbdiso_b200.so (sources in csrc/, C-ABI in
include/cbdiso_b200.h), built in-tree by `python -m sailfish_b200._build`.
"""

from ._hostio import pinned_empty  # noqa: F401
from .solvers import SolverInitializationError, make_solver, register_solver_extension  # noqa: F401

__all__ = ["make_solver", "register_solver_extension", "SolverInitializationError", "pinned_empty"]
