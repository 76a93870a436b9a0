"""
Solver registry with sailfish's plugin semantics (sailfish/solvers/__init__.py):
`make_solver(name, physics, options, **kwargs)` constructs `<module>.Solver`,
extension modules registered by import name override a built-in of the same
name, and a TypeError or ValueError from a constructor is re-raised as
SolverInitializationError.
"""

from importlib import import_module


class SolverInitializationError(Exception):
    """An invalid runtime configuration"""


_extension_modules = []


def register_solver_extension(solver_name):
    _extension_modules.append(solver_name)


def make_solver(name, physics, options, **kwargs):
    from . import cbdgam_2d, cbdiso_2d

    solvers = dict(cbdiso_2d=cbdiso_2d, cbdgam_2d=cbdgam_2d)
    for ext_name in _extension_modules:
        solvers[ext_name] = import_module(ext_name)
    try:
        return solvers[name].Solver(physics=physics or dict(), options=options or dict(), **kwargs)
    except (TypeError, ValueError) as e:
        raise SolverInitializationError(e)
