"""
Restart compatibility with the reference driver's checkpoint files.

The reference writes a checkpoint as a pickled dict (driver.py:143-178,
write_checkpoint) and restarts from it by rebuilding the setup from
`setup_name` and `model_parameters` and handing `time` and `solution` to
make_solver (driver.py:338-395). The pickle names classes of the reference
package: its mesh (sailfish.mesh.PlanarCartesian2DMesh), point masses and
sink-model enum (sailfish.physics.circumbinary), event records
(sailfish.event.Recurrence, RecurringEvent) and the driver's arguments
(sailfish.driver.DriverArgs), all NamedTuples or Enums.

`load_checkpoint` reads such a file without the reference installed, mapping
those classes onto this package's equivalents (same fields, same order);
`restart` builds this package's Solver from it. `write_checkpoint` writes
the same dict, pickling the same objects under the reference's class names,
so the reference's load_checkpoint can read it.
"""

from __future__ import annotations

import enum
import os
import pathlib
import pickle
from typing import Dict, NamedTuple, Optional

from . import mesh as _mesh
from . import physics as _physics


class Recurrence(NamedTuple):
    """A recurring event's rule (event.py:11-23): kind 0 linear, 1 log."""

    kind: int = None
    interval: float = None


class RecurringEvent(NamedTuple):
    """A recurring event's state (event.py:51-61)."""

    last_time: float = None
    number: int = 0


class DriverArgs(NamedTuple):
    """The driver's arguments as stored in a checkpoint (driver.py:228-245)."""

    setup_name: str = None
    chkpt_file: str = None
    model_parameters: dict = None
    solver_options: dict = None
    cfl_number: float = None
    end_time: float = None
    execution_mode: str = None
    fold: int = None
    resolution: int = None
    num_patches: int = None
    events: Dict[str, Recurrence] = dict()
    new_timestep_cadence: int = None
    verbose_output: str = ""


# (reference module, class name) <-> this package's class
_CLASSES = {
    ("sailfish.mesh", "PlanarCartesian2DMesh"): _mesh.PlanarCartesian2DMesh,
    ("sailfish.physics.circumbinary", "PointMass"): _physics.PointMass,
    ("sailfish.physics.circumbinary", "Diagnostic"): _physics.Diagnostic,
    ("sailfish.physics.circumbinary", "SinkModel"): _physics.SinkModel,
    ("sailfish.physics.circumbinary", "EquationOfState"): _physics.EquationOfState,
    ("sailfish.physics.circumbinary", "ViscosityModel"): _physics.ViscosityModel,
    ("sailfish.event", "Recurrence"): Recurrence,
    ("sailfish.event", "RecurringEvent"): RecurringEvent,
    ("sailfish.driver", "DriverArgs"): DriverArgs,
}
_NAMES = {cls: key for key, cls in _CLASSES.items()}


class CheckpointError(Exception):
    pass


class _Unpickler(pickle.Unpickler):
    def find_class(self, module, name):
        cls = _CLASSES.get((module, name))
        if cls is not None:
            return cls
        if module == "sailfish" or module.startswith("sailfish."):
            raise CheckpointError(f"checkpoint refers to {module}.{name}, which has no equivalent here")
        return super().find_class(module, name)


def load_checkpoint(chkpt_file):
    """The checkpoint dict of a reference (or this package's) checkpoint
    file (driver.py:181-189)."""
    try:
        with open(chkpt_file, "rb") as f:
            return _Unpickler(f).load()
    except FileNotFoundError:
        raise CheckpointError(f"could not open checkpoint file {chkpt_file}")


class RestartState(NamedTuple):
    """What the driver keeps besides the solver (driver.py:361-386)."""

    iteration: int
    time: float
    timestep_dt: Optional[float]
    cfl_number: float
    timeseries: list
    event_states: dict
    driver: DriverArgs
    setup: object
    mesh: object


def restart(chkpt, solver_options=None, **model_parameters):
    """
    (solver, RestartState) from a checkpoint dict or file name: the setup
    is rebuilt from setup_name and the stored model parameters, updated by
    `model_parameters`; the solver options are the stored ones updated by
    `solver_options`; the mesh, time and solution are the stored ones
    (driver.py:344-372).
    """
    from .setups import find_setup_class
    from .solvers import make_solver

    if not isinstance(chkpt, dict):
        chkpt = load_checkpoint(chkpt)
    setup_class = find_setup_class(chkpt["setup_name"])
    params = dict(chkpt["model_parameters"])
    params.update(model_parameters)
    setup = setup_class(**params)
    options = dict(chkpt.get("solver_options") or {})
    options.update(chkpt.get(EXTRA_OPTIONS_KEY) or {})
    options.update(solver_options or {})
    mesh = chkpt["mesh"]
    driver = chkpt.get("driver") or DriverArgs()
    solver = make_solver(setup.solver, setup.physics, options, setup=setup, mesh=mesh, time=chkpt["time"],
                         solution=chkpt["solution"], num_patches=getattr(driver, "num_patches", None) or 1)
    state = RestartState(iteration=chkpt["iteration"], time=chkpt["time"], timestep_dt=chkpt.get("timestep_dt"),
                         cfl_number=chkpt.get("cfl_number"), timeseries=chkpt.get("timeseries", []),
                         event_states=chkpt.get("event_states", {}), driver=driver, setup=setup, mesh=mesh)
    return solver, state


class _ReferenceName:
    """Pickles as the global `module.name` of the reference package."""

    def __init__(self, module, name):
        self.module, self.name = module, name

    def __reduce_ex__(self, protocol):
        return self.name

    def __call__(self, *args):  # stands for the reference class; never called here
        raise TypeError(f"{self.module}.{self.name} is a name only")


class _Pickler(pickle._Pickler):
    """Pickles this package's checkpoint classes under the reference's names
    (protocol 4, as the reference's pickle.dump writes)."""

    def reducer_override(self, obj):
        key = _NAMES.get(type(obj))
        if key is None:
            return NotImplemented
        args = (obj.value,) if isinstance(obj, enum.Enum) else tuple(obj)
        return _ReferenceName(*key), args

    def save_global(self, obj, name=None):
        if isinstance(obj, _ReferenceName):
            self.save(obj.module)
            self.save(obj.name)
            self.write(pickle.STACK_GLOBAL)
            self.memoize(obj)
            return
        super().save_global(obj, name)


# the reference's solver options per solver (cbdiso_2d.py:23-30,
# cbdgam_2d.py:23-27); the others this package's solvers take are stored
# under their own key, which the reference's restart does not read
REFERENCE_OPTIONS = {
    "cbdiso_2d": ("velocity_ceiling", "density_floor", "rk_order"),
    "cbdgam_2d": ("pressure_floor", "density_floor", "velocity_ceiling", "mach_ceiling"),
}
EXTRA_OPTIONS_KEY = "b200_solver_options"


def checkpoint_dict(solver, setup, mesh, iteration, timestep_dt, cfl_number, timeseries=(), event_states=None,
                    driver=None):
    """The dict the reference's write_checkpoint stores (driver.py:159-175),
    plus this package's own solver options under EXTRA_OPTIONS_KEY."""
    options = dict(solver.options)
    ref_keys = REFERENCE_OPTIONS[setup.solver]
    extra = {k: v for k, v in options.items() if k not in ref_keys}
    out = dict(
        iteration=iteration,
        time=solver.time,
        timestep_dt=timestep_dt,
        cfl_number=cfl_number,
        solution=solver.solution,
        primitive=solver.primitive,
        timeseries=list(timeseries),
        solver=setup.solver,
        solver_options={k: v for k, v in options.items() if k in ref_keys},
        event_states=dict(event_states or {}),
        driver=driver if driver is not None else DriverArgs(),
        model_parameters=setup.model_parameter_dict(),
        setup_name=setup.dash_case_class_name(),
        mesh=mesh,
        **setup.checkpoint_diagnostics(solver.time),
    )
    if extra:
        out[EXTRA_OPTIONS_KEY] = extra
    return out


def write_checkpoint(number, outdir, solver, setup, mesh, iteration, timestep_dt, cfl_number, timeseries=(),
                     event_states=None, driver=None):
    """Write chkpt.NNNN.pk (or chkpt.<str>.pk) as driver.py:143-178 names it;
    returns the file name."""
    if type(number) is int:
        filename = f"chkpt.{number:04d}.pk"
    elif type(number) is str:
        filename = f"chkpt.{number}.pk"
    else:
        raise ValueError("number arg must be int or str")
    if outdir is not None:
        pathlib.Path(outdir).mkdir(parents=True, exist_ok=True)
        filename = os.path.join(outdir, filename)
    state = checkpoint_dict(solver, setup, mesh, iteration, timestep_dt, cfl_number, timeseries, event_states,
                            driver)
    with open(filename, "wb") as f:
        _Pickler(f, protocol=4).dump(state)
    return filename
