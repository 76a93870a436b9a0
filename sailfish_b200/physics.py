"""
Physics configuration of the circumbinary-disk solvers, with the same names,
fields and defaults as sailfish/physics/circumbinary.py:5-226, so that a
physics dict produced by a sailfish setup constructs this class unchanged.
"""

from enum import Enum
from typing import Callable, List, NamedTuple, Union


class SinkModel(Enum):
    INACTIVE = 0
    ACCELERATION_FREE = 1
    TORQUE_FREE = 2
    FORCE_FREE = 3


class EquationOfState(Enum):
    GLOBALLY_ISOTHERMAL = 1
    LOCALLY_ISOTHERMAL = 2
    GAMMA_LAW = 3


class ViscosityModel(Enum):
    NONE = 0
    CONSTANT_NU = 1
    CONSTANT_ALPHA = 2


def enum_value(x):
    """Integer value of an enum member from this module or from sailfish's own."""
    return int(getattr(x, "value", x))


class Diagnostic(NamedTuple):
    """One reduction requested from the solver (circumbinary.py:24-38)."""

    quantity: str
    gravity: bool = False
    accretion: bool = False
    which_mass: Union[int, str] = None
    radial_cut: tuple = None


class PointMass(NamedTuple):
    """A gravitating, optionally accreting point mass (circumbinary.py:41-95)."""

    mass: float = 0.0
    position_x: float = 0.0
    position_y: float = 0.0
    velocity_x: float = 0.0
    velocity_y: float = 0.0
    softening_length: float = 0.0
    sink_model: SinkModel = SinkModel.INACTIVE
    sink_rate: float = 0.0
    sink_radius: float = 0.0


class Physics(NamedTuple):
    """Physics parameters of cbdiso_2d (circumbinary.py:98-193)."""

    eos_type: EquationOfState = EquationOfState.GLOBALLY_ISOTHERMAL
    sound_speed: float = 1.0
    mach_number: float = 10.0
    gamma_law_index: float = 5.0 / 3.0
    viscosity_model: ViscosityModel = ViscosityModel.NONE
    viscosity_coefficient: float = 0.0
    alpha: float = 0.0
    buffer_is_enabled: bool = False
    buffer_driving_rate: float = 1000.0
    buffer_onset_width: float = 0.1
    point_mass_function: Callable[[float], List[PointMass]] = None
    cooling_coefficient: float = 0.0
    constant_softening: bool = True
    diagnostics: List[Diagnostic] = []

    @property
    def num_particles(self):
        if self.point_mass_function is None:
            return 0
        return len(self.point_mass_function(0.0))

    def point_masses(self, time):
        """
        Zero, one or two masses from the callback, padded to two with
        massless, inactive ones (circumbinary.py:202-226).
        """
        if self.point_mass_function is None:
            return PointMass(), PointMass()
        masses = self.point_mass_function(time)
        if masses is None:
            return PointMass(), PointMass()
        if hasattr(masses, "position_x"):
            return masses, PointMass()
        if isinstance(masses, (tuple, list)):
            if len(masses) == 1:
                return masses[0], PointMass()
            if len(masses) == 2:
                return masses
        raise ValueError("point_mass_function returned an unsupported description of point masses")


class MassCache:
    """physics.point_masses(t) remembered for the last few times t: a solver
    asks for the same time several times (a step starts at the previous
    step's end, and the end-of-step reductions use it too)."""

    def __init__(self, physics, size=4):
        self.physics = physics
        self.size = size
        self.entries = []

    def __call__(self, t):
        for tc, masses in self.entries:
            if tc == t:
                return masses
        masses = self.physics.point_masses(t)
        self.entries.append((t, masses))
        if len(self.entries) > self.size:
            self.entries.pop(0)
        return masses
