"""
Circumbinary-disk setups that choose the cbdiso_2d solver, with sailfish's
setup interface (sailfish/setup_base.py:32-286): typed model parameters,
`primitive(t, coords, out)`, `mesh(resolution)`, `physics`, `solver`,
`boundary_condition`, `reference_time_scale`, `point_masses(t)`.

Besides the per-zone `primitive`, each setup here has `primitive_array(t, x,
y)`, a vectorised form used to build the initial state of large grids; it
returns the same doubles as the per-zone loop (checked by the tests).
"""

from math import exp, pi, sqrt
from typing import Any, NamedTuple

import numpy as np

from .kepler import OrbitalElements
from .mesh import PlanarCartesian2DMesh
from .physics import EquationOfState, PointMass, SinkModel, ViscosityModel


class SetupError(Exception):
    """Something went wrong during setup configuration"""


class Parameter(NamedTuple):
    default: Any
    about: str
    mutable: bool = False


param = Parameter


class SetupBase:
    """Typed model parameters as in setup_base.py:43-61."""

    def __init__(self, **kwargs):
        for key, val, _ in type(self).default_model_parameters():
            if key in kwargs:
                if type(kwargs[key]) != type(val):
                    raise SetupError(
                        f"parameter '{key}' has type {type(val).__name__} (got {type(kwargs[key]).__name__})")
                setattr(self, key, kwargs[key])
            else:
                setattr(self, key, val)
        for key in kwargs:
            if not hasattr(self, key):
                raise SetupError(f"'{type(self).__name__}' has no parameter '{key}'")
        self.validate()

    @classmethod
    def default_model_parameters(cls):
        for klass in reversed(cls.__mro__):
            for key, val in vars(klass).items():
                if type(val) == Parameter:
                    yield key, val.default, val.about

    def validate(self):
        pass

    def model_parameters(self):
        """(key, value, about) of every model parameter (setup_base.py:146-155)."""
        for key, _, about in type(self).default_model_parameters():
            yield key, getattr(self, key), about

    def model_parameter_dict(self):
        """The model parameters as a dict (setup_base.py:157-161)."""
        return {key: val for key, val, _ in self.model_parameters()}

    @classmethod
    def dash_case_class_name(cls):
        """The class name in dash case, as setups are named in configuration and
        checkpoint files (setup_base.py:94-103)."""
        return "".join("-" + c.lower() if c.isupper() else c for c in cls.__name__).lstrip("-")

    @property
    def boundary_condition(self):
        return "outflow"

    @property
    def reference_time_scale(self):
        return 1.0

    def checkpoint_diagnostics(self, time):
        return dict()


def _binary_point_masses(setup, time, x_offset=None):
    m1, m2 = setup.orbital_elements.orbital_state(time)
    out = []
    for m in (m1, m2):
        x = m.position_x if x_offset is None else m.position_x + x_offset
        out.append(PointMass(
            mass=m.mass, position_x=x, position_y=m.position_y, velocity_x=m.velocity_x,
            velocity_y=m.velocity_y, softening_length=setup.softening_length,
            sink_model=SinkModel[setup.sink_model.upper()], sink_rate=setup.sink_rate,
            sink_radius=setup.sink_radius))
    return tuple(out)


class CircumbinaryDisk(SetupBase):
    """
    Circumbinary disk, isothermal or gamma-law
    (sailfish/setups/circumbinary_disk.py:17-215): Keplerian rotation about
    the origin with a softened radius and a binary on a Kepler orbit. The
    isothermal disk has uniform surface density (cbdiso_2d); the gamma-law
    disk the power laws Sigma ~ r^-3/5, P ~ r^-3/2 with an inner taper
    (cbdgam_2d).
    """

    eos = param("isothermal", "equation of state, isothermal or gamma-law (picks cbdiso_2d or cbdgam_2d)")
    domain_radius = param(12.0, "the mesh spans [-R, R] in x and y; this is R")
    mach_number = param(10.0, "ratio of orbital speed to sound speed (isothermal disk)", mutable=True)
    eccentricity = param(0.0, "eccentricity e of the binary orbit", mutable=True)
    mass_ratio = param(1.0, "q = m2 / m1, at most 1", mutable=True)
    sink_rate = param(10.0, "accretion rate coefficient of each sink", mutable=True)
    sink_radius = param(0.05, "radius of each sink", mutable=True)
    softening_length = param(0.05, "softening of each mass's gravity", mutable=True)
    buffer_is_enabled = param(True, "relax the outer ring of the mesh toward the initial disk", mutable=True)
    sink_model = param("torque_free", "how a sink removes mass: acceleration_free, force_free or torque_free", mutable=True)
    initial_sigma = param(1.0, "surface density of the gamma-law disk at radius 1")
    initial_pressure = param(1e-2, "vertically integrated pressure of the gamma-law disk at radius 1")
    cooling_coefficient = param(0.0, "coefficient of the gamma-law disk's cooling term (0: no cooling)")
    alpha = param(0.1, "alpha of the gamma-law disk's viscosity (0: inviscid)")
    nu = param(0.001, "constant kinematic viscosity nu of the isothermal disk (0: inviscid)")
    constant_softening = param(True, "gamma-law disk: fixed softening length rather than one following the disk height")
    gamma_law_index = param(5.0 / 3.0, "ratio of specific heats of the gamma-law gas")
    which_diagnostics = param("none", "time series the solver reduces each step: none, or mdots (both accretion rates)")

    def validate(self):
        if not self.is_isothermal and not self.is_gamma_law:
            raise SetupError(f"unknown eos {self.eos!r}: use isothermal or gamma-law")
        if self.which_diagnostics not in ["none", "mdots"]:
            raise SetupError(f"unknown which_diagnostics {self.which_diagnostics!r}: use none or mdots")

    @property
    def is_isothermal(self):
        return self.eos == "isothermal"

    @property
    def is_gamma_law(self):
        return self.eos == "gamma-law"

    def primitive(self, t, coords, primitive):
        GM = 1.0
        x, y = coords
        r = sqrt(x * x + y * y)
        r_softened = sqrt(x * x + y * y + self.softening_length * self.softening_length)
        phi_hat_x = -y / max(r, 1e-12)
        phi_hat_y = +x / max(r, 1e-12)
        if self.is_isothermal:
            primitive[0] = self.initial_sigma
            primitive[1] = sqrt(GM / r_softened) * phi_hat_x
            primitive[2] = sqrt(GM / r_softened) * phi_hat_y
        elif self.is_gamma_law:
            # Goodman (2003) eq. (A2): power laws with an inner taper
            taper = 0.0001 + 0.9999 * exp(-((1.0 / r_softened) ** 30))
            primitive[0] = self.initial_sigma * r_softened ** (-3.0 / 5.0) * taper
            primitive[1] = sqrt(GM / r_softened) * phi_hat_x
            primitive[2] = sqrt(GM / r_softened) * phi_hat_y
            primitive[3] = self.initial_pressure * r_softened ** (-3.0 / 2.0) * taper

    def primitive_array(self, t, x, y):
        """primitive() on whole arrays of zone centres, bit for bit. The
        isothermal fields need only IEEE operations, which numpy performs
        exactly; the gamma-law power laws and taper call the C library's pow /
        exp as Python's float arithmetic does (numpy's own vectorised pow /
        exp can differ from those in the last place)."""
        GM = 1.0
        x, y = np.broadcast_arrays(np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64))
        if self.is_gamma_law:
            import ctypes

            from . import _capi

            xc, yc = np.ascontiguousarray(x), np.ascontiguousarray(y)
            out = np.empty(x.shape + (4,))
            _capi.lib().cbdgam_b200_disk_primitive(xc.size, ctypes.c_void_p(xc.ctypes.data),
                                                   ctypes.c_void_p(yc.ctypes.data), float(self.softening_length),
                                                   float(self.initial_sigma), float(self.initial_pressure),
                                                   ctypes.c_void_p(out.ctypes.data))
            return out
        r = np.sqrt(x * x + y * y)
        r_softened = np.sqrt(x * x + y * y + self.softening_length * self.softening_length)
        out = np.empty(x.shape + (3,))
        out[..., 0] = self.initial_sigma
        out[..., 1] = np.sqrt(GM / r_softened) * (-y / np.maximum(r, 1e-12))
        out[..., 2] = np.sqrt(GM / r_softened) * (+x / np.maximum(r, 1e-12))
        return out

    def mesh(self, resolution):
        return PlanarCartesian2DMesh.centered_square(self.domain_radius, resolution)

    @property
    def default_resolution(self):
        return 512

    @property
    def physics(self):
        if self.is_gamma_law:
            return dict(
                eos_type=EquationOfState.GAMMA_LAW,
                gamma_law_index=self.gamma_law_index,
                point_mass_function=self.point_masses,
                buffer_is_enabled=self.buffer_is_enabled,
                buffer_driving_rate=1000.0,
                buffer_onset_width=0.1,
                cooling_coefficient=self.cooling_coefficient,
                constant_softening=self.constant_softening,
                viscosity_model=ViscosityModel.CONSTANT_ALPHA if self.alpha > 0.0 else ViscosityModel.NONE,
                viscosity_coefficient=0.0,
                alpha=self.alpha,
                diagnostics=self.diagnostics,
            )
        return dict(
            eos_type=EquationOfState.LOCALLY_ISOTHERMAL,
            mach_number=self.mach_number,
            point_mass_function=self.point_masses,
            buffer_is_enabled=self.buffer_is_enabled,
            buffer_driving_rate=100.0,
            buffer_onset_width=1.0,
            cooling_coefficient=0.0,
            constant_softening=self.constant_softening,
            viscosity_model=ViscosityModel.CONSTANT_NU if self.nu > 0.0 else ViscosityModel.NONE,
            viscosity_coefficient=self.nu,
            alpha=0.0,
            diagnostics=self.diagnostics,
        )

    @property
    def diagnostics(self):
        if self.which_diagnostics != "none":
            return [
                dict(quantity="time"),
                dict(quantity="mdot", which_mass=1, accretion=True),
                dict(quantity="mdot", which_mass=2, accretion=True),
            ]
        return []

    @property
    def solver(self):
        return "cbdgam_2d" if self.is_gamma_law else "cbdiso_2d"

    @property
    def default_end_time(self):
        return 1000.0

    @property
    def reference_time_scale(self):
        return 2.0 * pi

    @property
    def orbital_elements(self):
        return OrbitalElements(semimajor_axis=1.0, total_mass=1.0, mass_ratio=self.mass_ratio,
                               eccentricity=self.eccentricity)

    def point_masses(self, time):
        return _binary_point_masses(self, time)

    def checkpoint_diagnostics(self, time):
        return dict(point_masses=self.point_masses(time))


class KitpCodeComparison(SetupBase):
    """
    The KITP code-comparison disk (circumbinary_disk.py:218-375): a cavity of
    radius 2.5, a sub-Keplerian profile and a small radial kick.
    """

    mach_number = param(10.0, "ratio of orbital speed to sound speed", mutable=True)
    eccentricity = param(0.0, "eccentricity e of the binary orbit")
    mass_ratio = param(1.0, "q = M2 / M1")
    sink_radius = param(0.05, "radius of each sink", mutable=True)
    softening_length = param(0.05, "softening of each mass's gravity", mutable=True)
    nu = param(0.001, "constant kinematic viscosity nu", mutable=True)
    single_point_mass = param(False, "one unit mass fixed at the origin instead of the binary")
    sink_model = param("acceleration_free", "how a sink removes mass: acceleration_free, force_free or torque_free", mutable=True)
    domain_radius = param(8.0, "the mesh spans [-R, R] in x and y; this is R")
    sink_rate = param(10.0, "accretion rate coefficient of each sink", mutable=True)
    buffer_is_enabled = param(True, "relax the outer ring of the mesh toward the initial disk", mutable=True)
    disk_kick = param(1e-4, "amplitude of the small radial velocity that breaks the cavity's symmetry")
    which_diagnostics = param("kitp", "time series the solver reduces each step: kitp or forces")

    def validate(self):
        if self.which_diagnostics not in ["kitp", "forces"]:
            raise SetupError(f"unknown which_diagnostics {self.which_diagnostics!r}: use kitp or forces")

    def primitive(self, t, coords, primitive):
        x, y = coords
        r = sqrt(x * x + y * y)
        r_cav = 2.5
        delta0 = 1e-5
        sigma0 = 1.0
        sigma = sigma0 * (delta0 + (1 - delta0) * exp(-((r_cav / r) ** 12)))
        GM = 1.0
        a = 1.0
        n = 4.0
        omegaB = (GM / a**3) ** 0.5
        omega0 = (GM / r**3 * (1.0 - 1.0 / self.mach_number**2)) ** 0.5
        omega = (omega0**-n + omegaB**-n) ** (-1 / n)
        vr_pert = self.disk_kick * y * exp(-((r / 3.5) ** 6))
        primitive[0] = sigma
        primitive[1] = omega * -y + vr_pert * x / r
        primitive[2] = omega * +x + vr_pert * y / r

    def mesh(self, resolution):
        return PlanarCartesian2DMesh.centered_square(self.domain_radius, resolution)

    @property
    def default_resolution(self):
        return 200

    @property
    def diagnostics(self):
        if self.which_diagnostics == "kitp":
            return [
                dict(quantity="time"),
                dict(quantity="mdot", which_mass=1, accretion=True),
                dict(quantity="mdot", which_mass=2, accretion=True),
                dict(quantity="torque", which_mass="both", gravity=True),
                dict(quantity="torque", which_mass="both", gravity=True, radial_cut=(1.0, self.domain_radius)),
                dict(quantity="sigma_m1"),
                dict(quantity="eccentricity_vector", radial_cut=(1.0, 6.0)),
            ]
        return [
            dict(quantity="time"),
            dict(quantity="mdot", which_mass=1, accretion=True),
            dict(quantity="mdot", which_mass=2, accretion=True),
            dict(quantity="fx", which_mass=1, gravity=True),
            dict(quantity="fx", which_mass=1, accretion=True),
            dict(quantity="fy", which_mass=1, gravity=True),
            dict(quantity="fy", which_mass=1, accretion=True),
            dict(quantity="fx", which_mass=2, gravity=True),
            dict(quantity="fx", which_mass=2, accretion=True),
            dict(quantity="fy", which_mass=2, gravity=True),
            dict(quantity="fy", which_mass=2, accretion=True),
        ]

    @property
    def physics(self):
        return dict(
            eos_type=EquationOfState.LOCALLY_ISOTHERMAL,
            mach_number=self.mach_number,
            point_mass_function=self.point_masses,
            buffer_is_enabled=self.buffer_is_enabled,
            buffer_driving_rate=100.0,
            buffer_onset_width=1.0,
            viscosity_coefficient=self.nu,
            viscosity_model=ViscosityModel.CONSTANT_NU if self.nu > 0.0 else ViscosityModel.NONE,
            diagnostics=self.diagnostics,
        )

    @property
    def solver(self):
        return "cbdiso_2d"

    @property
    def default_end_time(self):
        return 1.0

    @property
    def reference_time_scale(self):
        return 2.0 * pi

    @property
    def orbital_elements(self):
        return OrbitalElements(semimajor_axis=1.0, total_mass=1.0, mass_ratio=self.mass_ratio,
                               eccentricity=self.eccentricity)

    def point_masses(self, time):
        if self.single_point_mass:
            return PointMass(softening_length=self.softening_length,
                             sink_model=SinkModel[self.sink_model.upper()], sink_rate=self.sink_rate,
                             sink_radius=self.sink_radius, mass=1.0)
        return _binary_point_masses(self, time)

    def checkpoint_diagnostics(self, time):
        return dict(point_masses=self.point_masses(time), diagnostics=self.diagnostics)


class BinaryBondi(SetupBase):
    """A binary in a uniform wind, globally isothermal (sailfish/setups/binary_bondi.py:19-102)."""

    aspect = param(1, "mesh width divided by mesh height (an integer)")
    height = param(1.0, "mesh height, in units of the binary separation")
    x_bin = param(0.0, "x offset of the binary's centre of mass from the mesh centre")
    sound_speed = param(1.0, "the gas's uniform sound speed")
    wind_vel = param(1.0, "x velocity of the incoming wind")
    bh_sep = param(0.25, "semi-major axis of the binary")
    bh_mass = param(1.0, "mass of the heavier component")
    sink_radius = param(0.05, "radius of each sink")
    sink_model = param("acceleration_free", "how a sink removes mass: acceleration_free, force_free or torque_free")
    sink_rate = param(1e2, "accretion rate coefficient of each sink")
    mass_ratio = param(1.0, "q = m2 / m1, between 0 and 1")
    eccentricity = param(0.0, "eccentricity e of the binary orbit")
    softening_length = param(0.05, "softening of each mass's gravity", mutable=True)

    def primitive(self, t, coords, primitive):
        primitive[0] = 1.0
        primitive[1] = self.wind_vel
        primitive[2] = 0.0

    def primitive_array(self, t, x, y):
        out = np.zeros(np.broadcast(x, y).shape + (3,))
        out[..., 0] = 1.0
        out[..., 1] = self.wind_vel
        return out

    def mesh(self, resolution):
        return PlanarCartesian2DMesh.centered_rectangle(self.height, resolution, int(self.aspect))

    @property
    def physics(self):
        return dict(eos_type=EquationOfState.GLOBALLY_ISOTHERMAL, sound_speed=self.sound_speed,
                    point_mass_function=self.point_masses)

    @property
    def solver(self):
        return "cbdiso_2d"

    @property
    def orbital_elements(self):
        return OrbitalElements(semimajor_axis=self.bh_sep, total_mass=self.bh_mass * (1 + self.mass_ratio),
                               mass_ratio=self.mass_ratio, eccentricity=self.eccentricity)

    def point_masses(self, time):
        return _binary_point_masses(self, time, x_offset=self.x_bin)


SETUPS = {
    "circumbinary-disk": CircumbinaryDisk,
    "kitp-code-comparison": KitpCodeComparison,
    "binary-bondi": BinaryBondi,
}


def find_setup_class(name):
    try:
        return SETUPS[name]
    except KeyError:
        raise SetupError(f"no setup named {name}")
