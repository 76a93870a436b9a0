"""
Two-body Kepler orbit of a binary, the part the circumbinary setups use
(sailfish/physics/kepler.py:290-373, 414-421): component positions and
velocities from the time since periapse.

The floating-point operations follow the reference's order so that the
point-mass positions handed to the kernels are the same doubles.
"""

from math import cos, floor, pi, sin, sqrt
from typing import NamedTuple

NEWTON_G = 1.0


class KeplerBody(NamedTuple):
    """Mass, position and velocity of one component (kepler.py:14-23)."""

    mass: float
    position_x: float
    position_y: float
    velocity_x: float
    velocity_y: float


class OrbitalState(NamedTuple):
    primary: KeplerBody
    secondary: KeplerBody


def newton_solve(f, g, x):
    """Newton iteration with the reference's stopping rule: |f| <= 1e-15, at
    most 10 updates, else ValueError (kepler.py:414-421)."""
    n = 0
    while abs(f(x)) > 1e-15:
        x -= f(x) / g(x)
        n += 1
        if n > 10:
            raise ValueError("solve_newton_rapheson: no solution")
    return x


class OrbitalElements(NamedTuple):
    semimajor_axis: float
    total_mass: float
    mass_ratio: float
    eccentricity: float

    @property
    def omega(self):
        m = self.total_mass
        a = self.semimajor_axis
        return sqrt(NEWTON_G * m / a / a / a)

    @property
    def period(self):
        return 2.0 * pi / self.omega

    def eccentric_anomaly(self, time_since_periapse):
        p = self.period
        t = time_since_periapse - self.period * floor(time_since_periapse / p)
        e = self.eccentricity
        mean_anomaly = self.omega * t
        return newton_solve(
            lambda k: k - e * sin(k) - mean_anomaly, lambda k: 1.0 - e * cos(k), mean_anomaly)

    def orbital_state_from_eccentric_anomaly(self, eccentric_anomaly):
        a = self.semimajor_axis
        m = self.total_mass
        q = self.mass_ratio
        e = self.eccentricity
        w = self.omega
        m1 = m / (1.0 + q)
        m2 = m - m1
        ck = cos(eccentric_anomaly)
        sk = sin(eccentric_anomaly)
        x1 = -a * q / (1.0 + q) * (e - ck)
        y1 = +a * q / (1.0 + q) * (sk) * sqrt(1.0 - e * e)
        x2 = -x1 / q
        y2 = -y1 / q
        vx1 = -a * q / (1.0 + q) * w / (1.0 - e * ck) * sk
        vy1 = +a * q / (1.0 + q) * w / (1.0 - e * ck) * ck * sqrt(1.0 - e * e)
        vx2 = -vx1 / q
        vy2 = -vy1 / q
        return OrbitalState(KeplerBody(m1, x1, y1, vx1, vy1), KeplerBody(m2, x2, y2, vx2, vy2))

    def orbital_state(self, time_since_periapse):
        return self.orbital_state_from_eccentric_anomaly(self.eccentric_anomaly(time_since_periapse))
