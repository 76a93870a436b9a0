"""
CPU oracle, host side: a Python/numpy restatement of the cbdiso_2d solver
adapter (sailfish/solvers/cbdiso_2d.py), the two-body Kepler solution
(sailfish/physics/kepler.py) and the circumbinary setups' initial data
(sailfish/setups/circumbinary_disk.py).

TEST INFRASTRUCTURE ONLY. The product package never imports this module. It
drives either the C restatement of the kernels (oracle/cbdiso_2d_oracle.c) or
the reference kernels themselves built into oracle/_ref by build_ref.sh, and it
is pinned against fixtures produced by running the reference (tests/golden).

Scalar arithmetic (Kepler, time stepping) follows the reference operation by
operation so that point-mass positions and RK stage times agree bit for bit.
"""

from __future__ import annotations

import ctypes
import math
import os
from ctypes import POINTER, c_double, c_int
from typing import Callable, NamedTuple, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NG = 2
NQ = 3

# ---------------------------------------------------------------------------
# two-body problem (kepler.py:290-373, 414-421)
# ---------------------------------------------------------------------------


class Body(NamedTuple):
    mass: float
    x: float
    y: float
    vx: float
    vy: float


def kepler_omega(a: float, m: float) -> float:
    """kepler.py:300-307 (G = 1)."""
    return math.sqrt(1.0 * m / a / a / a)


def kepler_eccentric_anomaly(t: float, a: float, m: float, e: float) -> float:
    """kepler.py:356-366 with the Newton loop of kepler.py:414-421."""
    w = kepler_omega(a, m)
    p = 2.0 * math.pi / w
    tt = t - p * math.floor(t / p)
    n = w * tt
    k = n
    it = 0
    while abs(k - e * math.sin(k) - n) > 1e-15:
        k -= (k - e * math.sin(k) - n) / (1.0 - e * math.cos(k))
        it += 1
        if it > 10:
            raise ValueError("solve_newton_rapheson: no solution")
    return k


def kepler_state(t: float, a: float = 1.0, m: float = 1.0, q: float = 1.0, e: float = 0.0):
    """kepler.py:329-354: positions and velocities of the two components."""
    E = kepler_eccentric_anomaly(t, a, m, e)
    w = kepler_omega(a, m)
    m1 = m / (1.0 + q)
    m2 = m - m1
    ck = math.cos(E)
    sk = math.sin(E)
    x1 = -a * q / (1.0 + q) * (e - ck)
    y1 = +a * q / (1.0 + q) * (sk) * math.sqrt(1.0 - e * e)
    x2 = -x1 / q
    y2 = -y1 / q
    vx1 = -a * q / (1.0 + q) * w / (1.0 - e * ck) * sk
    vy1 = +a * q / (1.0 + q) * w / (1.0 - e * ck) * ck * math.sqrt(1.0 - e * e)
    vx2 = -vx1 / q
    vy2 = -vy1 / q
    return Body(m1, x1, y1, vx1, vy1), Body(m2, x2, y2, vx2, vy2)


# ---------------------------------------------------------------------------
# configuration
# ---------------------------------------------------------------------------


class Mass(NamedTuple):
    """One gravitating point mass as the kernels see it (physics/circumbinary.py:41-95)."""

    mass: float = 0.0
    x: float = 0.0
    y: float = 0.0
    vx: float = 0.0
    vy: float = 0.0
    softening_length: float = 0.0
    sink_model: int = 0
    sink_rate: float = 0.0
    sink_radius: float = 0.0

    def args(self, mass_scale=1.0, rate_scale=1.0):
        return (
            self.x,
            self.y,
            self.vx,
            self.vy,
            self.mass * mass_scale,
            self.softening_length,
            self.sink_rate * rate_scale,
            self.sink_radius,
            int(self.sink_model),
        )


SINK_MODELS = dict(inactive=0, acceleration_free=1, torque_free=2, force_free=3)


def binary_masses(a=1.0, m=1.0, q=1.0, e=0.0, softening=0.05, sink_model="torque_free",
                  sink_rate=10.0, sink_radius=0.05, x_offset=None):
    """Point-mass callback of the circumbinary setups (circumbinary_disk.py:194-212)."""
    model = SINK_MODELS[sink_model]

    def masses(t):
        b1, b2 = kepler_state(t, a, m, q, e)
        return tuple(
            Mass(b.mass, b.x if x_offset is None else b.x + x_offset, b.y, b.vx, b.vy,
                 softening, model, sink_rate, sink_radius)
            for b in (b1, b2)
        )

    return masses


class Config(NamedTuple):
    """Everything the solver adapter passes to the kernels, as plain values."""

    x0: float
    x1: float
    y0: float
    y1: float
    ni: int
    nj: int
    eos_type: int = 2  # 1 globally, 2 locally isothermal
    sound_speed: float = 1.0
    mach_number: float = 10.0
    nu: float = 0.0
    buffer_is_enabled: bool = False
    buffer_driving_rate: float = 1000.0
    buffer_onset_width: float = 0.1
    buffer_surface_density: float = 0.0
    masses: Optional[Callable[[float], Sequence[Mass]]] = None
    velocity_ceiling: float = 1e12
    density_floor: float = 1e-12
    rk_order: int = 2
    plm_theta: float = 1.8
    reference_time_scale: float = 2.0 * math.pi

    @property
    def dx(self):
        return (self.x1 - self.x0) / self.ni

    @property
    def dy(self):
        return (self.y1 - self.y0) / self.nj

    def point_masses(self, t):
        if self.masses is None:
            return Mass(), Mass()
        ms = self.masses(t)
        if isinstance(ms, Mass):
            return ms, Mass()
        if len(ms) == 1:
            return ms[0], Mass()
        return tuple(ms)


# ---------------------------------------------------------------------------
# initial data (vectorised; equal to the per-cell setup.primitive loop)
# ---------------------------------------------------------------------------


def cell_centres(cfg: Config):
    """mesh.py:237-240 on the whole grid."""
    i = np.arange(cfg.ni, dtype=np.float64)[:, None]
    j = np.arange(cfg.nj, dtype=np.float64)[None, :]
    x = cfg.x0 + (i + 0.5) * cfg.dx
    y = cfg.y0 + (j + 0.5) * cfg.dy
    return np.broadcast_to(x, (cfg.ni, cfg.nj)), np.broadcast_to(y, (cfg.ni, cfg.nj))


def circumbinary_disk_primitive(x, y, softening=0.05, initial_sigma=1.0):
    """CircumbinaryDisk.primitive, isothermal branch (circumbinary_disk.py:82-94)."""
    r = np.sqrt(x * x + y * y)
    rs = np.sqrt(x * x + y * y + softening * softening)
    px = -y / np.maximum(r, 1e-12)
    py = +x / np.maximum(r, 1e-12)
    out = np.empty(np.broadcast(x, y).shape + (3,))
    out[..., 0] = initial_sigma
    out[..., 1] = np.sqrt(1.0 / rs) * px
    out[..., 2] = np.sqrt(1.0 / rs) * py
    return out


def seeded_noise(ni, nj, seed, amplitude=1e-3):
    """Uniform noise in [-amplitude, amplitude) on the surface density, i-major."""
    rng = np.random.default_rng(seed)
    return amplitude * rng.uniform(-1.0, 1.0, size=(ni, nj))


# ---------------------------------------------------------------------------
# kernel backends
# ---------------------------------------------------------------------------

_DP = POINTER(c_double)


def _ptr(a):
    return a.ctypes.data_as(_DP)


class Kernels:
    """Thin ctypes facade over either the oracle C restatement or oracle/_ref."""

    def __init__(self, kind="oracle", theta=1.8, threads="omp"):
        self.kind = kind
        self.theta = float(theta)
        if kind == "oracle":
            path = os.path.join(HERE, "_build", "liboracle_cbdiso.so")
            if not os.path.exists(path):
                from oracle.build import build_oracle

                build_oracle()
            self.lib = ctypes.CDLL(path)
            prefix = "oracle_cbdiso_2d_"
        elif kind == "ref":
            tag = {1.8: "t18", 1.5: "t15"}[self.theta]
            path = os.path.join(HERE, "_ref", f"libref_{tag}_{'omp' if threads == 'omp' else 'cpu'}.so")
            if not os.path.exists(path):
                raise FileNotFoundError(f"{path} missing: run oracle/build_ref.sh where the reference tree exists")
            self.lib = ctypes.CDLL(path)
            prefix = "cbdiso_2d_"
        else:
            raise ValueError(kind)
        I, D, P = c_int, c_double, _DP
        m9 = [D] * 8 + [I]
        self.f_advance = getattr(self.lib, prefix + "advance_rk")
        self.f_advance.argtypes = (
            [I, I, D, D, D, D, P, P, P, D, D, D, D, D, I] + m9 + m9 + [D, D, I, D, D, D, D, D]
            + ([D] if kind == "oracle" else [])
        )
        self.f_p2c = getattr(self.lib, prefix + "primitive_to_conserved")
        self.f_p2c.argtypes = [I, I, P, P]
        self.f_src = getattr(self.lib, prefix + "point_mass_source_term")
        self.f_src.argtypes = [I, I, D, D, D, D] + m9 + [P, P]
        self.f_ws = getattr(self.lib, prefix + "wavespeed")
        self.f_ws.argtypes = [I, I, D, D, D, D, D, D, I] + m9 + m9 + [P, P]
        for f in (self.f_advance, self.f_p2c, self.f_src, self.f_ws):
            f.restype = None

    def advance_rk(self, ni, nj, xl, xr, yl, yr, u0, prd, pwr, buf, m1, m2, cs2, mach2, eos, nu, a, dt, vmax, rmin):
        extra = (self.theta,) if self.kind == "oracle" else ()
        self.f_advance(ni, nj, xl, xr, yl, yr, _ptr(u0), _ptr(prd), _ptr(pwr), *buf, *m1.args(), *m2.args(),
                       cs2, mach2, eos, nu, a, dt, vmax, rmin, *extra)

    def primitive_to_conserved(self, ni, nj, p, u):
        self.f_p2c(ni, nj, _ptr(p), _ptr(u))

    def point_mass_source_term(self, ni, nj, xl, xr, yl, yr, margs, p, rate):
        self.f_src(ni, nj, xl, xr, yl, yr, *margs, _ptr(p), _ptr(rate))

    def wavespeed(self, ni, nj, xl, xr, yl, yr, cs2, mach2, eos, m1, m2, p, ws):
        self.f_ws(ni, nj, xl, xr, yl, yr, cs2, mach2, eos, *m1.args(), *m2.args(), _ptr(p), _ptr(ws))


# ---------------------------------------------------------------------------
# the solver adapter (cbdiso_2d.py:49-590), one patch
# ---------------------------------------------------------------------------


class OracleSolver:
    """
    Single-patch restatement of cbdiso_2d.Solver. A one-patch run equals the
    reference's multi-patch run exactly: its guard-zone exchange followed by
    zero-gradient edges (cbdiso_2d.py:553-586) is equivalent to clamping
    indices into the whole grid.
    """

    def __init__(self, cfg: Config, primitive: np.ndarray, time: float = 0.0, kernels: Optional[Kernels] = None):
        self.cfg = cfg
        self.k = kernels or Kernels("oracle", cfg.plm_theta)
        ni, nj = cfg.ni, cfg.nj
        self.p1 = np.zeros((ni + 2 * NG, nj + 2 * NG, NQ))
        self.p1[NG:-NG, NG:-NG] = primitive
        self.p2 = self.p1.copy()
        self.u0 = np.zeros_like(self.p1)
        self.ws = np.zeros(self.p1.shape[:2])
        self.time = self.time0 = float(time)
        # patch bounds from vertex coordinates (cbdiso_2d.py:79-80, mesh.py:242-248)
        self.xl = cfg.x0 + 0 * cfg.dx
        self.yl = cfg.y0 + 0 * cfg.dy
        self.xr = cfg.x0 + ni * cfg.dx
        self.yr = cfg.y0 + nj * cfg.dy
        if cfg.buffer_is_enabled:
            self.buffer_outer_radius = cfg.x1
        else:
            self.buffer_outer_radius = 0.0

    @property
    def solution(self):
        return self.p1[NG:-NG, NG:-NG].copy()

    def _set_bc(self):
        p = self.p1
        for i in range(NG):
            p[i] = p[NG]
        for i in range(p.shape[0] - NG, p.shape[0]):
            p[i] = p[-NG - 1]
        for j in range(NG):
            p[:, j] = p[:, NG]
        for j in range(p.shape[1] - NG, p.shape[1]):
            p[:, j] = p[:, -NG - 1]

    def maximum_wavespeed(self):
        c = self.cfg
        m1, m2 = c.point_masses(self.time)
        self.k.wavespeed(c.ni, c.nj, self.xl, self.xr, self.yl, self.yr, c.sound_speed ** 2, c.mach_number ** 2,
                         c.eos_type, m1, m2, self.p1, self.ws)
        return float(self.ws.max())

    def _advance_rk(self, a, dt):
        c = self.cfg
        self._set_bc()
        m1, m2 = c.point_masses(self.time)
        buf = (c.buffer_surface_density, m1.mass + m2.mass, c.buffer_driving_rate, self.buffer_outer_radius,
               c.buffer_onset_width, int(c.buffer_is_enabled))
        self.k.advance_rk(c.ni, c.nj, self.xl, self.xr, self.yl, self.yr, self.u0, self.p1, self.p2, buf, m1, m2,
                          c.sound_speed ** 2, c.mach_number ** 2, c.eos_type, c.nu, a, dt, c.velocity_ceiling,
                          c.density_floor)
        self.time = self.time0 * a + (self.time + dt) * (1.0 - a)
        self.p1, self.p2 = self.p2, self.p1

    def advance(self, dt):
        c = self.cfg
        self.time0 = self.time
        self.k.primitive_to_conserved(c.ni, c.nj, self.p1, self.u0)
        for a in {1: (0.0,), 2: (0.0, 0.5), 3: (0.0, 0.75, 1.0 / 3.0)}[c.rk_order]:
            self._advance_rk(a, dt)

    def source_rates(self, which, gravity=False, accretion=False):
        """cbdiso_2d.py:105-137: interior view of one mass's source rates."""
        c = self.cfg
        m = c.point_masses(self.time)[which - 1]
        rate = np.zeros_like(self.u0)
        self.k.point_mass_source_term(c.ni, c.nj, self.xl, self.xr, self.yl, self.yr,
                                      m.args(float(gravity), float(accretion)), self.p1, rate)
        return rate[NG:-NG, NG:-NG]

    def reductions(self, diagnostics, num_patches=1, absolute=False):
        """
        cbdiso_2d.py:370-503 with the same numpy arithmetic. `num_patches`
        reproduces the reference's summation order for a run split into that
        many slabs along i (subdivide.py:35-60): per-slab sums of per-slab
        fields, then their sum. With `absolute`, sums |f| instead of f: the
        scale against which a cancelling sum's rounding error is measured.
        """
        c = self.cfg
        acc = [self.source_rates(1, accretion=True), self.source_rates(2, accretion=True)]
        grv = [self.source_rates(1, gravity=True), self.source_rates(2, gravity=True)]
        dx, dy = c.dx, c.dy
        prim_all = self.p1[NG:-NG, NG:-NG]
        slabs = []
        a = 0
        for n in range(num_patches):
            b = a + c.ni // num_patches + (1 if n < c.ni % num_patches else 0)
            slabs.append((a, b))
            a = b

        def slab_sum(d, a, b):
            xl = c.x0 + a * dx
            xr = c.x0 + b * dx
            x = np.linspace(xl + 0.5 * dx, xr - 0.5 * dx, b - a)[:, None]
            y = np.linspace(self.yl + 0.5 * dy, self.yr - 0.5 * dy, c.nj)[None, :]
            r = (x ** 2 + y ** 2) ** 0.5
            prim = prim_all[a:b]

            def cut(f, rc):
                if rc is None:
                    return f
                r0, r1 = rc
                return f * (r0 < r) * (r < r1)

            def field(d, q=None):
                quantity = d.get("quantity")
                rc = d.get("radial_cut")
                mass = d.get("which_mass")
                if q is None:
                    if quantity == "mdot":
                        q = 0
                    elif quantity == "fx":
                        q = 1
                    elif quantity == "fy":
                        q = 2
                    elif quantity == "torque":
                        return x * field(d, 2) - y * field(d, 1)
                    elif quantity == "sigma_m1":
                        return cut(prim[..., 0], rc) * (x / r + 1.0j * (y / r))
                    elif quantity == "eccentricity_vector":
                        s, vx, vy = (cut(prim[..., k], rc) for k in range(3))
                        vv = vx * vx + vy * vy
                        vr = vx * x + vy * y
                        ex = (vv * x - vr * vx) / 1.0 - x / r
                        ey = (vv * y - vr * vy) / 1.0 - y / r
                        return s * (ex + 1.0j * ey)
                    elif quantity == "angular_momentum":
                        s, vx, vy = (cut(prim[..., k], rc) for k in range(3))
                        return s * (x * vy - y * vx)
                    elif quantity == "mass":
                        return cut(prim[..., 0], rc)
                    elif quantity == "power":
                        fx, fy = field(d, 1), field(d, 2)
                        m1, m2 = c.point_masses(self.time)
                        if mass == 1:
                            return m1.vx * fx + m1.vy * fy
                        if mass == 2:
                            return m2.vx * fx + m2.vy * fy
                        raise ValueError("Mass option for 'power' must be 1 or 2.")
                    else:
                        raise ValueError(quantity)
                rates = acc if d.get("accretion") else grv
                if mass == "both":
                    f = rates[0][a:b, :, q] + rates[1][a:b, :, q]
                elif mass == 1:
                    f = rates[0][a:b, :, q]
                else:
                    f = rates[1][a:b, :, q]
                return cut(f, rc)

            f = field(d)
            return np.abs(f).sum() if absolute else f.sum()

        out = []
        for d in diagnostics:
            if d["quantity"] == "time":
                out.append(self.time / c.reference_time_scale)
            else:
                out.append(sum(slab_sum(d, a, b) for a, b in slabs) * (dx * dy))
        return out


def driver_dt(solver: OracleSolver, cfl: float) -> float:
    """driver.py:508-510 with new_timestep_cadence = 1."""
    c = solver.cfg
    return min(c.dx, c.dy) / solver.maximum_wavespeed() * cfl


def run(solver: OracleSolver, steps: int, cfl: float = 0.3, diagnostics=None, num_patches=1):
    """Advance `steps` iterations; returns (dts, time series rows)."""
    dts, series = [], []
    for _ in range(steps):
        dt = driver_dt(solver, cfl)
        solver.advance(dt)
        dts.append(dt)
        if diagnostics:
            series.append(solver.reductions(diagnostics, num_patches))
    return dts, series
