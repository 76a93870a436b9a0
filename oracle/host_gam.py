"""
Host-side restatement of sailfish's gamma-law circumbinary-disk solver
adapter (sailfish/solvers/cbdgam_2d.py) over either the oracle C kernels
(oracle/cbdgam_2d_oracle.c) or the reference's own build (oracle/_ref).

TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and bench.py's
CPU leg to check and time the CUDA product; never by the product itself.
"""

from __future__ import annotations

import ctypes
import math
import os
from ctypes import POINTER, c_double, c_int
from typing import Callable, NamedTuple, Optional, Sequence

import numpy as np

from .host import Mass, binary_masses  # noqa: F401  (shared point-mass model)

HERE = os.path.dirname(os.path.abspath(__file__))
NG = 2
NF = 4


class GamConfig(NamedTuple):
    """Everything the gamma-law adapter passes to the kernels."""

    x0: float
    x1: float
    y0: float
    y1: float
    ni: int
    nj: int
    gamma_law_index: float = 5.0 / 3.0
    alpha: float = 0.0
    cooling_coefficient: float = 0.0
    constant_softening: bool = True
    buffer_is_enabled: bool = False
    buffer_driving_rate: float = 1000.0
    buffer_onset_width: float = 0.1
    buffer_surface_density: float = 0.0
    buffer_surface_pressure: float = 0.0
    masses: Optional[Callable[[float], Sequence[Mass]]] = None
    pressure_floor: float = 1e-12
    density_floor: float = 1e-10
    velocity_ceiling: float = 1e16
    mach_ceiling: float = 1e5
    plm_theta: float = 1.5
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
        return tuple(self.masses(t))


def gamma_disk_primitive(x, y, softening=0.05, sigma0=1.0, pressure0=1e-2):
    """The gamma-law branch of CircumbinaryDisk.primitive
    (setups/circumbinary_disk.py:95-110), zone by zone in Python floats."""
    r = math.sqrt(x * x + y * y)
    rs = math.sqrt(x * x + y * y + softening * softening)
    phx, phy = -y / max(r, 1e-12), +x / max(r, 1e-12)
    taper = 0.0001 + 0.9999 * math.exp(-((1.0 / rs) ** 30))
    return (sigma0 * rs ** (-3.0 / 5.0) * taper, math.sqrt(1.0 / rs) * phx, math.sqrt(1.0 / rs) * phy,
            pressure0 * rs ** (-3.0 / 2.0) * taper)


_DP = POINTER(c_double)


def _ptr(a):
    return a.ctypes.data_as(_DP)


class GamKernels:
    """ctypes facade over the gamma-law oracle or the reference build."""

    def __init__(self, kind="oracle", theta=1.5, threads="omp"):
        self.kind = kind
        self.theta = float(theta)
        if kind == "oracle":
            path = os.path.join(HERE, "_build", "liboracle_cbdgam.so")
            if not os.path.exists(path):
                from oracle.build import build_oracle

                build_oracle()
            prefix = "oracle_cbdgam_2d_"
        elif kind == "ref":
            if self.theta != 1.5:
                raise ValueError("the reference gamma-law kernels are built with theta 1.5")
            path = os.path.join(HERE, "_ref", f"libref_gam_{'omp' if threads == 'omp' else 'cpu'}.so")
            if not os.path.exists(path):
                raise FileNotFoundError(f"{path} missing: run oracle/build_ref.sh where the reference tree exists")
            prefix = "cbdgam_2d_"
        else:
            raise ValueError(kind)
        self.lib = ctypes.CDLL(path)
        I, D, P = c_int, c_double, _DP
        m9 = [D] * 8 + [I]
        self.f_advance = getattr(self.lib, prefix + "advance_rk")
        self.f_advance.argtypes = ([I, I, D, D, D, D, P, P, P, D, D, D, D, D, D, D, I] + m9 + m9
                                   + [D, D, D, D, D, D, D, D, I] + ([D] if kind == "oracle" else []))
        self.f_ws = getattr(self.lib, prefix + "wavespeed")
        self.f_ws.argtypes = [I, I, P, P, D]
        self.f_p2c = getattr(self.lib, prefix + "primitive_to_conserved")
        self.f_p2c.argtypes = [I, I, P, P, D]
        self.f_src = getattr(self.lib, prefix + "point_mass_source_term")
        self.f_src.argtypes = [I, I, D, D, D, D] + m9 + m9 + [I, P, P, I, D]
        for f in (self.f_advance, self.f_ws, self.f_p2c, self.f_src):
            f.restype = None

    def advance_rk(self, c: GamConfig, xl, xr, yl, yr, u0, prd, pwr, buf, m1, m2, a, dt):
        extra = (self.theta,) if self.kind == "oracle" else ()
        self.f_advance(c.ni, c.nj, xl, xr, yl, yr, _ptr(u0), _ptr(prd), _ptr(pwr), c.gamma_law_index, *buf,
                       *m1.args(), *m2.args(), c.alpha, a, dt, c.velocity_ceiling, c.cooling_coefficient,
                       c.mach_ceiling, c.density_floor, c.pressure_floor, int(c.constant_softening), *extra)

    def wavespeed(self, ni, nj, p, ws, gamma):
        self.f_ws(ni, nj, _ptr(p), _ptr(ws), gamma)

    def primitive_to_conserved(self, ni, nj, p, u, gamma):
        self.f_p2c(ni, nj, _ptr(p), _ptr(u), gamma)

    def point_mass_source_term(self, ni, nj, xl, xr, yl, yr, m1args, m2args, which, p, rate, constant_softening,
                               gamma):
        self.f_src(ni, nj, xl, xr, yl, yr, *m1args, *m2args, which, _ptr(p), _ptr(rate), int(constant_softening),
                   gamma)


class GamOracleSolver:
    """
    One-patch restatement of cbdgam_2d.Solver (cbdgam_2d.py:226-520): RK2,
    zero-gradient guards before each stage, the reductions' per-patch
    summation order.
    """

    def __init__(self, cfg: GamConfig, primitive, time=0.0, kernels: Optional[GamKernels] = None):
        self.cfg = cfg
        self.k = kernels or GamKernels("oracle", cfg.plm_theta)
        ni, nj = cfg.ni, cfg.nj
        self.p1 = np.zeros((ni + 2 * NG, nj + 2 * NG, NF))
        self.p1[NG:-NG, NG:-NG] = primitive
        self.p2 = self.p1.copy()
        self.u0 = np.zeros_like(self.p1)
        self.ws = np.zeros(self.p1.shape[:2])
        self.time = self.time0 = float(time)
        self.xl = cfg.x0 + 0 * cfg.dx
        self.yl = cfg.y0 + 0 * cfg.dy
        self.xr = cfg.x0 + ni * cfg.dx
        self.yr = cfg.y0 + nj * cfg.dy
        self.buffer_outer_radius = cfg.x1 if cfg.buffer_is_enabled else 0.0

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
        self.k.wavespeed(c.ni, c.nj, self.p1, self.ws, c.gamma_law_index)
        return float(self.ws.max())

    def _advance_rk(self, a, dt):
        c = self.cfg
        self._set_bc()
        m1, m2 = c.point_masses(self.time)
        buf = (c.buffer_surface_density, c.buffer_surface_pressure, m1.mass + m2.mass, c.buffer_driving_rate,
               self.buffer_outer_radius, c.buffer_onset_width, int(c.buffer_is_enabled))
        self.k.advance_rk(c, self.xl, self.xr, self.yl, self.yr, self.u0, self.p1, self.p2, buf, m1, m2, a, dt)
        self.time = self.time0 * a + (self.time + dt) * (1.0 - a)
        self.p1, self.p2 = self.p2, self.p1

    def advance(self, dt):
        c = self.cfg
        self.time0 = self.time
        self.k.primitive_to_conserved(c.ni, c.nj, self.p1, self.u0, c.gamma_law_index)
        self._advance_rk(0.0, dt)
        self._advance_rk(0.5, dt)

    def source_rates(self, which, gravity=False, accretion=False):
        c = self.cfg
        m1, m2 = c.point_masses(self.time)
        rate = np.zeros_like(self.p1)
        self.k.point_mass_source_term(c.ni, c.nj, self.xl, self.xr, self.yl, self.yr,
                                      m1.args(float(gravity), float(accretion)),
                                      m2.args(float(gravity), float(accretion)), which, self.p1, rate,
                                      c.constant_softening, c.gamma_law_index)
        return rate[NG:-NG, NG:-NG]

    def reductions(self, diagnostics, num_patches=1, absolute=False):
        """cbdgam_2d.py:338-456 with the same numpy arithmetic; quantities
        mdot, torque, sigma_m1 and eccentricity_vector (with radial cuts)."""
        c = self.cfg
        acc = [self.source_rates(1, accretion=True), self.source_rates(2, accretion=True)]
        grv = [self.source_rates(1, gravity=True), self.source_rates(2, gravity=True)]
        dx, dy = c.dx, c.dy
        prim_all = self.p1[NG:-NG, NG:-NG]
        slabs, a = [], 0
        for n in range(num_patches):
            b = a + c.ni // num_patches + (1 if n < c.ni % num_patches else 0)
            slabs.append((a, b))
            a = b

        def slab_sum(d, a, b):
            xl, xr = c.x0 + a * dx, c.x0 + b * dx
            x = np.linspace(xl + 0.5 * dx, xr - 0.5 * dx, b - a)[:, None]
            y = np.linspace(self.yl + 0.5 * dy, self.yr - 0.5 * dy, c.nj)[None, :]
            r = (x ** 2 + y ** 2) ** 0.5
            prim = prim_all[a:b]
            rc = d.get("radial_cut")

            def cut(f):
                if rc is None:
                    return f
                return f * (rc[0] < r) * (r < rc[1])

            def rates(q):
                mass = d.get("which_mass")
                rs = acc if d.get("accretion") else grv
                if mass == "both":
                    f = rs[0][a:b, :, q] + rs[1][a:b, :, q]
                elif mass == 1:
                    f = rs[0][a:b, :, q]
                else:
                    f = rs[1][a:b, :, q]
                return cut(f)

            quantity = d["quantity"]
            if quantity == "mdot":
                f = rates(0)
            elif quantity == "torque":
                f = x * rates(2) - y * rates(1)
            elif quantity == "sigma_m1":
                f = cut(prim[..., 0]) * (x / r + 1.0j * (y / r))
            elif quantity == "eccentricity_vector":
                s, vx, vy = (cut(prim[..., k]) for k in range(3))
                vv = vx * vx + vy * vy
                vr = vx * x + vy * y
                f = s * (((vv * x - vr * vx) / 1.0 - x / r) + 1.0j * ((vv * y - vr * vy) / 1.0 - y / r))
            else:
                raise ValueError(f"cbdgam_2d has no diagnostic {quantity}")
            return np.abs(f).sum() if absolute else f.sum()

        out = []
        for d in diagnostics:
            if d["quantity"] == "time":
                out.append(self.time / c.reference_time_scale)
            else:
                out.append(sum(slab_sum(d, a, b) for a, b in slabs) * (dx * dy))
        return out


def driver_dt(solver: GamOracleSolver, cfl: float) -> float:
    """driver.py:508-510"""
    c = solver.cfg
    return min(c.dx, c.dy) / solver.maximum_wavespeed() * cfl
