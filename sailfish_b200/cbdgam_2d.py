"""
Drop-in replacement for sailfish's gamma-law circumbinary-disk solver
adapter, cbdgam_2d (sailfish/solvers/cbdgam_2d.py:1-520), running on one
B200.

Same constructor (setup, mesh, time, solution, num_patches, mode, physics,
options), validation errors, properties and methods (`solution`,
`primitive`, `time`, `options`, `physics`, `recommended_cfl`,
`maximum_cfl`, `maximum_wavespeed()`, `advance(dt)`, `reductions()`).

The state stays in device memory in the reference's (ni + 4, nj + 4, 4)
layout (Sigma, vx, vy, pressure). Each RK stage is one kernel of
libcbdiso_b200.so that rebuilds u_n from the step's starting primitives and
writes the zero-gradient guard zones itself, so the reference's separate
primitive-to-conserved and boundary passes disappear; the second stage also
takes the maximum signal speed of the state it writes, so
`maximum_wavespeed()` after `advance()` reads back one double. The whole
grid is one device patch whatever `num_patches` says: the reference's patch
split changes nothing but the summation order of its reductions.

Extra option beyond the reference's (pressure_floor, density_floor,
velocity_ceiling, mach_ceiling): `plm_theta` (default 1.5, the reference's
compile-time PLM_THETA, cbdgam_2d.c:15).
"""

from __future__ import annotations

import ctypes
import math
from logging import getLogger
from typing import NamedTuple

import numpy as np

from . import _capi, _hostio
from .cbdiso_2d import _as_diagnostic, _diag_struct, _mass_struct
from .mesh import is_planar_cartesian_2d
from .physics import MassCache, Physics, enum_value
from .solver_base import SolverBase

logger = getLogger(__name__)

NG = 2
NQ = 4
DEVICE_QUANTITIES = ("mdot", "torque", "sigma_m1", "eccentricity_vector")
COMPLEX_QUANTITIES = ("sigma_m1", "eccentricity_vector")


class Options(NamedTuple):
    """Solver options (cbdgam_2d.py:23-27, plus the PLM parameter and
    `face_cache`: a step's first stage loads the scale-height geometry and
    gravity factors that the previous step's second stage computed for the
    same point masses; the same bits either way)."""

    pressure_floor: float = 1e-12
    density_floor: float = 1e-10
    velocity_ceiling: float = 1e16
    mach_ceiling: float = 1e5
    plm_theta: float = 1.5
    face_cache: bool = True


def initial_condition(setup, mesh, time, rows=None):
    """Primitive data (ni, nj, 4) from a setup (cbdgam_2d.py:30-43), or only
    the rows a <= i < b of it for rows=(a, b); setups with a vectorised
    `primitive_array(t, x, y)` are evaluated at once."""
    ni, nj = mesh.shape
    a, b = rows if rows is not None else (0, ni)
    if hasattr(setup, "primitive_array"):
        i = np.arange(a, b, dtype=np.float64)[:, None]
        j = np.arange(nj, dtype=np.float64)[None, :]
        x = np.broadcast_to(mesh.x0 + (i + 0.5) * mesh.dx, (b - a, nj))
        y = np.broadcast_to(mesh.y0 + (j + 0.5) * mesh.dy, (b - a, nj))
        out = np.ascontiguousarray(setup.primitive_array(time, x, y), dtype=np.float64)
        if out.shape == (b - a, nj, NQ):
            return out
    primitive = np.zeros([b - a, nj, NQ])
    for i in range(a, b):
        for j in range(nj):
            setup.primitive(time, mesh.cell_coordinates(i, j), primitive[i - a, j])
    return primitive


class Solver(SolverBase):
    """Adapter driving the gamma-law sm_100a kernels of libcbdiso_b200.so."""

    def __init__(self, setup=None, mesh=None, time=0.0, solution=None, num_patches=1, mode="gpu",
                 physics=dict(), options=dict(), index_range=None):
        """
        `index_range` (a, b) makes this solver one patch of the mesh: rows
        a <= i < b, with the patch's own edge coordinates as the reference's
        Patch has them (cbdgam_2d.py:66-78); `solution` is then the whole
        mesh's or the patch's. The multi-GPU solver (distributed.py) runs one
        patch per rank and exchanges the guard rows between stages.
        """
        import torch

        physics = dict(physics)
        physics["diagnostics"] = [_as_diagnostic(v) for v in physics.get("diagnostics", [])]
        self._physics = physics = Physics(**physics)
        self._options = options = Options(**options)

        # the reference's checks and messages (cbdgam_2d.py:251-264)
        if not is_planar_cartesian_2d(mesh):
            raise ValueError("solver only supports 2D cartesian mesh")
        if setup.boundary_condition != "outflow":
            raise ValueError("solver only supports outflow boundary condition")
        if enum_value(physics.viscosity_model) not in (0, 2):
            raise ValueError("solver only supports constant-alpha viscosity")
        if enum_value(physics.eos_type) != 3:
            raise ValueError("solver only supports isothermal equation of states")
        if not 1.0 <= options.plm_theta <= 2.0:
            raise ValueError(f"plm_theta must be in [1, 2], got {options.plm_theta}")
        if not torch.cuda.is_available():
            raise RuntimeError("sailfish_b200 needs a CUDA device (there is no CPU fallback)")

        self._lib = _capi.lib()
        self.mesh = mesh
        self.setup = setup
        self.num_guard = NG
        self.num_cons = NQ
        self.num_patches = num_patches
        self.device = torch.device("cuda", torch.cuda.current_device())
        ni_mesh, nj = mesh.shape
        a, b = index_range if index_range is not None else (0, ni_mesh)
        if not 0 <= a < b <= ni_mesh:
            raise ValueError(f"index_range {index_range} is outside the mesh's {ni_mesh} rows")
        self.index_range = (a, b)
        ni = b - a
        # called after each RK stage with (stage, output buffer) and after each
        # step, on the launching stream (the multi-GPU solver's exchanges)
        self._stage_hook = None
        self._step_hook = None

        logger.info(f"initiate with time={time:0.4f}")
        logger.info(f"mesh is {mesh}")
        logger.info("boundary condition is outflow")

        if solution is None:
            primitive = initial_condition(setup, mesh, time, rows=(a, b))
        else:
            primitive = np.asarray(solution, dtype=np.float64)
        if primitive.shape == (ni_mesh, nj, NQ) and ni != ni_mesh:
            primitive = primitive[a:b]
        if primitive.shape != (ni, nj, NQ):
            raise ValueError(f"solution has shape {primitive.shape}, expected {(ni, nj, NQ)}")

        if physics.buffer_is_enabled:
            # the buffer's targets are the setup's data at the onset radius on
            # the x axis (cbdgam_2d.py:293-306)
            buffer_prim = [0.0] * 4
            buffer_outer_radius = mesh.x1
            buffer_onset_radius = buffer_outer_radius - physics.buffer_onset_width
            setup.primitive(time, [buffer_onset_radius, 0.0], buffer_prim)
            buffer_surface_density = buffer_prim[0]
            buffer_surface_pressure = buffer_prim[3]
        else:
            buffer_outer_radius = 0.0
            buffer_surface_density = 0.0
            buffer_surface_pressure = 0.0

        g = _capi.GamGrid()
        g.ni, g.nj = ni, nj
        g.xl, g.yl = mesh.vertex_coordinates(a, 0)
        g.xr, g.yr = mesh.vertex_coordinates(b, nj)
        g.plm_theta = options.plm_theta
        g.gamma_law_index = physics.gamma_law_index
        g.alpha = physics.alpha
        g.cooling_coefficient = physics.cooling_coefficient
        g.mach_ceiling = options.mach_ceiling
        g.velocity_ceiling = options.velocity_ceiling
        g.density_floor = options.density_floor
        g.pressure_floor = options.pressure_floor
        g.constant_softening = int(bool(physics.constant_softening))
        g.buffer_is_enabled = int(bool(physics.buffer_is_enabled))
        g.buffer_surface_density = buffer_surface_density
        g.buffer_surface_pressure = buffer_surface_pressure
        g.buffer_driving_rate = physics.buffer_driving_rate
        g.buffer_outer_radius = buffer_outer_radius
        g.buffer_onset_width = physics.buffer_onset_width
        self._grid = g

        f64 = dict(dtype=torch.float64, device=self.device)
        self._buf = [torch.empty((ni + 2 * NG, nj + 2 * NG, NQ), **f64) for _ in range(2)]
        _hostio.upload(primitive, self._buf[0][NG:-NG, NG:-NG])
        self._check(self._lib.cbdgam_b200_fill_guards(ctypes.byref(g), self._ptr(self._buf[0]), self._stream()),
                    "fill_guards")
        nscratch = int(self._lib.cbdgam_b200_scratch_bytes(ctypes.byref(g)))
        self._scratch = torch.zeros(nscratch // 8 + 8, **f64)
        self._fcache = None
        if self._options.face_cache:
            self._fcache = torch.empty(int(self._lib.cbdgam_b200_face_cache_bytes(ctypes.byref(g))) // 8, **f64)
            self._fcache[:32].zero_()
        # the wavespeed maximum of the current state (slot 0; the multi-GPU
        # solver all-reduces it in place) and, apart, the diagnostic sums
        self._result = torch.zeros(1 + 2 * _capi.GAM_MAX_DIAG, **f64)
        self._sums = torch.zeros(1 + 2 * _capi.GAM_MAX_DIAG, **f64)
        self._result_host = torch.zeros(1 + 2 * _capi.GAM_MAX_DIAG, dtype=torch.float64).pin_memory()
        self._ws_valid = False
        self._time = float(time)
        self.h2d_bytes = 0
        self.d2h_bytes = 0

    # ------------------------------------------------------------------
    # helpers
    # ------------------------------------------------------------------

    @staticmethod
    def _ptr(t):
        return ctypes.c_void_p(t.data_ptr())

    @staticmethod
    def _stream():
        import torch

        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def _check(status, where):
        _capi.check(status, where)

    def _stage(self, time, a, dt):
        st = _capi.GamStage()
        m1, m2 = self._point_masses(time)
        _mass_struct(m1, st.mass[0])
        _mass_struct(m2, st.mass[1])
        st.buffer_central_mass = m1.mass + m2.mass
        st.a, st.dt = a, dt
        return st

    def _launch(self, st, rd, pn, wr, ws, role, stream):
        """One product stage; `role` (1 writer, 2 reader) is used when the
        solver keeps a face cache."""
        lib, g = self._lib, self._grid
        args = (ctypes.byref(g), ctypes.byref(st), self._ptr(rd), self._ptr(pn) if pn is not None else None,
                self._ptr(wr), self._ptr(ws) if ws is not None else None)
        if self._fcache is not None and role:
            status = lib.cbdgam_b200_advance_stage_cached(*args, self._ptr(self._fcache), role, stream)
        else:
            status = lib.cbdgam_b200_advance_stage(*args, stream)
        self._check(status, "advance_stage")

    @staticmethod
    def _same_masses(a, b):
        """Whether two stages' masses agree in every input of the cached
        values (position, mass, softening)."""
        return all(x.x == y.x and x.y == y.y and x.mass == y.mass and x.softening_length == y.softening_length
                   for x, y in zip(a.mass, b.mass))

    def _point_masses(self, t):
        masses = self.__dict__.get("_mass_cache")
        if masses is None or masses.physics is not self._physics:
            masses = self._mass_cache = MassCache(self._physics)
        return masses(t)

    def _read(self, n, source=None):
        import torch

        source = self._result if source is None else source
        self._result_host[:n].copy_(source[:n], non_blocking=True)
        torch.cuda.current_stream().synchronize()
        self.d2h_bytes += 8 * n
        return self._result_host[:n].numpy().copy()

    def _reduce(self, diags):
        """The sums of `diags` (at most 4) on the current state into
        self._sums; with no diagnostics, the wavespeed maximum into
        self._result."""
        masses = (_capi.Mass * 2)()
        m1, m2 = self._point_masses(self._time)
        _mass_struct(m1, masses[0])
        _mass_struct(m2, masses[1])
        structs = (_capi.Diag * max(1, len(diags)))()
        for k, d in enumerate(diags):
            _diag_struct(d, structs[k])
        out = self._sums if diags else self._result
        self._check(self._lib.cbdgam_b200_reduce(ctypes.byref(self._grid), masses, structs, len(diags),
                                                 self._ptr(self._buf[0]), self._ptr(self._scratch),
                                                 self._ptr(out), self._stream()), "reduce")
        if not diags:
            self._ws_valid = True

    # ------------------------------------------------------------------
    # SolverBase
    # ------------------------------------------------------------------

    @property
    def solution(self):
        return _hostio.download(self._buf[0][NG:-NG, NG:-NG])

    @property
    def primitive(self):
        """This solver uses primitive data as the solution array."""
        return None

    @property
    def time(self):
        return self._time

    @property
    def options(self):
        return self._options._asdict()

    @property
    def physics(self):
        return self._physics._asdict()

    @property
    def recommended_cfl(self):
        return 0.1

    @property
    def maximum_cfl(self):
        return 0.4

    def maximum_wavespeed(self):
        """Largest |v +- cs| over the grid (cbdgam_2d.c:685-708). Raises
        CbdError (CBD_ERR_NONFINITE) when it is not finite (a NaN or infinity
        in the state), where the reference returns it and runs on."""
        if not self._ws_valid:
            self._reduce([])
        value = float(self._read(1)[0])
        if not math.isfinite(value):
            raise _capi.CbdError(_capi.NONFINITE, "maximum_wavespeed")
        return value

    def advance(self, dt):
        """One RK2 step (cbdgam_2d.py:473-489): two stage kernels, masses at
        each stage's start time, the stage times as the reference updates
        them."""
        dt = float(dt)
        if not math.isfinite(dt):
            raise _capi.CbdError(_capi.NONFINITE, "advance: time step")
        lib, g = self._lib, self._grid
        stream = self._stream()
        t0 = self._time
        t1 = t0 * 0.0 + (t0 + dt) * (1.0 - 0.0)
        t2 = t0 * 0.5 + (t1 + dt) * (1.0 - 0.5)
        a_buf, b_buf = self._buf
        s1 = self._stage(t0, 0.0, dt)
        self._result[:1].zero_()
        self._launch(s1, a_buf, None, b_buf, None, 2, stream)
        if self._stage_hook is not None:
            self._stage_hook(0, b_buf)
        # the second stage's orbit is solved while the first stage runs; it
        # fills the face cache when its masses are the step's end masses
        s2 = self._stage(t1, 0.5, dt)
        writer = self._same_masses(s2, self._stage(t2, 0.5, dt))
        self._launch(s2, b_buf, a_buf, a_buf, self._result, 1 if writer else 0, stream)
        if self._stage_hook is not None:
            self._stage_hook(1, a_buf)
        self._time = t2
        self._ws_valid = True
        if self._step_hook is not None:
            self._step_hook()

    # hooks of the multi-GPU solver (distributed.py)

    def state_buffer(self):
        """The padded device state (its guard rows are exchanged in place)."""
        return self._buf[0]

    def wavespeed_buffer(self):
        """One-element device view holding the wavespeed maximum of the
        current state once ensure_wavespeed() has run."""
        return self._result[0:1]

    def ensure_wavespeed(self):
        """Compute the wavespeed maximum of the current state if it is not
        already known; True if it was computed now."""
        if self._ws_valid:
            return False
        self._reduce([])
        return True

    def wavespeed_changed(self):
        """The wavespeed buffer was rewritten on the device (all-reduced);
        nothing of it is cached on the host."""

    def _device_sums(self):
        diagnostics = self._physics.diagnostics
        device = [d for d in diagnostics if d.quantity != "time"]
        for d in device:
            if d.quantity not in DEVICE_QUANTITIES:
                raise ValueError(f"cbdgam_2d has no diagnostic {d.quantity}")
            if d.quantity in ("mdot", "torque"):
                if not (d.accretion or d.gravity):
                    raise ValueError(f"diagnostic {d.quantity} needs gravity or accretion")
                if d.which_mass not in (1, 2, "both"):
                    raise ValueError(f"which_mass must be 1, 2 or 'both', got {d.which_mass}")
        sums = []
        for first in range(0, len(device), _capi.GAM_MAX_DIAG):
            chunk = device[first:first + _capi.GAM_MAX_DIAG]
            self._reduce(chunk)
            res = self._read(1 + 2 * len(chunk), self._sums)
            sums += [(res[1 + 2 * k], res[2 + 2 * k]) for k in range(len(chunk))]
        return device, sums

    def reduction_sums(self):
        """The diagnostic sums over this solver's zones before the dx dy
        factor (float or complex per non-time diagnostic)."""
        device, sums = self._device_sums()
        return [complex(re, im) if d.quantity in COMPLEX_QUANTITIES else float(re)
                for d, (re, im) in zip(device, sums)]

    def reductions(self):
        """
        Time series row in the order of physics.diagnostics
        (cbdgam_2d.py:341-447): time in units of the setup's reference time
        scale, then each sum times dx dy; sigma_m1 and eccentricity_vector
        are complex. mdot and torque take the accretion rates when the
        diagnostic asks for accretion, else the gravity rates.
        """
        diagnostics = self._physics.diagnostics
        _, sums = self._device_sums()
        da = self.mesh.dx * self.mesh.dy
        out, k = [], 0
        for d in diagnostics:
            if d.quantity == "time":
                out.append(self._time / self.setup.reference_time_scale)
                continue
            re, im = sums[k]
            k += 1
            out.append(complex(re, im) * da if d.quantity in COMPLEX_QUANTITIES else float(re) * da)
        return out


def main(argv=None):
    """A gamma-law circumbinary disk driven as the reference's driver does
    (dt = CFL min(dx, dy) / max wavespeed every step; a profiling and smoke
    case): python -m sailfish_b200.cbdgam_2d --resolution 2048 --steps 10"""
    import argparse
    import time

    import torch

    from .setups import CircumbinaryDisk

    p = argparse.ArgumentParser(description=main.__doc__)
    p.add_argument("--resolution", type=int, default=1024)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--cfl", type=float, default=0.1)
    p.add_argument("--alpha", type=float, default=0.1)
    p.add_argument("--cooling", type=float, default=0.0)
    a = p.parse_args(argv)
    setup = CircumbinaryDisk(eos="gamma-law", alpha=a.alpha, cooling_coefficient=a.cooling)
    mesh = setup.mesh(a.resolution)
    s = Solver(setup=setup, mesh=mesh, physics=setup.physics)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        s.advance(mesh.min_spacing() / s.maximum_wavespeed() * a.cfl)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    print(f"{a.steps} steps at {a.resolution}^2: {el / a.steps * 1e3:.3f} ms/step, "
          f"{a.resolution ** 2 * a.steps / el:.3e} zone-updates/s, t = {s.time:.6f}, "
          f"max wavespeed {s.maximum_wavespeed():.6f}")


if __name__ == "__main__":
    main()
