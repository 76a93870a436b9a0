"""
Drop-in replacement for sailfish's cbdiso_2d solver adapter
(sailfish/solvers/cbdiso_2d.py:1-590), running on one B200.

Same constructor (setup, mesh, time, solution, num_patches, mode, physics,
options), same validation errors, same properties and methods
(`solution`, `primitive`, `time`, `options`, `physics`, `recommended_cfl`,
`maximum_cfl`, `maximum_wavespeed()`, `advance(dt)`, `reductions()`).

What differs is how a step executes. The state stays in device memory in the
reference's (ni + 4, nj + 4, 3) layout; each RK stage is one fused kernel of
libcbdiso_b200.so that also writes the guard zones, so there is no separate
boundary-condition pass and no separate primitive-to-conserved pass; and the
final stage of each step computes the next step's wavespeed maximum and the
diagnostic sums, so `maximum_wavespeed()` and `reductions()` after `advance()`
only read a few doubles back. The whole grid is one device patch whatever
`num_patches` says: the reference's patch split is exact (its guard exchange
followed by zero-gradient edges equals index clamping on the whole grid), so
only its reduction summation order depends on it.

Extra solver options beyond the reference's (velocity_ceiling, density_floor,
rk_order): `plm_theta` (default 1.8, the reference's compile-time
PLM_THETA), `precision` ("exact" | "fma" | "fast"), `fuse_reductions`,
`tile` ((columns, rows[, occupancy]) of the stage kernel's CTA tile, or
None for the library default), and `face_cache` (default True: a step's
first stage loads the face sound speeds and gravity factors that the previous
step's last stage computed for the same point masses, instead of recomputing
them; bit-identical results in EXACT precision).
"""

from __future__ import annotations

import ctypes
import math
from logging import getLogger
from typing import NamedTuple, Optional

import numpy as np

from . import _capi, _hostio
from ._graphs import capture
from .mesh import is_planar_cartesian_2d
from .physics import Diagnostic, MassCache, Physics, enum_value
from .solver_base import SolverBase

logger = getLogger(__name__)

NG = 2
NQ = 3
RK_WEIGHTS = {1: (0.0,), 2: (0.0, 0.5), 3: (0.0, 0.75, 1.0 / 3.0)}
COMPLEX_QUANTITIES = ("sigma_m1", "eccentricity_vector")
# rows of the device time series a run allocates at least: a longer run
# reallocates it, which drops the captured step graphs (they hold its address)
SERIES_ROWS = 1024


class Options(NamedTuple):
    """Solver options (cbdiso_2d.py:23-30, plus this build's extensions)."""

    velocity_ceiling: float = 1e12
    density_floor: float = 1e-12
    rk_order: int = 2
    plm_theta: float = 1.8
    precision: str = "exact"
    fuse_reductions: bool = True
    tile: Optional[tuple] = None
    face_cache: bool = True


def initial_condition(setup, mesh, time, rows=None):
    """
    Primitive data (ni, nj, 3) from a setup (cbdiso_2d.py:33-46), or only the
    rows a <= i < b of it for rows=(a, b). Setups with a vectorised
    `primitive_array(t, x, y)` are evaluated on the whole block at once;
    others zone by zone as the reference does.
    """
    ni, nj = mesh.shape
    a, b = rows if rows is not None else (0, ni)
    if hasattr(setup, "primitive_array"):
        i = np.arange(a, b, dtype=np.float64)[:, None]
        j = np.arange(nj, dtype=np.float64)[None, :]
        x = np.broadcast_to(mesh.x0 + (i + 0.5) * mesh.dx, (b - a, nj))
        y = np.broadcast_to(mesh.y0 + (j + 0.5) * mesh.dy, (b - a, nj))
        return np.ascontiguousarray(setup.primitive_array(time, x, y), dtype=np.float64)
    primitive = np.zeros([b - a, nj, 3])
    for i in range(a, b):
        for j in range(nj):
            setup.primitive(time, mesh.cell_coordinates(i, j), primitive[i - a, j])
    return primitive


def _as_diagnostic(d):
    if isinstance(d, dict):
        return Diagnostic(**d)
    if isinstance(d, Diagnostic):
        return d
    return Diagnostic(d.quantity, d.gravity, d.accretion, d.which_mass, d.radial_cut)


def _mass_struct(m, out):
    out.x = m.position_x
    out.y = m.position_y
    out.vx = m.velocity_x
    out.vy = m.velocity_y
    out.mass = m.mass
    out.softening_length = m.softening_length
    out.sink_rate = m.sink_rate
    out.sink_radius = m.sink_radius
    out.sink_model = enum_value(m.sink_model)


def _diag_struct(d: Diagnostic, out):
    out.quantity = _capi.QUANTITY[d.quantity]
    wm = d.which_mass
    out.which_mass = 3 if wm == "both" else (int(wm) if wm in (1, 2) else 1)
    out.gravity = int(bool(d.gravity))
    out.accretion = int(bool(d.accretion))
    if d.radial_cut is not None:
        out.has_cut = 1
        out.r0, out.r1 = float(d.radial_cut[0]), float(d.radial_cut[1])
    else:
        out.has_cut = 0


class Solver(SolverBase):
    """Adapter driving the fused sm_100a kernels of libcbdiso_b200.so."""

    def __init__(self, setup=None, mesh=None, time=0.0, solution=None, num_patches=1, mode="gpu",
                 physics=dict(), options=dict(), index_range=None):
        """
        `index_range` (a, b) makes this solver one patch of the mesh: rows
        a <= i < b, with the patch's own edge coordinates as the reference's
        Patch has them (cbdiso_2d.py:69-80); `solution` is then the whole
        mesh's or the patch's. The multi-GPU solver (distributed.py) runs one
        patch per rank and exchanges the guard rows between stages.
        """
        import torch

        physics = dict(physics)
        physics["diagnostics"] = [_as_diagnostic(v) for v in physics.get("diagnostics", [])]
        self._physics = physics = Physics(**physics)
        self._options = options = Options(**options)

        if not is_planar_cartesian_2d(mesh):
            raise ValueError("solver only supports 2D cartesian mesh")
        if setup.boundary_condition != "outflow":
            raise ValueError("solver only supports outflow boundary condition")
        if enum_value(physics.viscosity_model) not in (0, 1):
            raise ValueError("solver only supports constant-nu viscosity")
        if enum_value(physics.eos_type) not in (1, 2):
            raise ValueError("solver only supports isothermal equation of states")
        if physics.cooling_coefficient != 0.0:
            raise ValueError("solver does not support thermal cooling")
        if not physics.constant_softening:
            raise ValueError("solver only supports constant gravitational softening")
        if options.rk_order not in RK_WEIGHTS:
            raise ValueError(f"rk_order must be 1, 2 or 3, got {options.rk_order}")
        if options.precision not in _capi.PRECISION:
            raise ValueError(f"precision must be one of {sorted(_capi.PRECISION)}, got {options.precision}")
        for d in physics.diagnostics:
            if d.quantity != "time" and d.quantity not in _capi.QUANTITY:
                raise ValueError(f"unknown diagnostic quantity {d.quantity}")
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
            # The buffer's target density is the setup's data at the onset
            # radius on the x axis, as in cbdiso_2d.py:325-334.
            buffer_prim = [0.0] * 3
            buffer_outer_radius = mesh.x1
            buffer_onset_radius = buffer_outer_radius - physics.buffer_onset_width
            setup.primitive(time, [buffer_onset_radius, 0.0], buffer_prim)
            buffer_surface_density = buffer_prim[0]
        else:
            buffer_outer_radius = 0.0
            buffer_surface_density = 0.0

        g = _capi.Grid()
        g.ni, g.nj = ni, nj
        g.xl, g.yl = mesh.vertex_coordinates(a, 0)
        g.xr, g.yr = mesh.vertex_coordinates(b, nj)
        g.plm_theta = options.plm_theta
        g.eos_type = enum_value(physics.eos_type)
        g.precision = _capi.PRECISION[options.precision]
        g.cs2 = physics.sound_speed ** 2
        g.mach2 = physics.mach_number ** 2
        g.nu = physics.viscosity_coefficient
        g.velocity_ceiling = options.velocity_ceiling
        g.density_floor = options.density_floor
        g.buffer_is_enabled = int(bool(physics.buffer_is_enabled))
        g.buffer_surface_density = buffer_surface_density
        g.buffer_driving_rate = physics.buffer_driving_rate
        g.buffer_outer_radius = buffer_outer_radius
        g.buffer_onset_width = physics.buffer_onset_width
        if options.tile:
            g.tile_columns, g.tile_rows = int(options.tile[0]), int(options.tile[1])
            if len(options.tile) > 2:
                g.tile_occupancy = int(options.tile[2])
        self._grid = g

        f64 = dict(dtype=torch.float64, device=self.device)
        nbuf = 3 if options.rk_order == 3 else 2
        self._buf = [torch.empty((ni + 2 * NG, nj + 2 * NG, NQ), **f64) for _ in range(nbuf)]
        _hostio.upload(primitive, self._buf[0][NG:-NG, NG:-NG])
        self._check(self._lib.cbdiso_b200_fill_guards(ctypes.byref(g), self._ptr(self._buf[0]), self._stream()),
                    "fill_guards")
        nscratch = int(self._lib.cbdiso_b200_scratch_bytes(ctypes.byref(g)))
        self._scratch = torch.zeros(nscratch // 8 + 8, **f64)
        # face sound speeds and gravity factors carried from a step's last
        # stage to the next step's first (same bits as recomputing them)
        self._fcache = None
        if options.face_cache:
            self._fcache = torch.empty(int(self._lib.cbdiso_b200_face_cache_bytes(ctypes.byref(g))) // 8, **f64)
            self._fcache[:32].zero_()
        self._result = torch.zeros(1 + 2 * _capi.MAX_DIAG, **f64)
        self._result_host = torch.zeros(1 + 2 * _capi.MAX_DIAG, dtype=torch.float64).pin_memory()

        # stage records: a small ring of pinned host slots, one device block
        self._rec_bytes = int(self._lib.cbdiso_b200_stage_record_bytes())
        nstage = len(RK_WEIGHTS[options.rk_order])
        self._ring = [torch.zeros(nstage * self._rec_bytes, dtype=torch.uint8).pin_memory() for _ in range(4)]
        self._ring_events = [None] * len(self._ring)
        self._ring_next = 0
        self._records = torch.zeros(nstage * self._rec_bytes, dtype=torch.uint8, device=self.device)

        self._device_diags = [d for d in physics.diagnostics if d.quantity != "time"]
        self._fused = options.fuse_reductions and len(self._device_diags) <= _capi.MAX_FUSED
        self._time = float(time)
        self._cached = None  # result block valid for the current state, read lazily
        self._result_valid = False
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

    def _check(self, status, where):
        _capi.check(status, where)

    def _epilogue(self, time, want_ws, diags):
        ep = _capi.Epilogue()
        m1, m2 = self._point_masses(time)
        _mass_struct(m1, ep.mass[0])
        _mass_struct(m2, ep.mass[1])
        ep.want_wavespeed = int(want_ws)
        ep.num_diag = len(diags)
        for k, d in enumerate(diags):
            _diag_struct(d, ep.diag[k])
        return ep

    def _read_result(self):
        import torch

        if self._cached is None:
            n = 1 + 2 * len(self._device_diags)
            self._result_host[:n].copy_(self._result[:n], non_blocking=True)
            torch.cuda.current_stream().synchronize()
            self.d2h_bytes += 8 * n
            self._cached = self._result_host[:n].numpy().copy()
        return self._cached

    def _reduce_now(self, want_ws, diags):
        ep = self._epilogue(self._time, want_ws, diags)
        self._check(self._lib.cbdiso_b200_reduce(ctypes.byref(self._grid), ctypes.byref(ep),
                                                 self._ptr(self._buf[0]), self._ptr(self._scratch),
                                                 self._ptr(self._result), self._stream()), "reduce")
        self._cached = None
        self._result_valid = True

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
        return 0.3

    @property
    def maximum_cfl(self):
        return 0.4

    def maximum_wavespeed(self):
        """Largest |v +- cs| over the grid, with point masses at the current
        time. Raises CbdError (CBD_ERR_NONFINITE) when it is not finite: the
        state holds a NaN or infinity, from which the driver's CFL rule would
        take a NaN time step (the reference returns the value and runs on)."""
        if not self._result_valid:
            self._reduce_now(True, self._device_diags if self._fused else [])
        value = float(self._read_result()[0])
        if not math.isfinite(value):
            raise _capi.CbdError(_capi.NONFINITE, "maximum_wavespeed")
        return value

    def advance(self, dt):
        """One step of the configured RK order. The first stage goes out as
        soon as its point masses (at the step's start, usually known from the
        previous step's end) are set, its record carried by the launch's own
        parameters, so that the device idles as little as possible between
        the caller's wavespeed read and this step; the later stages' orbits
        and records are built on the host while it runs and reach the device
        as one copy ahead of their launches."""
        import torch

        dt = float(dt)
        if not math.isfinite(dt):
            raise _capi.CbdError(_capi.NONFINITE, "advance: time step")
        weights = RK_WEIGHTS[self._options.rk_order]
        time0 = self._time
        lib, g = self._lib, self._grid
        stream = self._stream()

        # stage times follow cbdiso_2d.py:239 exactly
        times = []
        t = time0
        for a in weights:
            times.append(t)
            t = time0 * a + (t + dt) * (1.0 - a)
        time_end = t

        plan = self._stage_plan(len(weights))
        diags = self._device_diags if self._fused else []

        def stage(s):
            st = _capi.Stage()
            m1, m2 = self._point_masses(times[s])
            _mass_struct(m1, st.mass[0])
            _mass_struct(m2, st.mass[1])
            st.a = weights[s]
            st.dt = dt
            st.buffer_central_mass = m1.mass + m2.mass
            return st

        last = len(weights) - 1
        # the first stage, its record as launch parameters; without an
        # epilogue (RK2, RK3) its record's end-of-step masses are never read
        epilogue = self._epilogue(time_end, True, diags) if last == 0 else None
        self._launch_stage(0, plan, weights, epilogue, stream, stage=stage(0))
        rb = self._rec_bytes
        if last > 0:
            # the later stages' records: a slot of the pinned ring whose
            # previous copy has completed, then one copy to the device
            slot = self._ring_next
            self._ring_next = (slot + 1) % len(self._ring)
            if self._ring_events[slot] is not None:
                self._ring_events[slot].synchronize()
            host = self._ring[slot]
            epilogue = self._epilogue(time_end, True, diags)
            for s in range(1, last + 1):
                self._check(lib.cbdiso_b200_stage_record(ctypes.byref(g), ctypes.byref(stage(s)),
                                                         ctypes.byref(epilogue),
                                                         ctypes.c_void_p(host.data_ptr() + s * rb)), "stage_record")
            self._records[rb:].copy_(host[rb:], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record()
            self._ring_events[slot] = ev
            for s in range(1, last + 1):
                self._launch_stage(s, plan, weights, epilogue if s == last else None, stream)
        self.h2d_bytes += len(weights) * rb  # every stage's record: launch parameters or the copy
        self._finish_stages(len(weights), None)
        self._time = time_end
        self._cached = None
        self._result_valid = True

    def _point_masses(self, t):
        masses = self.__dict__.get("_mass_cache")
        if masses is None or masses.physics is not self._physics:
            masses = self._mass_cache = MassCache(self._physics)
        return masses(t)

    # ------------------------------------------------------------------
    # device-resident stepping
    # ------------------------------------------------------------------

    def _device_orbit(self):
        """
        The binary's Kepler orbit as the device stepper needs it, taken from a
        setup with `orbital_elements` and uniform sink / softening parameters
        (the circumbinary setups). Checked against the physics callback.
        """
        setup = self.setup
        need = ("orbital_elements", "softening_length", "sink_model", "sink_rate", "sink_radius")
        if not all(hasattr(setup, a) for a in need):
            raise ValueError("device stepping needs a setup with a Kepler binary (orbital_elements)")
        el = setup.orbital_elements
        o = _capi.Orbit()
        o.semimajor_axis, o.total_mass = float(el.semimajor_axis), float(el.total_mass)
        o.mass_ratio, o.eccentricity = float(el.mass_ratio), float(el.eccentricity)
        o.softening_length, o.sink_rate = float(setup.softening_length), float(setup.sink_rate)
        o.sink_radius = float(setup.sink_radius)
        model = setup.sink_model
        o.sink_model = enum_value(model) if not isinstance(model, str) else (
            dict(inactive=0, acceleration_free=1, torque_free=2, force_free=3)[model.lower()])
        x_off = getattr(setup, "x_bin", None)
        if x_off is not None:
            o.has_x_offset, o.x_offset = 1, float(x_off)
        from .kepler import OrbitalElements

        orb = OrbitalElements(o.semimajor_axis, o.total_mass, o.mass_ratio, o.eccentricity)
        for t in (self._time, self._time + 1.2345):
            got = self._physics.point_masses(t)
            want = orb.orbital_state(t)
            for g_, w_ in zip(got, want):
                wx = w_.position_x + (o.x_offset if o.has_x_offset else 0.0)
                if (g_.mass, g_.position_x, g_.position_y, g_.velocity_x, g_.velocity_y) != (
                        w_.mass, wx, w_.position_y, w_.velocity_x, w_.velocity_y) or \
                        g_.softening_length != o.softening_length or g_.sink_rate != o.sink_rate or \
                        g_.sink_radius != o.sink_radius or enum_value(g_.sink_model) != o.sink_model:
                    raise ValueError("the physics point masses are not the setup's Kepler binary")
        return o

    def run(self, steps, cfl=None, fixed_dt=None, graph=True, steps_per_graph=16, dt_sequence=None,
            history=None, trajectory=None, checkpoints=None):
        """
        Advance `steps` iterations entirely on the device: each step's dt is
        min(dx, dy) / max wavespeed * cfl (driver.py:508-510) from the previous
        step's fused wavespeed (or `fixed_dt`, or the device array
        `dt_sequence` of per-step values), and the point masses come from the
        binary's Kepler orbit solved on the device. With `graph`, a group of
        `steps_per_graph` steps is captured once in a CUDA graph (cached on
        the solver) and replayed. `history` (a device uint8 tensor of
        steps * rk_order stage records) receives every step's stage records.
        `trajectory` (RK2 only; a device float64 tensor of 2 * steps + 1
        padded states) receives the whole run instead of the two solver
        buffers: [0] the current state, then per step n the first stage's
        output [2n + 1] and the step's result [2n + 2]; the last is copied
        back into the solver. `checkpoints` (RK2 only; a sequence of device
        tensors shaped like the padded state, at least steps / steps_per_graph
        of them) receives the state before every group of `steps_per_graph`
        steps: checkpoints[g] holds the state after g * steps_per_graph steps,
        copied on the launching stream with no host synchronisation. Returns
        the time series: one row per step, the `reductions()` row followed by
        dt.
        """
        import torch

        steps = int(steps)
        if steps <= 0:
            return []
        cfl = self.recommended_cfl if cfl is None else float(cfl)
        lib, g = self._lib, self._grid
        orbit = self._device_orbit()
        if not self._result_valid:
            self._reduce_now(True, self._device_diags if self._fused else [])
            if self._step_hook is not None:
                self._step_hook()
        if self._stage_hook is not None or self._step_hook is not None:
            graph = False  # the hooks' collectives stay outside graph capture
        nvals = 2 * len(self._device_diags) if self._fused else 0
        if self._options.rk_order == 1 and steps_per_graph % 2:
            steps_per_graph += 1  # RK1 swaps the two buffers each step: capture whole pairs
        nbytes = int(lib.cbdiso_b200_stepper_bytes())
        if getattr(self, "_stepper_dev", None) is None:
            self._stepper_dev = torch.zeros(nbytes, dtype=torch.uint8, device=self.device)
            self._graphs = {}
        if getattr(self, "_series_dev", None) is None or self._series_dev.shape[0] < steps or \
                self._series_dev.shape[1] != 3 + nvals:
            self._series_dev = torch.zeros((max(steps, SERIES_ROWS), 3 + nvals), dtype=torch.float64, device=self.device)
            self._graphs = {}
        stepper, series = self._stepper_dev, self._series_dev
        host = torch.zeros(nbytes, dtype=torch.uint8).pin_memory()
        self._check(lib.cbdiso_b200_stepper_init(ctypes.byref(g), ctypes.byref(orbit), self._options.rk_order,
                                                 self._time, cfl, float(self.mesh.min_spacing()),
                                                 float(fixed_dt or 0.0), series.shape[0],
                                                 ctypes.c_void_p(host.data_ptr())), "stepper_init")
        if dt_sequence is not None or history is not None:
            if dt_sequence is not None and dt_sequence.numel() < steps:
                raise ValueError("dt_sequence is shorter than steps")
            self._check(lib.cbdiso_b200_stepper_attach(
                ctypes.c_void_p(host.data_ptr()),
                self._ptr(dt_sequence) if dt_sequence is not None else None,
                int(dt_sequence.numel()) if dt_sequence is not None else 0,
                self._ptr(history) if history is not None else None,
                int(history.numel() // (self._rec_bytes * self._options.rk_order)) if history is not None else 0),
                "stepper_attach")
        stepper.copy_(host, non_blocking=True)
        self.h2d_bytes += nbytes
        epilogue = self._epilogue(self._time, True, self._device_diags if self._fused else [])
        weights = RK_WEIGHTS[self._options.rk_order]
        # what trajectory_launches() replays: this run's initial stepper record
        # and epilogue
        self._last_run = dict(record=host, nvals=nvals, epilogue=epilogue)

        def one_step(n=None):
            stream = self._stream()
            self._check(lib.cbdiso_b200_step_prologue(self._ptr(stepper), self._ptr(self._result),
                                                      self._ptr(self._records), self._ptr(series), nvals, 0,
                                                      stream), "step_prologue")
            if n is None:
                self._launch_stages(weights, epilogue, stream)
            else:
                self._launch_stages(weights, epilogue, stream,
                                    (trajectory[2 * n], trajectory[2 * n + 1], trajectory[2 * n + 2]))

        if checkpoints is not None:
            if self._options.rk_order != 2 or trajectory is not None:
                raise ValueError("checkpoints are taken in RK2 runs without a trajectory")
            if len(checkpoints) < -(-steps // steps_per_graph):
                raise ValueError("fewer checkpoints than groups of steps_per_graph steps")
        launched = 0

        def group_start():
            # the state before each group of steps_per_graph steps
            if checkpoints is not None and launched % steps_per_graph == 0:
                checkpoints[launched // steps_per_graph].copy_(self._buf[0])

        remaining = steps
        if trajectory is not None:
            if self._options.rk_order != 2:
                raise ValueError("a trajectory is recorded for RK2 only")
            if trajectory.shape[0] < 2 * steps + 1 or trajectory.shape[1:] != self._buf[0].shape or \
                    trajectory.dtype != self._buf[0].dtype or not trajectory.is_contiguous():
                raise ValueError("trajectory must hold 2 * steps + 1 padded float64 states")
            trajectory[0].copy_(self._buf[0])
            if graph:
                # one graph for the whole run: every step writes its own slots
                key = ("trajectory", steps, trajectory.data_ptr(), nvals)
                cuda_graph = self._graphs.get(key)
                if cuda_graph is None:
                    side = torch.cuda.Stream()
                    side.wait_stream(torch.cuda.current_stream())
                    cuda_graph = torch.cuda.CUDAGraph()
                    with capture(cuda_graph, side):
                        for n in range(steps):
                            one_step(n)
                    torch.cuda.current_stream().wait_stream(side)
                    self._graphs[key] = cuda_graph
                cuda_graph.replay()
            else:
                for n in range(steps):
                    one_step(n)
            self._buf[0].copy_(trajectory[2 * steps])
            remaining = 0
        if graph and remaining >= steps_per_graph:
            # the graph bakes in buffer addresses: RK1 alternates two assignments
            key = (steps_per_graph, nvals, self._buf[0].data_ptr())
            cuda_graph = self._graphs.get(key)
            if cuda_graph is None:
                side = torch.cuda.Stream()
                side.wait_stream(torch.cuda.current_stream())
                cuda_graph = torch.cuda.CUDAGraph()
                with capture(cuda_graph, side):
                    for _ in range(steps_per_graph):
                        one_step()
                torch.cuda.current_stream().wait_stream(side)
                self._graphs[key] = cuda_graph
            while remaining >= steps_per_graph:
                group_start()
                cuda_graph.replay()
                remaining -= steps_per_graph
                launched += steps_per_graph
        for _ in range(remaining):
            group_start()
            one_step()
            launched += 1
        self._check(lib.cbdiso_b200_step_prologue(self._ptr(stepper), self._ptr(self._result),
                                                  self._ptr(self._records), self._ptr(series), nvals, 1,
                                                  self._stream()), "step_prologue")
        state = stepper.cpu()
        time, status = self._stepper_fields(state)
        if status != 0:
            raise _capi.CbdError(status, "device stepping")
        self._time = time
        self._cached = None
        self._result_valid = True
        rows = series[:steps].cpu().numpy()
        self.d2h_bytes += rows.nbytes + state.numel()
        self.last_series = rows  # raw device rows (time, dt, wavespeed, sums)
        return self._series_rows(rows)

    def trajectory_launches(self, steps, trajectory, record):
        """
        The launches of a device-stepped RK2 run of `steps` steps that writes
        the run into `trajectory` (as run(trajectory=...)), starting from the
        state in trajectory[0] and the stepper record in `record` (a device
        copy of the record the last run started from; see
        last_stepper_record), followed by the final series prologue. Nothing
        synchronises with the host, so that the launches can be captured into
        a larger CUDA graph; the time series is left in the device series
        buffer (read it with series_after_launches). Requires a previous
        run(trajectory=...) of the same length on this solver, which set up
        the buffers.
        """
        lib = self._lib
        last = self._last_run
        nvals, epilogue = last["nvals"], last["epilogue"]
        stepper, series = self._stepper_dev, self._series_dev
        weights = RK_WEIGHTS[self._options.rk_order]
        stepper.copy_(record)
        for n in range(steps):
            stream = self._stream()
            self._check(lib.cbdiso_b200_step_prologue(self._ptr(stepper), self._ptr(self._result),
                                                      self._ptr(self._records), self._ptr(series), nvals, 0,
                                                      stream), "step_prologue")
            self._launch_stages(weights, epilogue, stream,
                                (trajectory[2 * n], trajectory[2 * n + 1], trajectory[2 * n + 2]))
        self._check(lib.cbdiso_b200_step_prologue(self._ptr(stepper), self._ptr(self._result),
                                                  self._ptr(self._records), self._ptr(series), nvals, 1,
                                                  self._stream()), "step_prologue")

    def last_stepper_record(self):
        """A device copy of the stepper record the last run() started from."""
        return self._last_run["record"].to(self.device)

    def series_after_launches(self, steps):
        """The time series rows of trajectory_launches() (as run() returns
        them), read from the device; also checks the stepper's status."""
        state = self._stepper_dev.cpu()
        _, status = self._stepper_fields(state)
        if status != 0:
            raise _capi.CbdError(status, "device stepping")
        return self._series_rows(self._series_dev[:steps].cpu().numpy())

    def _stepper_fields(self, state):
        raw = state.numpy().tobytes()
        time = np.frombuffer(raw[0:8], dtype=np.float64)[0]
        # status follows the orbit record; its offset is fixed by the struct layout
        status = int(np.frombuffer(raw[self._status_offset():self._status_offset() + 4], dtype=np.int32)[0])
        return float(time), status

    @staticmethod
    def _status_offset():
        # StepperDev: 6 doubles, weights[3], cbd_orbit_t, then num_stages, step, status
        return 8 * 6 + 8 * 3 + ctypes.sizeof(_capi.Orbit) + 8

    def _series_rows(self, rows):
        """
        Device time-series rows -> reductions()-shaped rows plus dt. Without
        fused diagnostics (more than four, or fuse_reductions off) the
        per-step sums are not recorded and appear as None.
        """
        out = []
        da = self.mesh.dx * self.mesh.dy
        have = rows.shape[1] > 3
        for row in rows:
            t, dt = float(row[0]), float(row[1])
            vals = []
            k = 0
            for d in self._physics.diagnostics:
                if d.quantity == "time":
                    vals.append(t / self.setup.reference_time_scale)
                    continue
                if not have:
                    vals.append(None)
                    continue
                re, im = row[3 + 2 * k], row[4 + 2 * k]
                k += 1
                vals.append(complex(re, im) * da if d.quantity in COMPLEX_QUANTITIES else float(re) * da)
            out.append(vals + [dt])
        return out

    def _stage_plan(self, nstages, rk2_buffers=None):
        """(read, u_n source, write) buffers of each RK stage: RK1 A -> B
        (then swapped), RK2 A -> B, B (+A) -> A, RK3 A -> B, B (+A) -> C,
        C (+A) -> A; or, for RK2, the given (u_n, stage 1 output, result)."""
        A = self._buf[0]
        B = self._buf[1]
        if rk2_buffers is not None:
            un, mid, out = rk2_buffers
            return [(un, None, mid), (mid, un, out)]
        if nstages == 1:
            return [(A, None, B)]
        if nstages == 2:
            return [(A, None, B), (B, A, A)]
        C = self._buf[2]
        return [(A, None, B), (B, A, C), (C, A, A)]

    def _launch_stage(self, s, plan, weights, epilogue, stream, stage=None):
        """Stage s of one step, reading its record in self._records, or, when
        `stage` (a host cbd_stage_t) is given, taking the record from it as a
        launch parameter; the last stage carries the epilogue."""
        rd, pn, wr = plan[s]
        if stage is None:
            stage = _capi.Stage()
            stage.a = weights[s]
            rec = ctypes.c_void_p(self._records.data_ptr() + s * self._rec_bytes)
        else:
            rec = None
        common = (ctypes.byref(self._grid), ctypes.byref(stage), rec, self._ptr(rd),
                  self._ptr(pn) if pn is not None else None, self._ptr(wr),
                  ctypes.byref(epilogue) if epilogue is not None else None, self._ptr(self._scratch),
                  self._ptr(self._result))
        role = self._cache_role(s, len(weights))
        if role:
            status = self._lib.cbdiso_b200_advance_stage_cached(*common, self._ptr(self._fcache), role, stream)
        else:
            status = self._lib.cbdiso_b200_advance_stage(*common, stream)
        self._check(status, "advance_stage")
        if self._stage_hook is not None:
            self._stage_hook(s, wr)

    def _cache_role(self, s, nstages):
        """Face-cache role of stage s of a step (0 none, 1 writer, 2 reader):
        the stage at t0 + dt (RK2's and RK3's second) computes the values in
        its stencil and stores them, the next step's first stage reads them
        (behind a fill pass that recomputes them only when the cached masses
        are not its own); RK1 has no stage at t0 + dt. On one grid this
        costs less than a separate fill pass every step (measured)."""
        if self._fcache is None or nstages == 1:
            return 0
        if s == 0:
            return 2
        return 1 if s == 1 else 0

    def _finish_stages(self, nstages, rk2_buffers):
        if nstages == 1 and rk2_buffers is None:
            self._buf[0], self._buf[1] = self._buf[1], self._buf[0]
        if self._step_hook is not None:
            self._step_hook()

    def _launch_stages(self, weights, epilogue, stream, rk2_buffers=None):
        """The RK stages of one step, reading the stage records in
        self._records; the last stage carries the epilogue."""
        plan = self._stage_plan(len(weights), rk2_buffers)
        for s in range(len(weights)):
            self._launch_stage(s, plan, weights, epilogue if s == len(weights) - 1 else None, stream)
        self._finish_stages(len(weights), rk2_buffers)

    def reset(self, solution, time=0.0):
        """Start again from `solution` (host (ni, nj, 3)) at `time`, keeping
        the device buffers (and the CUDA graphs that refer to them)."""
        import torch

        primitive = np.asarray(solution, dtype=np.float64)
        ni, nj = self._grid.ni, self._grid.nj
        if primitive.shape != (ni, nj, NQ):
            raise ValueError(f"solution has shape {primitive.shape}, expected {(ni, nj, NQ)}")
        _hostio.upload(primitive, self._buf[0][NG:-NG, NG:-NG])
        self._check(self._lib.cbdiso_b200_fill_guards(ctypes.byref(self._grid), self._ptr(self._buf[0]),
                                                      self._stream()), "fill_guards")
        self._time = float(time)
        self._cached = None
        self._result_valid = False

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
        if self._result_valid:
            return False
        self._reduce_now(True, self._device_diags if self._fused else [])
        return True

    def wavespeed_changed(self):
        """The wavespeed buffer was rewritten on the device (all-reduced)."""
        self._cached = None

    def reduction_sums(self):
        """The diagnostic sums over this solver's zones before the dx dy
        factor (float or complex per non-time diagnostic)."""
        if not self._device_diags:
            return []
        if not (self._fused and self._result_valid):
            self._reduce_now(True, self._device_diags)
        res = self._read_result()
        out = []
        for k, d in enumerate(self._device_diags):
            re, im = res[1 + 2 * k], res[2 + 2 * k]
            out.append(complex(re, im) if d.quantity in COMPLEX_QUANTITIES else float(re))
        return out

    def reductions(self):
        """
        Time series row in the order of physics.diagnostics: time in units of
        the setup's reference time scale, then each sum times dx dy
        (cbdiso_2d.py:370-503). Real quantities are floats, sigma_m1 and
        eccentricity_vector complex.
        """
        diagnostics = self._physics.diagnostics
        if self._device_diags:
            if not (self._fused and self._result_valid):
                self._reduce_now(True, self._device_diags)
            res = self._read_result()
        da = self.mesh.dx * self.mesh.dy
        out = []
        k = 0
        for d in diagnostics:
            if d.quantity == "time":
                out.append(self._time / self.setup.reference_time_scale)
                continue
            re, im = res[1 + 2 * k], res[2 + 2 * k]
            k += 1
            if d.quantity in COMPLEX_QUANTITIES:
                out.append(complex(re, im) * da)
            else:
                out.append(float(re) * da)
        return out
