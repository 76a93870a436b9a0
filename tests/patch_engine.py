"""
A CPU engine for DistributedSolver, restated on the oracle's kernels: one
patch of the mesh per rank, with the same hooks as cbdiso_2d.Solver (stage
and step hooks, wavespeed buffer, reduction sums). Test infrastructure only:
it lets the multi-rank host logic (patch split, guard-row exchange, the
wavespeed all-reduce, patch-ordered sums) run as gloo ranks without a GPU.
"""

import numpy as np
import torch

from oracle import host as oh
from sailfish_b200.cbdiso_2d import NG

RK = {1: (0.0,), 2: (0.0, 0.5), 3: (0.0, 0.75, 1.0 / 3.0)}


def zero_gradient(p):
    for i in range(NG):
        p[i] = p[NG]
        p[-1 - i] = p[-NG - 1]
    for j in range(NG):
        p[:, j] = p[:, NG]
        p[:, -1 - j] = p[:, -NG - 1]


class OraclePatch:
    def __init__(self, setup, mesh, time, solution, physics, options, index_range):
        a, b = index_range
        ni, nj = mesh.shape
        self.setup, self.mesh = setup, mesh
        self.rk = options.get("rk_order", 2)
        self.options = dict(options)
        from sailfish_b200.cbdiso_2d import _as_diagnostic

        self.physics = dict(physics, diagnostics=[_as_diagnostic(d) for d in physics.get("diagnostics", [])])
        self.diagnostics = [d for d in physics.get("diagnostics", []) if d["quantity"] != "time"]
        onset = physics["buffer_onset_width"]
        prim = [0.0] * 3
        setup.primitive(time, [mesh.x1 - onset, 0.0], prim)
        xl, yl = mesh.vertex_coordinates(a, 0)
        xr, yr = mesh.vertex_coordinates(b, nj)
        cfg = oh.Config(x0=xl, x1=xr, y0=yl, y1=yr, ni=b - a, nj=nj, eos_type=2, mach_number=setup.mach_number,
                        nu=setup.nu, buffer_is_enabled=setup.buffer_is_enabled,
                        buffer_driving_rate=physics["buffer_driving_rate"], buffer_onset_width=onset,
                        buffer_surface_density=prim[0],
                        masses=oh.binary_masses(1.0, 1.0, setup.mass_ratio, setup.eccentricity,
                                                setup.softening_length, setup.sink_model, setup.sink_rate,
                                                setup.sink_radius),
                        rk_order=self.rk, plm_theta=options.get("plm_theta", 1.8))
        sol = np.asarray(solution)
        self.o = oh.OracleSolver(cfg, sol[a:b] if sol.shape[0] == ni else sol, time)
        # the reference's patch edges (vertex coordinates) and the whole mesh's buffer radius
        self.o.xl, self.o.xr, self.o.yl, self.o.yr = xl, xr, yl, yr
        self.o.buffer_outer_radius = mesh.x1 if setup.buffer_is_enabled else 0.0
        zero_gradient(self.o.p1)
        self._stage_hook = None
        self._step_hook = None
        self._ws = torch.zeros(1, dtype=torch.float64)
        self._valid = False

    @property
    def time(self):
        return self.o.time

    @property
    def solution(self):
        return self.o.solution

    recommended_cfl = 0.3
    maximum_cfl = 0.4

    def state_buffer(self):
        return torch.from_numpy(self.o.p1)

    def advance(self, dt):
        o, c = self.o, self.o.cfg
        o.time0 = o.time
        o.k.primitive_to_conserved(c.ni, c.nj, o.p1, o.u0)
        for s, a in enumerate(RK[self.rk]):
            m1, m2 = c.point_masses(o.time)
            buf = (c.buffer_surface_density, m1.mass + m2.mass, c.buffer_driving_rate, o.buffer_outer_radius,
                   c.buffer_onset_width, int(c.buffer_is_enabled))
            o.k.advance_rk(c.ni, c.nj, o.xl, o.xr, o.yl, o.yr, o.u0, o.p1, o.p2, buf, m1, m2, c.sound_speed ** 2,
                           c.mach_number ** 2, c.eos_type, c.nu, a, dt, c.velocity_ceiling, c.density_floor)
            o.time = o.time0 * a + (o.time + dt) * (1.0 - a)
            o.p1, o.p2 = o.p2, o.p1
            zero_gradient(o.p1)
            if self._stage_hook is not None:
                self._stage_hook(s, torch.from_numpy(o.p1))
        self._valid = False
        self.ensure_wavespeed()
        if self._step_hook is not None:
            self._step_hook()

    def wavespeed_buffer(self):
        return self._ws

    def ensure_wavespeed(self):
        if self._valid:
            return False
        self._ws[0] = self.o.maximum_wavespeed()
        self._valid = True
        return True

    def wavespeed_changed(self):
        pass

    def maximum_wavespeed(self):
        self.ensure_wavespeed()
        return float(self._ws[0])

    def reduction_sums(self):
        da = self.o.cfg.dx * self.o.cfg.dy
        return [v / da for v in self.o.reductions(self.diagnostics)]


class SerialPatches:
    """The same patches advanced in one process, the guard rows copied
    between them directly: the reference's multi-patch scheme."""

    def __init__(self, setup, mesh, solution, physics, options, parts):
        from sailfish_b200.distributed import subdivide

        self.p = [OraclePatch(setup, mesh, 0.0, solution, physics, options, r)
                  for r in subdivide(mesh.shape[0], parts)]
        self._copy()

    def _copy(self):
        for lo, hi in zip(self.p[:-1], self.p[1:]):
            lo.o.p1[-NG:] = hi.o.p1[NG:2 * NG]
            hi.o.p1[:NG] = lo.o.p1[-2 * NG:-NG]

    def advance(self, dt):
        # stage by stage across the patches, copying guard rows in between
        gens = [self._stages(p, dt) for p in self.p]
        for _ in RK[self.p[0].rk]:
            for g in gens:
                next(g)
            self._copy()

    @staticmethod
    def _stages(p, dt):
        o, c = p.o, p.o.cfg
        o.time0 = o.time
        o.k.primitive_to_conserved(c.ni, c.nj, o.p1, o.u0)
        for a in RK[p.rk]:
            m1, m2 = c.point_masses(o.time)
            buf = (c.buffer_surface_density, m1.mass + m2.mass, c.buffer_driving_rate, o.buffer_outer_radius,
                   c.buffer_onset_width, int(c.buffer_is_enabled))
            o.k.advance_rk(c.ni, c.nj, o.xl, o.xr, o.yl, o.yr, o.u0, o.p1, o.p2, buf, m1, m2, c.sound_speed ** 2,
                           c.mach_number ** 2, c.eos_type, c.nu, a, dt, c.velocity_ceiling, c.density_floor)
            o.time = o.time0 * a + (o.time + dt) * (1.0 - a)
            o.p1, o.p2 = o.p2, o.p1
            zero_gradient(o.p1)
            yield

    def maximum_wavespeed(self):
        return max(p.o.maximum_wavespeed() for p in self.p)

    @property
    def solution(self):
        return np.concatenate([p.o.solution for p in self.p], axis=0)


class GamOraclePatch:
    """The gamma-law solver's patch (cbdgam_2d.py:46-223) on the gamma-law
    oracle's kernels, with the same hooks as cbdgam_2d.Solver."""

    def __init__(self, setup, mesh, time, solution, physics, options, index_range):
        from oracle import host_gam as og
        from sailfish_b200.cbdiso_2d import _as_diagnostic

        a, b = index_range
        ni, nj = mesh.shape
        self.setup, self.mesh = setup, mesh
        self.options = dict(options)
        self.physics = dict(physics, diagnostics=[_as_diagnostic(d) for d in physics.get("diagnostics", [])])
        self.diagnostics = [d for d in physics.get("diagnostics", []) if d["quantity"] != "time"]
        onset = physics["buffer_onset_width"]
        prim = [0.0] * 4
        setup.primitive(time, [mesh.x1 - onset, 0.0], prim)
        on = physics["buffer_is_enabled"]
        xl, yl = mesh.vertex_coordinates(a, 0)
        xr, yr = mesh.vertex_coordinates(b, nj)
        cfg = og.GamConfig(xl, xr, yl, yr, b - a, nj, gamma_law_index=physics["gamma_law_index"],
                           alpha=physics["alpha"], cooling_coefficient=physics["cooling_coefficient"],
                           constant_softening=physics["constant_softening"], buffer_is_enabled=on,
                           buffer_driving_rate=physics["buffer_driving_rate"], buffer_onset_width=onset,
                           buffer_surface_density=prim[0] if on else 0.0,
                           buffer_surface_pressure=prim[3] if on else 0.0,
                           masses=oh.binary_masses(1.0, 1.0, setup.mass_ratio, setup.eccentricity,
                                                   setup.softening_length, setup.sink_model, setup.sink_rate,
                                                   setup.sink_radius),
                           plm_theta=options.get("plm_theta", 1.5))
        sol = np.asarray(solution)
        self.o = og.GamOracleSolver(cfg, sol[a:b] if sol.shape[0] == ni else sol, time)
        self.o.xl, self.o.xr, self.o.yl, self.o.yr = xl, xr, yl, yr
        self.o.buffer_outer_radius = mesh.x1 if on else 0.0
        zero_gradient(self.o.p1)
        self._stage_hook = None
        self._step_hook = None
        self._ws = torch.zeros(1, dtype=torch.float64)
        self._valid = False

    time = OraclePatch.time
    solution = OraclePatch.solution
    recommended_cfl = 0.1
    maximum_cfl = 0.4
    state_buffer = OraclePatch.state_buffer
    wavespeed_buffer = OraclePatch.wavespeed_buffer
    ensure_wavespeed = OraclePatch.ensure_wavespeed
    wavespeed_changed = OraclePatch.wavespeed_changed
    maximum_wavespeed = OraclePatch.maximum_wavespeed
    reduction_sums = OraclePatch.reduction_sums

    def advance(self, dt):
        o, c = self.o, self.o.cfg
        o.time0 = o.time
        o.k.primitive_to_conserved(c.ni, c.nj, o.p1, o.u0, c.gamma_law_index)
        for s, a in enumerate((0.0, 0.5)):
            m1, m2 = c.point_masses(o.time)
            buf = (c.buffer_surface_density, c.buffer_surface_pressure, m1.mass + m2.mass, c.buffer_driving_rate,
                   o.buffer_outer_radius, c.buffer_onset_width, int(c.buffer_is_enabled))
            o.k.advance_rk(c, o.xl, o.xr, o.yl, o.yr, o.u0, o.p1, o.p2, buf, m1, m2, a, dt)
            o.time = o.time0 * a + (o.time + dt) * (1.0 - a)
            o.p1, o.p2 = o.p2, o.p1
            zero_gradient(o.p1)
            if self._stage_hook is not None:
                self._stage_hook(s, torch.from_numpy(o.p1))
        self._valid = False
        self.ensure_wavespeed()
        if self._step_hook is not None:
            self._step_hook()
