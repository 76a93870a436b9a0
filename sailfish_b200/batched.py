"""
Many circumbinary disks advanced together on one GPU.

Each disk is a full cbdiso_2d problem with its own mesh size, binary orbit
(mass ratio, eccentricity), Mach number, viscosity and time step. Per RK stage
all disks are advanced by ONE persistent kernel launch whose CTAs pull tiles
(disk, strip, segment) from a device work queue, largest disks first; the
per-disk CFL time step, stage times and Kepler orbit are computed on the
device; the epilogue's per-tile partials are reduced per disk; and groups of
steps are replayed from a CUDA graph. The tile shape of each disk comes from
the autotuner (sailfish_b200.autotune) keyed by grid size.

Each disk's state is bit-identical to running it alone through
cbdiso_2d.Solver.run with the same tile shape: the same stencil code runs on
the same data, and the per-disk reductions sum the same tile partials in the
same order.
"""

from __future__ import annotations

import ctypes
import math
from typing import List, NamedTuple, Optional, Sequence

import numpy as np

from . import _capi, _hostio
from ._graphs import capture
from .cbdiso_2d import COMPLEX_QUANTITIES, NG, NQ, RK_WEIGHTS, Options, Solver, _diag_struct
from .physics import Diagnostic, Physics, enum_value

RESULT_STRIDE = 1 + 2 * _capi.MAX_FUSED


class Disk(NamedTuple):
    """One member of a batch: a setup, its mesh, optionally its initial primitive state."""

    setup: object
    mesh: object
    solution: Optional[np.ndarray] = None


def default_tile(ni, nj):
    """Tile shape (strip_width, rows) used when no tuned shape is known."""
    width = 128 if nj > 96 else 64
    rows = 32 if ni >= 512 else 16
    return width, rows


class BatchedSolver:
    """
    Advance a list of `Disk`s together. `diagnostics` (a list of dicts or
    Diagnostic, at most four besides "time") are reduced for every disk every
    step. `tiles` maps (ni, nj) to (strip_width, rows); missing sizes use
    `default_tile` unless `autotune` is set, in which case they are measured
    once and cached.
    """

    def __init__(self, disks: Sequence[Disk], rk_order=2, plm_theta=1.5, precision="exact", diagnostics=None,
                 tiles=None, autotune=False, options=None):
        import torch

        if rk_order not in (2, 3):
            raise ValueError("batched stepping supports rk_order 2 and 3")
        if precision not in _capi.PRECISION:
            raise ValueError(f"precision must be one of {sorted(_capi.PRECISION)}")
        if not torch.cuda.is_available():
            raise RuntimeError("sailfish_b200 needs a CUDA device (there is no CPU fallback)")
        self._lib = lib = _capi.lib()
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.rk_order = rk_order
        self.precision = precision
        self.diagnostics = [Diagnostic(**d) if isinstance(d, dict) else d for d in (diagnostics or [])]
        self._device_diags = [d for d in self.diagnostics if d.quantity != "time"]
        if len(self._device_diags) > _capi.MAX_FUSED:
            raise ValueError(f"at most {_capi.MAX_FUSED} diagnostics besides time")
        opts = dict(options or {})
        # the batch keeps one face-cache arena for all disks (option
        # face_cache, default on); the per-disk solvers need none
        face_cache = bool(opts.pop("face_cache", True))
        opts.update(rk_order=rk_order, plm_theta=plm_theta, precision=precision, face_cache=False)

        # One single-disk Solver per disk builds the grid record, the initial
        # state with its guard zones, and validates the physics exactly as the
        # drop-in does; its device buffers are dropped after the copy.
        # (the same Disk object listed several times shares one constructed
        # Solver: its state is copied into each slot)
        self.disks = list(disks)
        self.solvers: List[Solver] = []
        built = {}
        for d in self.disks:
            s = built.get(id(d))
            if s is None:
                physics = d.setup.physics
                physics["diagnostics"] = list(self.diagnostics)
                s = Solver(setup=d.setup, mesh=d.mesh, solution=d.solution, physics=physics, options=opts)
                s._device_orbit()  # every disk must be a Kepler binary
                built[id(d)] = s
            self.solvers.append(s)
        n = len(self.solvers)
        sizes = [s.mesh.shape for s in self.solvers]
        self.order = sorted(range(n), key=lambda i: -sizes[i][0] * sizes[i][1])

        # batch buffers and disk records (in work order)
        if autotune:
            from .autotune import tuned_tiles

            tiles = dict(tiles or {})
            tiles.update(tuned_tiles(sorted(set(sizes)), precision))
        tiles = dict(tiles or {})
        self.tiles = {}
        rec_bytes = int(lib.cbdiso_b200_batch_disk_bytes())
        records = bytearray(rec_bytes * n)
        offset = 0
        unit = 0
        cache_offset = 0
        cache_offsets = []
        self.offsets = [0] * n
        # the last stage's epilogue form: 2 (the kernel compiled for source-rate
        # diagnostics) when every disk's diagnostics allow it
        self._epilogue_form = 2
        for slot, i in enumerate(self.order):
            s = self.solvers[i]
            ni, nj = s.mesh.shape
            width, rows = tiles.get((ni, nj), default_tile(ni, nj))
            self.tiles[(ni, nj)] = (width, rows)
            ep = s._epilogue(s.time, True, self._device_diags)
            if lib.cbdiso_b200_epilogue_rates_only(ctypes.byref(ep)) != 1:
                self._epilogue_form = 1
            units = ctypes.c_int(0)
            buf = (ctypes.c_char * rec_bytes)()
            _capi.check(lib.cbdiso_b200_batch_disk_record(ctypes.byref(s._grid), ctypes.byref(ep), width, rows,
                                                          offset, unit, ctypes.byref(units), buf),
                        "batch_disk_record")
            if face_cache:
                _capi.check(lib.cbdiso_b200_batch_disk_set_face_cache(buf, cache_offset), "batch_disk_set_face_cache")
                cache_offsets.append(cache_offset)
                cache_offset += int(lib.cbdiso_b200_face_cache_bytes(ctypes.byref(s._grid))) // 8
            records[slot * rec_bytes:(slot + 1) * rec_bytes] = bytes(buf)
            self.offsets[i] = offset
            offset += (ni + 2 * NG) * (nj + 2 * NG) * NQ
            unit += units.value
        self.total_units = unit
        self.total_zones = sum(a * b for a, b in sizes)
        f64 = dict(dtype=torch.float64, device=self.device)
        nbuf = 3 if rk_order == 3 else 2
        self._buf = [torch.empty(offset, **f64) for _ in range(nbuf)]
        # per-disk face caches (carried from the stage at t0 + dt to the next
        # step's first stage), each with its key header zeroed
        self._fcache = None
        if face_cache:
            self._fcache = torch.empty(cache_offset, **f64)
            for c in cache_offsets:
                self._fcache[c:c + 32].zero_()
        for i, s in enumerate(self.solvers):
            self._buf[0][self.offsets[i]:self.offsets[i] + s._buf[0].numel()] = s._buf[0].reshape(-1)
        self._disks_dev = torch.frombuffer(records, dtype=torch.uint8).to(self.device)
        self._stage_bytes = int(lib.cbdiso_b200_stage_record_bytes())
        self._records = torch.zeros(n * rk_order * self._stage_bytes, dtype=torch.uint8, device=self.device)
        self._results = torch.zeros(n * RESULT_STRIDE, **f64)
        self._partials = torch.zeros(self.total_units * RESULT_STRIDE, **f64)
        self._counters = torch.zeros(2, dtype=torch.int32, device=self.device)
        self._stepper_bytes = int(lib.cbdiso_b200_stepper_bytes())
        self._steppers = torch.zeros(n * self._stepper_bytes, dtype=torch.uint8, device=self.device)
        self._series = None
        self._graphs = {}
        self.times = [s.time for s in self.solvers]
        # initial wavespeeds (and sums) per disk, from the standalone reduction
        done = {}
        for slot, i in enumerate(self.order):
            s = self.solvers[i]
            if id(s) not in done:
                s._reduce_now(True, self._device_diags)
                done[id(s)] = s._result[:RESULT_STRIDE].clone()
            self._results[slot * RESULT_STRIDE:(slot + 1) * RESULT_STRIDE].copy_(done[id(s)])
        for s in self.solvers:  # free the single-disk buffers
            s._buf = None
            s._scratch = None

    @staticmethod
    def _ptr(t, offset_bytes=0):
        return ctypes.c_void_p(t.data_ptr() + offset_bytes)

    @staticmethod
    def _stream():
        import torch

        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def _one_step(self, nvals):
        lib = self._lib
        n = len(self.solvers)
        stream = self._stream()
        prec = _capi.PRECISION[self.precision]
        _capi.check(lib.cbdiso_b200_batched_prologue(self._ptr(self._steppers), n, self._ptr(self._results),
                                                     RESULT_STRIDE, self._ptr(self._records),
                                                     self._ptr(self._series), nvals, 0, stream), "batched_prologue")
        A, B = self._buf[0], self._buf[1]
        if self.rk_order == 2:
            plan = [(A, None, B), (B, A, A)]
        else:
            C = self._buf[2]
            plan = [(A, None, B), (B, A, C), (C, A, A)]
        for stage, (rd, pn, wr) in enumerate(plan):
            last = stage == len(plan) - 1
            common = (self._ptr(self._disks_dev), n, self.total_units, self._ptr(rd),
                      self._ptr(pn) if pn is not None else None, self._ptr(wr), self._ptr(self._records),
                      self.rk_order, stage, self._epilogue_form if last else 0, self._ptr(self._partials),
                      self._ptr(self._counters), prec)
            # face-cache role: the stage at t0 + dt writes the cache, the next step's first stage reads
            role = 0 if self._fcache is None else (2 if stage == 0 else (1 if stage == 1 else 0))
            if role:
                status = lib.cbdiso_b200_batched_stage_cached(*common, self._ptr(self._fcache), role, stream)
            else:
                status = lib.cbdiso_b200_batched_stage(*common, stream)
            _capi.check(status, "batched_stage")
        _capi.check(lib.cbdiso_b200_batched_finalize(self._ptr(self._disks_dev), n, self._ptr(self._partials),
                                                     self._ptr(self._results), RESULT_STRIDE, stream),
                    "batched_finalize")

    def run(self, steps, cfl=0.3, graph=True, steps_per_graph=8):
        """
        Advance every disk by `steps` iterations, each with its own CFL time
        step. Returns per disk (in the order given) its time series: rows of
        the diagnostics (time first if requested) followed by dt.
        """
        import torch

        lib = self._lib
        n = len(self.solvers)
        steps = int(steps)
        nvals = 2 * len(self._device_diags)
        if self._series is None or self._series.shape[1] < steps:
            self._series = torch.zeros((n, max(steps, 64), 3 + nvals), dtype=torch.float64, device=self.device)
            self._graphs = {}
        cap = self._series.shape[1]
        host = bytearray(n * self._stepper_bytes)
        for slot, i in enumerate(self.order):
            s = self.solvers[i]
            buf = (ctypes.c_char * self._stepper_bytes)()
            _capi.check(lib.cbdiso_b200_stepper_init(ctypes.byref(s._grid), ctypes.byref(s._device_orbit()),
                                                     self.rk_order, self.times[i], float(cfl),
                                                     float(s.mesh.min_spacing()), 0.0, cap, buf), "stepper_init")
            host[slot * self._stepper_bytes:(slot + 1) * self._stepper_bytes] = bytes(buf)
        self._steppers.copy_(torch.frombuffer(host, dtype=torch.uint8))
        remaining = steps
        if graph and steps >= steps_per_graph:
            key = (steps_per_graph, nvals)
            g = self._graphs.get(key)
            if g is None:
                side = torch.cuda.Stream()
                side.wait_stream(torch.cuda.current_stream())
                g = torch.cuda.CUDAGraph()
                with capture(g, side):
                    for _ in range(steps_per_graph):
                        self._one_step(nvals)
                torch.cuda.current_stream().wait_stream(side)
                self._graphs[key] = g
            while remaining >= steps_per_graph:
                g.replay()
                remaining -= steps_per_graph
        for _ in range(remaining):
            self._one_step(nvals)
        _capi.check(lib.cbdiso_b200_batched_prologue(self._ptr(self._steppers), n, self._ptr(self._results),
                                                     RESULT_STRIDE, self._ptr(self._records),
                                                     self._ptr(self._series), nvals, 1, self._stream()),
                    "batched_prologue")
        state = self._steppers.cpu().numpy().tobytes()
        rows = self._series[:, :steps].cpu().numpy()
        out = [None] * n
        status_off = Solver._status_offset()
        for slot, i in enumerate(self.order):
            rec = state[slot * self._stepper_bytes:(slot + 1) * self._stepper_bytes]
            self.times[i] = float(np.frombuffer(rec[0:8], dtype=np.float64)[0])
            status = int(np.frombuffer(rec[status_off:status_off + 4], dtype=np.int32)[0])
            if status != 0:
                raise _capi.CbdError(status, f"batched stepping, disk {i}")
            out[i] = self._rows(i, rows[slot])
        return out

    def _rows(self, i, rows):
        s = self.solvers[i]
        da = s.mesh.dx * s.mesh.dy
        out = []
        for row in rows:
            vals, k = [], 0
            for d in self.diagnostics:
                if d.quantity == "time":
                    vals.append(float(row[0]) / s.setup.reference_time_scale)
                    continue
                re, im = row[3 + 2 * k], row[4 + 2 * k]
                k += 1
                vals.append(complex(re, im) * da if d.quantity in COMPLEX_QUANTITIES else float(re) * da)
            out.append(vals + [float(row[1])])
        return out

    def solution(self, i):
        """Primitive state (ni, nj, 3) of disk i, on the host."""
        ni, nj = self.solvers[i].mesh.shape
        a = self._buf[0][self.offsets[i]:self.offsets[i] + (ni + 2 * NG) * (nj + 2 * NG) * NQ]
        return _hostio.download(a.reshape(ni + 2 * NG, nj + 2 * NG, NQ)[NG:-NG, NG:-NG])


def config2_disks(num=64, seed=2024, sizes=(128, 192, 256, 384, 512, 768, 1024)):
    """
    The batched workload: `num` circumbinary disks on [-8, 8]^2 with sizes
    drawn uniformly from `sizes`, mass ratio q ~ U[0.1, 1], eccentricity
    e ~ U[0, 0.5], Mach ~ U[10, 40], nu ~ logU[1e-4, 1e-2], otherwise the
    config-0 physics (sink rate 10, sink radius 0.05, softening 0.05,
    torque-free sinks, buffer), each with its setup's disk plus seeded 1e-3
    noise on Sigma.
    """
    from .cbdiso_2d import initial_condition
    from .setups import CircumbinaryDisk

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(num):
        n = int(rng.choice(sizes))
        q = float(rng.uniform(0.1, 1.0))
        e = float(rng.uniform(0.0, 0.5))
        mach = float(rng.uniform(10.0, 40.0))
        nu = float(10.0 ** rng.uniform(-4.0, -2.0))
        setup = CircumbinaryDisk(domain_radius=8.0, mach_number=mach, mass_ratio=q, eccentricity=e, nu=nu)
        mesh = setup.mesh(n)
        prim = initial_condition(setup, mesh, 0.0)
        prim[..., 0] += 1e-3 * rng.uniform(-1.0, 1.0, size=(n, n))
        out.append(Disk(setup, mesh, prim))
    return out


def main(argv=None):
    """A few steps of a seeded batch of disks without graphs (a profiling /
    smoke case): python -m sailfish_b200.batched --disks 16 --sizes 256,512"""
    import argparse

    import torch

    p = argparse.ArgumentParser(description=main.__doc__)
    p.add_argument("--disks", type=int, default=16)
    p.add_argument("--sizes", default="256,512")
    p.add_argument("--steps", type=int, default=4)
    p.add_argument("--seed", type=int, default=2024)
    a = p.parse_args(argv)
    sizes = tuple(int(v) for v in a.sizes.split(","))
    diags = [dict(quantity="mdot", which_mass=1, accretion=True), dict(quantity="mdot", which_mass=2, accretion=True),
             dict(quantity="torque", which_mass="both", gravity=True)]
    b = BatchedSolver(config2_disks(a.disks, seed=a.seed, sizes=sizes), diagnostics=diags)
    b.run(a.steps, graph=False)
    torch.cuda.synchronize()
    print("zones", b.total_zones)


if __name__ == "__main__":
    main()
