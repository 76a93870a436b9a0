"""
The plain solver split over several GPUs: one process per GPU, each holding
one patch of the mesh (a slab of rows), as the reference's patches split it
(subdivide.py:35-60: rows divided as evenly as possible, the first ones one
longer; each patch with its own edge coordinates, cbdiso_2d.py:69-80).

Per RK stage each rank runs the fused stage kernel on its slab (which writes
zero-gradient guards on all four sides), then replaces the guard rows that
face a neighbouring patch with the neighbour's two edge rows, as the
reference's set_bc copies them between patches (cbdiso_2d.py:553-586): one
contiguous block of 2 (nj + 4) 3 doubles each way (4 fields for the
gamma-law solver), exchanged with
torch.distributed point-to-point operations (NCCL over NVLink between GPUs,
gloo between CPU processes). After each step the wavespeed maximum is
all-reduced (MAX, exact), so every rank's next dt is the same; the
diagnostic sums are gathered and added in patch order, then scaled by
dx dy, as the reference sums its patches (cbdiso_2d.py:478-503).

No TMA or bulk copy with cluster multicast is involved: the exchange is a
plain collective library transfer between device buffers.
"""

from __future__ import annotations

from typing import Callable, Optional

import numpy as np

from .cbdiso_2d import COMPLEX_QUANTITIES, NG, Solver
from .solver_base import SolverBase


def subdivide(n, parts):
    """Row ranges of the patches (subdivide.py:35-60)."""
    q, r = divmod(n, parts)
    a = 0
    for k in range(parts):
        b = a + q + (1 if k < r else 0)
        yield a, b
        a = b


class DistributedSolver(SolverBase):
    """
    cbdiso_2d (or cbdgam_2d) over the ranks of a torch.distributed process
    group, one patch per rank. Same interface as the single-GPU Solver;
    `solution` gathers the whole mesh on every rank. `engine` builds the
    per-rank patch solver from the same arguments plus index_range (default:
    cbdgam_2d.Solver for a gamma-law physics dict, else cbdiso_2d.Solver).
    """

    def __init__(self, setup=None, mesh=None, time=0.0, solution=None, physics=dict(), options=dict(), group=None,
                 engine: Optional[Callable] = None, comm=None):
        """`comm` stands in for torch.distributed (the functions used here:
        get_rank, get_world_size, get_global_rank, P2POp, isend, irecv,
        batch_isend_irecv, all_reduce, ReduceOp, all_gather_object)."""
        if comm is None:
            import torch.distributed as comm
        dist = comm

        self._dist = dist
        self._group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        ni, nj = mesh.shape
        if self.world > ni:
            raise ValueError(f"{self.world} patches for {ni} rows")
        self.ranges = list(subdivide(ni, self.world))
        self.mesh = mesh
        self.setup = setup
        if engine is None:
            from .physics import enum_value

            if enum_value(dict(physics).get("eos_type", 1)) == 3:
                from .cbdgam_2d import Solver as engine  # the gamma-law solver's patches
            else:
                engine = Solver
        make = engine
        self.local = make(setup=setup, mesh=mesh, time=time, solution=solution, physics=physics, options=options,
                          index_range=self.ranges[self.rank])
        self.local._stage_hook = self._exchange
        self.local._step_hook = self._reduce_wavespeed
        # the patch starts with zero-gradient guards everywhere: the rows facing
        # a neighbour take the neighbour's edge rows before the first stage
        self._exchange(-1, self.local.state_buffer())

    def _peer(self, r):
        if self._group is None:
            return r
        return self._dist.get_global_rank(self._group, r)

    def _exchange(self, stage, buf):
        """Guard rows facing a neighbour <- the neighbour's two edge rows."""
        dist = self._dist
        ops = []
        if self.rank > 0:
            lo = self._peer(self.rank - 1)
            ops.append(dist.P2POp(dist.isend, buf[NG:2 * NG], lo, self._group))
            ops.append(dist.P2POp(dist.irecv, buf[0:NG], lo, self._group))
        if self.rank < self.world - 1:
            hi = self._peer(self.rank + 1)
            ops.append(dist.P2POp(dist.isend, buf[-2 * NG:-NG], hi, self._group))
            ops.append(dist.P2POp(dist.irecv, buf[-NG:], hi, self._group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()

    def _reduce_wavespeed(self):
        self._dist.all_reduce(self.local.wavespeed_buffer(), op=self._dist.ReduceOp.MAX, group=self._group)
        self.local.wavespeed_changed()

    # ------------------------------------------------------------------
    # SolverBase
    # ------------------------------------------------------------------

    @property
    def solution(self):
        parts = [None] * self.world
        self._dist.all_gather_object(parts, self.local.solution, group=self._group)
        return np.concatenate(parts, axis=0)

    @property
    def primitive(self):
        return None

    @property
    def time(self):
        return self.local.time

    @property
    def options(self):
        return self.local.options

    @property
    def physics(self):
        return self.local.physics

    @property
    def recommended_cfl(self):
        return self.local.recommended_cfl

    @property
    def maximum_cfl(self):
        return self.local.maximum_cfl

    def maximum_wavespeed(self):
        if self.local.ensure_wavespeed():
            self._reduce_wavespeed()
        return self.local.maximum_wavespeed()

    def advance(self, dt):
        self.local.advance(dt)

    def _sum_patches(self, sums):
        """Per-rank sums -> their sum in patch order (Python's sum from 0)."""
        gathered = [None] * self.world
        self._dist.all_gather_object(gathered, sums, group=self._group)
        return [sum(g[k] for g in gathered) for k in range(len(sums))]

    def reductions(self):
        loc = self.local
        totals = self._sum_patches(loc.reduction_sums())
        da = self.mesh.dx * self.mesh.dy
        out, k = [], 0
        for d in loc.physics["diagnostics"]:
            if d.quantity == "time":
                out.append(loc.time / self.setup.reference_time_scale)
                continue
            v = totals[k]
            k += 1
            out.append(complex(v) * da if d.quantity in COMPLEX_QUANTITIES else float(v) * da)
        return out

    def run(self, steps, cfl=None, fixed_dt=None, **kwargs):
        """The device-resident loop of cbdiso_2d.Solver.run on every rank
        (no CUDA graphs: the exchanges run between the launches); the time
        series' sums are added over the patches."""
        loc = self.local
        loc.run(steps, cfl=cfl, fixed_dt=fixed_dt, graph=False, **kwargs)
        raw = loc.last_series
        gathered = [None] * self.world
        self._dist.all_gather_object(gathered, raw, group=self._group)
        total = raw.copy()
        for col in range(3, raw.shape[1]):
            for r in range(raw.shape[0]):
                total[r, col] = sum(g[r, col] for g in gathered)
        return loc._series_rows(total)
