"""
Gradients of time-averaged sink accretion rate and gravitational torque of a
circumbinary-disk run, by a hand-written discrete adjoint of the RK2 stage.

Objective (dt sequence frozen at the forward run's values):

    J = ( w_mdot * sum_n dt_n (-(mdot_1 + mdot_2))_n + w_torque * sum_n dt_n torque_n ) / sum_n dt_n

with mdot and torque the reductions of cbdiso_2d.Solver.reductions()
(cbdiso_2d.py:370-503) of the state after step n, with the end-of-step point
masses. Gradients are with respect to the initial primitive state (its
density component is dJ / dSigma_0) and to the parameters
(q, e, nu, sink_rate) of a CircumbinaryDisk.

Forward: the device stepper (Solver.run) advances the run in segments of
`checkpoint_every` steps with the frozen dt sequence, keeps a copy of the
state at each segment start and writes every stage record (point masses, dt,
RK weight) into a history array.

Reverse sweep: each segment is recomputed forward from its checkpoint with the
recorded stage records, keeping every state; the branches each stage took
(limiter, HLLE waves, floors) are recorded with
cbdiso_b200_stage_record_branches, and the chained adjoint kernels replay
them backward through the segment. Point-mass parameter derivatives are
contracted on the device with d(mass parameters)/d(q, e) of each stage's time
(complex-step derivatives of the Kepler orbit, exact to rounding: the orbit is
analytic in q and e) and accumulated per block across the whole sweep.

The forward-mode tangent of the same run (cbdiso_b200_stage_tangent) gives
the directional derivative for the dot-product test.
"""

from __future__ import annotations

import cmath
import ctypes
import math
from typing import NamedTuple, Optional

import numpy as np

from . import _capi
from ._graphs import capture
from .cbdiso_2d import NG, NQ, Solver, initial_condition
from .kepler import OrbitalElements
from .setups import CircumbinaryDisk

NPAR = 12
PARAM_NAMES = ("mass_ratio", "eccentricity", "nu", "sink_rate")


class Params(NamedTuple):
    mass_ratio: float = 0.5
    eccentricity: float = 0.1
    nu: float = 1e-3
    sink_rate: float = 10.0


def _kepler_complex(t, a, m, q, e):
    """kepler.py:329-366 evaluated with complex q and e (complex-step)."""
    w = math.sqrt(1.0 * m / a / a / a)
    p = 2.0 * math.pi / w
    tt = t - p * math.floor(t / p)
    n = w * tt
    k = complex(n)
    it = 0
    while abs(k - e * cmath.sin(k) - n) > 1e-15:
        k -= (k - e * cmath.sin(k) - n) / (1.0 - e * cmath.cos(k))
        it += 1
        if it > 10:
            raise ValueError("solve_newton_rapheson: no solution")
    m1 = m / (1.0 + q)
    m2 = m - m1
    ck, sk = cmath.cos(k), cmath.sin(k)
    x1 = -a * q / (1.0 + q) * (e - ck)
    y1 = +a * q / (1.0 + q) * sk * cmath.sqrt(1.0 - e * e)
    vx1 = -a * q / (1.0 + q) * w / (1.0 - e * ck) * sk
    vy1 = +a * q / (1.0 + q) * w / (1.0 - e * ck) * ck * cmath.sqrt(1.0 - e * e)
    return [x1, y1, vx1, vy1, m1, -x1 / q, -y1 / q, -vx1 / q, -vy1 / q, m2]


def mass_jacobian(t, q, e, a=1.0, m=1.0, h=1e-30):
    """d(x, y, vx, vy, mass of both masses)/d(q, e) at time t: 10 x 2."""
    jq = [v.imag / h for v in _kepler_complex(t, a, m, complex(q, h), complex(e, 0.0))]
    je = [v.imag / h for v in _kepler_complex(t, a, m, complex(q, 0.0), complex(e, h))]
    return np.array([jq, je]).T


def _kepler_complex_many(t, a, m, q, e):
    """_kepler_complex over an array of times (the same Newton iteration and
    stopping rule, per element): 10 x len(t) complex."""
    w = math.sqrt(1.0 * m / a / a / a)
    p = 2.0 * math.pi / w
    t = np.asarray(t, dtype=np.float64)
    n = w * (t - p * np.floor(t / p))
    k = n.astype(np.complex128)
    for it in range(11):
        f = k - e * np.sin(k) - n
        todo = np.abs(f) > 1e-15
        if not todo.any():
            break
        if it == 10:
            raise ValueError("solve_newton_rapheson: no solution")
        k = np.where(todo, k - f / (1.0 - e * np.cos(k)), k)
    m1 = m / (1.0 + q)
    m2 = m - m1
    ck, sk = np.cos(k), np.sin(k)
    x1 = -a * q / (1.0 + q) * (e - ck)
    y1 = +a * q / (1.0 + q) * sk * np.sqrt(1.0 - e * e)
    vx1 = -a * q / (1.0 + q) * w / (1.0 - e * ck) * sk
    vy1 = +a * q / (1.0 + q) * w / (1.0 - e * ck) * ck * np.sqrt(1.0 - e * e)
    ones = np.ones_like(n)
    return np.stack([x1, y1, vx1, vy1, m1 * ones, -x1 / q, -y1 / q, -vx1 / q, -vy1 / q, m2 * ones])


# segment rows of the stage adjoints when many sweeps share the GPU: longer
# segments do less lead-row work per CTA, and the concurrent sweeps supply the
# CTAs (32 disks of 256^2 and 512^2, forward and adjoint as one captured
# graph: 4 rows 978 ms, 8 rows 853, 16 rows 791, 32 rows 762; over 8 eager
# streams 8 and 32 rows ran within 1.5 % of each other)
SHARED_SWEEP_ROWS = 32


def mass_jacobians(times, q, e, a=1.0, m=1.0, h=1e-30):
    """mass_jacobian at every time of `times`: len(times) x 10 x 2."""
    jq = _kepler_complex_many(times, a, m, complex(q, h), complex(e, 0.0)).imag / h
    je = _kepler_complex_many(times, a, m, complex(q, 0.0), complex(e, h)).imag / h
    return np.stack([jq.T, je.T], axis=-1)


class AdjointRun:
    """
    A differentiable circumbinary-disk run on one GPU: config-0 physics on
    [-8, 8]^2 with the given (q, e, nu, sink_rate), RK2, `steps` steps at CFL
    `cfl` (dt frozen after the first forward run), EXACT precision.
    """

    def __init__(self, resolution=512, steps=400, checkpoint_every=20, cfl=0.3, plm_theta=1.5, mach=10.0,
                 domain_radius=8.0, store_states=None):
        self.n = resolution
        self.steps = steps
        self.checkpoint_every = checkpoint_every
        # keep every stage state of the forward run (no recompute) when it
        # fits: None = when it takes under half the free device memory
        self.store_states = store_states
        self.cfl = cfl
        self.plm_theta = plm_theta
        self.mach = mach
        self.domain_radius = domain_radius
        self.dts: Optional[np.ndarray] = None
        self._lib = _capi.lib()

    # ------------------------------------------------------------------
    def setup(self, params: Params):
        return CircumbinaryDisk(domain_radius=self.domain_radius, mach_number=self.mach,
                                mass_ratio=float(params.mass_ratio), eccentricity=float(params.eccentricity),
                                nu=float(params.nu), sink_rate=float(params.sink_rate))

    def initial_state(self, seed=0):
        setup = self.setup(Params())
        mesh = setup.mesh(self.n)
        prim = initial_condition(setup, mesh, 0.0)
        prim[..., 0] += 1e-3 * np.random.default_rng(seed).uniform(-1.0, 1.0, size=(self.n, self.n))
        return prim

    def _forward_solver(self, params, prim0):
        """The solver of forward runs, kept while the parameters stay (its
        buffers, and the CUDA graphs recorded on them, are reused)."""
        key = tuple(float(v) for v in params)
        cached = getattr(self, "_fwd_solver", None)
        if cached is not None and cached[0] == key:
            cached[1].reset(prim0, 0.0)
            return cached[1]
        self._fwd_solver = None
        s = self._solver(params, prim0)
        self._fwd_solver = (key, s)
        return s

    def _solver(self, params, prim0):
        setup = self.setup(params)
        mesh = setup.mesh(self.n)
        physics = setup.physics
        physics["diagnostics"] = [dict(quantity="mdot", which_mass=1, accretion=True),
                                  dict(quantity="mdot", which_mass=2, accretion=True),
                                  dict(quantity="torque", which_mass="both", gravity=True)]
        return make_solver_exact(setup, mesh, physics, prim0, self.plm_theta)

    # ------------------------------------------------------------------
    def forward(self, prim0, params: Params, freeze=False, keep=False):
        """
        Run the steps; returns J = (mean accretion rate, mean torque). The
        first call (or freeze=True) fixes the dt sequence from the CFL rule;
        later calls reuse it. With keep, checkpoints and the stage-record
        history are kept for gradient().
        """
        import torch

        s = self._forward_solver(params, prim0)
        steps, K = self.steps, self.checkpoint_every
        fresh = self.dts is None or freeze
        dts_dev = None
        if not fresh:
            dts_dev = self._kept("_dts_dev", (steps,), torch.float64, s.device)
            dts_dev.copy_(torch.from_numpy(np.ascontiguousarray(self.dts)))
        nb = int(self._lib.cbdiso_b200_stage_record_bytes())
        history = self._kept("_history", (steps * 2 * nb,), torch.uint8, s.device) if keep else None
        t_start = s.time
        rows, cps, trajectory = [], {}, None
        if keep and self._keep_all(s):
            trajectory = self._kept("_trajectory", (2 * steps + 1,) + tuple(s._buf[0].shape), torch.float64,
                                    s.device)
            rows = s.run(steps, cfl=self.cfl, dt_sequence=dts_dev, history=history, trajectory=trajectory)
        else:
            # one run: a checkpoint before every segment of K steps, taken on
            # the device between the segments' graph replays
            store = self._checkpoint_store(s) if keep else None
            rows = s.run(steps, cfl=self.cfl, steps_per_graph=K, dt_sequence=dts_dev, history=history,
                         checkpoints=store)
            if keep:
                cps = {start: store[start // K] for start in range(0, steps, K)}
        dts = np.array([r[-1] for r in rows])
        if fresh:
            self.dts = dts
        mdot = np.array([-(r[0] + r[1]) for r in rows])
        torque = np.array([r[2] for r in rows])
        w = self.dts / self.dts.sum()
        J = np.array([np.dot(w, mdot), np.dot(w, torque)])
        if keep:
            self._fwd = dict(solver=s, t_start=t_start, checkpoints=cps, params=params, history=history,
                             record_bytes=nb, trajectory=trajectory)
        return J

    def _kept(self, name, shape, dtype, device):
        """A device buffer kept on the run and reused by later forward runs
        of the same shape (so that the reverse sweep's graph stays valid)."""
        import torch

        t = getattr(self, name, None)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype or t.device != device:
            setattr(self, name, None)
            t = torch.empty(shape, dtype=dtype, device=device)
            setattr(self, name, t)
        return t

    def _checkpoint_store(self, s):
        """Checkpoint slots (one per segment), kept on the run and reused."""
        import torch

        shape = (-(-self.steps // self.checkpoint_every),) + tuple(s._buf[0].shape)
        store = getattr(self, "_checkpoints", None)
        if store is None or tuple(store.shape) != shape or store.device != s._buf[0].device:
            store = self._checkpoints = torch.empty(shape, dtype=torch.float64, device=s._buf[0].device)
        return store

    def _keep_all(self, s):
        if self.store_states is not None:
            return bool(self.store_states)
        import torch

        need = (2 * self.steps + 1) * s._buf[0].numel() * 8
        free, _ = torch.cuda.mem_get_info(s.device)
        return need < free // 2

    def stage_times(self, t_start):
        """(t0, t1, t_end) of every step, from the frozen dt sequence with the
        solver's stage-time rule (cbdiso_2d.py:239): steps x 3."""
        out = np.empty((self.steps, 3))
        t = t_start
        for n, dt in enumerate(self.dts):
            dt = float(dt)
            t1 = t * 0.0 + (t + dt) * 1.0
            t_end = t * 0.5 + (t1 + dt) * 0.5
            out[n] = (t, t1, t_end)
            t = t_end
        return out

    # ------------------------------------------------------------------
    def _records(self, s, t0, dt):
        """Device stage records of one RK2 step starting at t0."""
        import torch

        lib = self._lib
        t1 = t0 * 0.0 + (t0 + dt) * 1.0
        t_end = t0 * 0.5 + (t1 + dt) * 0.5
        ep = s._epilogue(t_end, True, [])
        nb = int(lib.cbdiso_b200_stage_record_bytes())
        host = bytearray(2 * nb)
        for k, (a, ts) in enumerate(((0.0, t0), (0.5, t1))):
            st = _capi.Stage()
            m1, m2 = s._physics.point_masses(ts)
            from .cbdiso_2d import _mass_struct

            _mass_struct(m1, st.mass[0])
            _mass_struct(m2, st.mass[1])
            st.a, st.dt, st.buffer_central_mass = a, dt, m1.mass + m2.mass
            buf = (ctypes.c_char * nb)()
            _capi.check(lib.cbdiso_b200_stage_record(ctypes.byref(s._grid), ctypes.byref(st), ctypes.byref(ep),
                                                     buf), "stage_record")
            host[k * nb:(k + 1) * nb] = bytes(buf)
        dev = torch.frombuffer(host, dtype=torch.uint8).to(s.device)
        return dev, nb, (t0, t1, t_end)

    def gradient(self, weights=(1.0, 0.0), graph=True):
        """
        dJ/dprim0 (ni, nj, 3) and dJ/d(q, e, nu, sink_rate) for
        J = weights[0] * mean accretion + weights[1] * mean torque, at the
        last forward(keep=True) run. With `graph`, the sweep runs from CUDA
        graphs: over a stored trajectory one graph for the whole run;
        otherwise one graph per full segment that reverses it while the
        segment before it in time is recomputed from its checkpoint on a
        second stream (two buffer sets, the stage records and Jacobians staged
        into them). The results are the same bits either way.
        """
        import torch

        f = self._fwd
        s: Solver = f["solver"]
        steps, K = self.steps, self.checkpoint_every
        history, nb = f["history"], f["record_bytes"]
        w, jac = self._sweep_inputs(weights)
        trajectory = f["trajectory"]
        sweep = self._sweep(s, 0 if trajectory is not None else min(K, steps), w)
        sweep.chain.zero_()
        sweep._lam3.zero_()
        if trajectory is not None:
            # every state of the forward run is at hand: no recompute
            if graph:
                sweep.replay_stored(history, jac, steps, trajectory)
            else:
                sweep.run(history, jac, steps, states=trajectory)
            return sweep.finish()
        segments = [(start, min(start + K, steps)) for start in reversed(range(0, steps, K))]
        cps = f["checkpoints"]
        if graph and segments and segments[0][1] - segments[0][0] != sweep.k:
            # a short last segment (reversed first): eagerly
            start, stop = segments.pop(0)
            sweep.p[0].copy_(cps[start])
            sweep.run(history[start * 2 * nb:stop * 2 * nb], jac[start:stop], stop - start)
        if not graph:
            for start, stop in segments:
                sweep.p[0].copy_(cps[start])
                sweep.run(history[start * 2 * nb:stop * 2 * nb], jac[start:stop], stop - start)
            return sweep.finish()
        # full segments, pipelined: segment i is reversed while segment i + 1
        # (earlier in time) is recomputed into the other buffer set
        if segments:
            start, stop = segments[0]
            sweep.stage(0, cps[start], history[start * 2 * nb:stop * 2 * nb], jac[start:stop])
            sweep.replay_recompute(0)
        b = 0
        for i in range(len(segments)):
            more = i + 1 < len(segments)
            if more:
                start, stop = segments[i + 1]
                sweep.stage(1 - b, cps[start], history[start * 2 * nb:stop * 2 * nb], jac[start:stop])
            sweep.replay_pipeline(b, more)
            b = 1 - b
        return sweep.finish()

    def _sweep_inputs(self, weights):
        """The chained objective weights (per unit time, times the zone area)
        and the device array of every stage's Kepler Jacobians (steps x 60)
        of the last forward(keep=True) run."""
        import torch

        f = self._fwd
        s: Solver = f["solver"]
        params: Params = f["params"]
        c = s.mesh.dx * s.mesh.dy / self.dts.sum()
        w = (weights[0] * c, weights[1] * c)
        times = self.stage_times(f["t_start"])
        jac = torch.from_numpy(mass_jacobians(times.reshape(-1), params.mass_ratio,
                                              params.eccentricity).reshape(self.steps, 60)).to(s.device)
        return w, jac

    def _sweep(self, s, k, w):
        """The reverse-sweep buffers and graph for segments of k steps, cached
        on the run while the grid (its Consts), k and the weights stay."""
        key = (bytes(s._grid), k, w)
        cached = getattr(self, "_sweep_cache", None)
        if cached is None or cached.key != key:
            self._sweep_cache = _ReverseSweep(self._lib, s, k, w, key)
        return self._sweep_cache

    # ------------------------------------------------------------------
    def tangent(self, prim0, params: Params, dprim0, dparams, weights=(1.0, 0.0)):
        """
        Directional derivative of J along (dprim0, dparams) by the
        forward-mode tangent kernels, with the frozen dt sequence.
        """
        import torch

        lib = self._lib
        s = self._solver(params, prim0)
        g = ctypes.byref(s._grid)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        P = lambda t: ctypes.c_void_p(t.data_ptr())
        shape = s._buf[0].shape
        f64 = dict(dtype=torch.float64, device=s.device)
        p = s._buf[0].clone()
        dp = torch.zeros(shape, **f64)
        dp[NG:-NG, NG:-NG] = torch.from_numpy(np.ascontiguousarray(dprim0)).to(s.device)
        _capi.check(lib.cbdiso_b200_fill_guards(g, P(dp), stream), "fill_guards")
        q, e = params.mass_ratio, params.eccentricity
        dq, de, dnu, drate = (float(v) for v in dparams)
        total = self.dts.sum()
        da = s.mesh.dx * s.mesh.dy
        parts = torch.zeros(256, **f64)
        acc = 0.0
        t = s.time
        for n in range(self.steps):
            dt = float(self.dts[n])
            dev, nb, (t0, t1, t_end) = self._records(s, t, dt)
            dm0 = mass_jacobian(t0, q, e) @ np.array([dq, de])
            dm1 = mass_jacobian(t1, q, e) @ np.array([dq, de])
            dme = mass_jacobian(t_end, q, e) @ np.array([dq, de])
            star, dstar = torch.empty(shape, **f64), torch.empty(shape, **f64)
            out, dout = torch.empty(shape, **f64), torch.empty(shape, **f64)
            d0 = (ctypes.c_double * 10)(*dm0)
            d1 = (ctypes.c_double * 10)(*dm1)
            de_ = (ctypes.c_double * 10)(*dme)
            _capi.check(lib.cbdiso_b200_stage_tangent(g, P(dev), d0, dnu, drate, P(p), P(dp), None, None, P(star),
                                                      P(dstar), stream), "stage_tangent")
            _capi.check(lib.cbdiso_b200_stage_tangent(g, ctypes.c_void_p(dev.data_ptr() + nb), d1, dnu, drate,
                                                      P(star), P(dstar), P(p), P(dp), P(out), P(dout), stream),
                        "stage_tangent")
            c = dt / total * da
            _capi.check(lib.cbdiso_b200_objective_tangent(g, ctypes.c_void_p(dev.data_ptr() + nb), de_, drate,
                                                          P(out), P(dout), weights[0] * c, weights[1] * c,
                                                          P(parts), 256, stream), "objective_tangent")
            acc += float(parts.sum().item())
            p, dp = out, dout
            t = t_end
        return acc


class _ReverseSweep:
    """
    Buffers of the reverse sweep over segments of k steps: two sets (0, 1) of
    the recomputed states p[0..k] and stage-1 outputs with their staged stage
    records and Jacobians (none for k = 0: the states come from a recorded
    trajectory), the adjoint states, the adjoint workspace and the chained
    parameter accumulator; and CUDA graphs of a full segment. The recompute of
    a segment needs only its checkpoint and stage records, not the adjoint, so
    in the graphed sweep one set's segment is reversed while the other set's
    (the next segment back in time) is recomputed on a second stream.
    """

    def __init__(self, lib, s, k, w, key):
        import torch

        self.key, self.k, self.w, self.lib = key, k, w, lib
        self.grid = _capi.Grid.from_buffer_copy(s._grid)
        g = ctypes.byref(self.grid)
        shape = s._buf[0].shape
        f64 = dict(dtype=torch.float64, device=s.device)
        self.nb = int(lib.cbdiso_b200_stage_record_bytes())
        nsets = 2 if k > 0 else 1
        self.pset = [[torch.empty(shape, **f64) for _ in range(k + 1)] for _ in range(nsets)]
        self.sset = [[torch.empty(shape, **f64) for _ in range(k)] for _ in range(nsets)]
        self.p, self.stars = self.pset[0], self.sset[0]
        # lambda, lambda_star, lambda_n side by side: the two buffers cleared
        # after each reversed step (lambda_star and the next lambda_n) are
        # always adjacent, one fill for both
        self._lam3 = torch.zeros((3,) + tuple(shape), **f64)
        self.lam, self.lam_star, self.lam_n = self._lam3[0], self._lam3[1], self._lam3[2]
        self.ws = torch.empty(int(lib.cbdiso_b200_adjoint_workspace_bytes(g)) // 8 + 8, **f64)
        self.rows = int(lib.cbdiso_b200_adjoint_chain_blocks(g))
        self.chain = torch.zeros(self.rows * 4, **f64)
        self.scratch = torch.zeros(int(lib.cbdiso_b200_scratch_bytes(g)) // 8 + 8, **f64)
        self.result = torch.zeros(64, **f64)
        # the recompute's face cache (recomputes never overlap one another);
        # a zeroed header holds no valid key
        self.fcache = torch.zeros(int(lib.cbdiso_b200_face_cache_bytes(g)) // 8, **f64) if k > 0 else None
        self.hset = [torch.empty(max(k, 1) * 2 * self.nb, dtype=torch.uint8, device=s.device) for _ in range(nsets)]
        self.jset = [torch.empty((max(k, 1), 60), **f64) for _ in range(nsets)]
        self.hist, self.jac = self.hset[0], self.jset[0]
        self.graphs = {}

    def recompute(self, p, stars, hist, count):
        """The segment's states from p[0] with the recorded stage records,
        keeping every state (the in-place final stage is replayed out of
        place: inputs star, p[n] -> p[n + 1]), on the current stream. The
        stages use the sweep's face cache as the forward run does (first
        stage reader, second writer): the same bits as without it, with the
        first stage's face sound speeds and gravity factors loaded rather
        than evaluated (a segment's first step fills the cache)."""
        import torch

        lib, g, nb = self.lib, ctypes.byref(self.grid), self.nb
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        P = lambda t: ctypes.c_void_p(t.data_ptr())
        rec = lambda n, k: ctypes.c_void_p(hist.data_ptr() + (2 * n + k) * nb)
        s1, s2 = _capi.Stage(), _capi.Stage()
        s2.a = 0.5
        fc = P(self.fcache)
        for n in range(count):
            _capi.check(lib.cbdiso_b200_advance_stage_cached(g, ctypes.byref(s1), rec(n, 0), P(p[n]), None,
                                                             P(stars[n]), None, None, None, fc, 2, stream),
                        "advance_stage_cached")
            _capi.check(lib.cbdiso_b200_advance_stage_cached(g, ctypes.byref(s2), rec(n, 1), P(stars[n]), P(p[n]),
                                                             P(p[n + 1]), None, None, None, fc, 1, stream),
                        "advance_stage_cached")

    def reverse(self, p, stars, hist, jac, count):
        """The reverse sweep over one segment of `count` steps whose states
        are p[0..count] and stars, with stage records `hist` (2 per step) and
        Jacobians `jac` (count x 60: stage 1, stage 2, end of step, 10 x 2
        each), on the current stream."""
        import torch

        lib, g, nb = self.lib, ctypes.byref(self.grid), self.nb
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        P = lambda t: ctypes.c_void_p(t.data_ptr())
        rec = lambda n, k: ctypes.c_void_p(hist.data_ptr() + (2 * n + k) * nb)
        jp = lambda n, k: ctypes.c_void_p(jac.data_ptr() + (60 * n + 20 * k) * 8)
        ws, chain = P(self.ws), P(self.chain)
        check = _capi.check
        lam, lam_n, lam_star = self.lam, self.lam_n, self.lam_star
        for n in reversed(range(count)):
            pn, star, out = p[n], stars[n], p[n + 1]
            # objective term of step n (state after the step, end masses;
            # the chained weights are per unit time: dt_n / sum(dt) * dA)
            check(lib.cbdiso_b200_objective_adjoint_chained(g, rec(n, 1), P(out), self.w[0], self.w[1], P(lam),
                                                            jp(n, 2), chain, ws, stream), "objective_adjoint")
            # stage 2: inputs star (read), pn (u_n); lam_star starts at zero
            check(lib.cbdiso_b200_stage_adjoint_chained(g, rec(n, 1), P(star), P(pn), P(out), P(lam), P(lam_star),
                                                        P(lam_n), jp(n, 1), chain, ws, stream), "stage_adjoint")
            # stage 1: input pn
            check(lib.cbdiso_b200_stage_adjoint_chained(g, rec(n, 0), P(pn), None, P(star), P(lam_star), P(lam_n),
                                                        None, jp(n, 0), chain, ws, stream), "stage_adjoint")
            lam, lam_n = lam_n, lam
            # lam_star and the next lam_n back to zero (adjacent in _lam3)
            lo = 0 if lam_n.data_ptr() == self._lam3[0].data_ptr() else 1
            self._lam3[lo:lo + 2].zero_()
        if lam is not self.lam:
            # an odd count leaves the adjoint in the other buffer
            self.lam.copy_(lam)
            self.lam_n.zero_()

    def run(self, hist, jac, count, states=None):
        """Recompute (into set 0) and reverse one segment of `count` steps.
        With `states` (a recorded trajectory: u_n at 2n, the first stage's
        output at 2n + 1) nothing is recomputed."""
        if states is not None:
            p, stars = states[0::2], states[1::2]
        else:
            p, stars = self.p, self.stars
            self.recompute(p, stars, hist, count)
        self.reverse(p, stars, hist, jac, count)

    def stage(self, b, checkpoint, hist, jac):
        """Stage a full segment's inputs into set b."""
        self.pset[b][0].copy_(checkpoint)
        self.hset[b].copy_(hist)
        self.jset[b].copy_(jac)

    def _graph(self, key, body):
        import torch

        graph = self.graphs.get(key)
        if graph is None:
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            graph = torch.cuda.CUDAGraph()
            # capture records the launches without running them
            with capture(graph, side):
                body(side)
            torch.cuda.current_stream().wait_stream(side)
            self.graphs[key] = graph
        graph.replay()

    def replay_recompute(self, b):
        """Recompute the segment staged in set b (one CUDA graph)."""
        self._graph(("recompute", b),
                    lambda side: self.recompute(self.pset[b], self.sset[b], self.hset[b], self.k))

    def replay_pipeline(self, b, recompute_other):
        """Reverse the segment of set b and, when `recompute_other`, recompute
        the segment staged in the other set on a second stream at the same
        time (one CUDA graph)."""
        import torch

        o = 1 - b

        def body(side):
            if recompute_other:
                other = torch.cuda.Stream()
                other.wait_stream(side)
                with torch.cuda.stream(other):
                    self.recompute(self.pset[o], self.sset[o], self.hset[o], self.k)
            self.reverse(self.pset[b], self.sset[b], self.hset[b], self.jset[b], self.k)
            if recompute_other:
                side.wait_stream(other)

        self._graph(("pipeline", b, bool(recompute_other)), body)

    def replay_stored(self, hist, jac, count, states):
        """The whole sweep over a stored trajectory from one CUDA graph,
        captured on the first call for these trajectory and record buffers;
        the Jacobians are staged into a buffer of the sweep."""
        import torch

        key = (hist.data_ptr(), states.data_ptr(), count, tuple(states.shape))
        if getattr(self, "_stored_key", None) != key:
            self._stored_graph = None
            self._stored_jac = torch.empty_like(jac)
            self._stored_jac.copy_(jac)
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            graph = torch.cuda.CUDAGraph()
            with capture(graph, side):
                self.run(hist, self._stored_jac, count, states=states)
            torch.cuda.current_stream().wait_stream(side)
            self._stored_graph, self._stored_key = graph, key
        else:
            self._stored_jac.copy_(jac)
        self._stored_graph.replay()

    def finish(self):
        import torch

        out4 = torch.zeros(4, dtype=torch.float64, device=self.chain.device)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _capi.check(self.lib.cbdiso_b200_adjoint_chain_finish(ctypes.c_void_p(self.chain.data_ptr()), self.rows,
                                                              ctypes.c_void_p(out4.data_ptr()), stream),
                    "chain_finish")
        grad_state = self.lam[NG:-NG, NG:-NG].cpu().numpy()
        return grad_state, out4.cpu().numpy()


def make_solver_exact(setup, mesh, physics, prim0, plm_theta):
    return Solver(setup=setup, mesh=mesh, solution=prim0, physics=physics,
                  options=dict(rk_order=2, plm_theta=plm_theta, precision="exact"))


# ---------------------------------------------------------------------------
# many disks
# ---------------------------------------------------------------------------


class AdjointDisk(NamedTuple):
    """One disk of a batched adjoint: grid size, parameters, Mach number and
    the initial primitive state (ni, nj, 3) (None: the setup's disk with
    seeded noise)."""

    resolution: int
    params: Params
    mach: float = 10.0
    prim0: Optional[np.ndarray] = None


class BatchedAdjoint:
    """
    Forward runs and gradients of many independent disks on one GPU. Each
    disk is an AdjointRun (its own dt sequence, stage records and adjoint
    buffers); the disks are spread over `streams` CUDA streams, each driven
    by its own host thread, so that the kernels of different disks overlap
    on the device and their host-side launch work overlaps on the CPU. Each
    disk's results are identical to running its AdjointRun alone.
    """

    def __init__(self, disks, steps=200, checkpoint_every=20, cfl=0.3, plm_theta=1.5, streams=8,
                 store_states=None):
        self.disks = list(disks)
        self.runs = [AdjointRun(resolution=d.resolution, steps=steps, checkpoint_every=checkpoint_every, cfl=cfl,
                                plm_theta=plm_theta, mach=d.mach, store_states=store_states) for d in self.disks]
        self.prims = [d.prim0 if d.prim0 is not None else r.initial_state(seed=i)
                      for i, (d, r) in enumerate(zip(self.disks, self.runs))]
        self.num_streams = max(1, min(int(streams), len(self.disks)))
        self._streams = None

    def _each(self, fn):
        """fn(i) for every disk, disk i on stream i % num_streams; returns the
        results in disk order."""
        import threading

        import torch

        if self._streams is None:
            # torch hands out pooled streams round-robin; the workers take theirs
            # from the high-priority pool so that no graph capture (whose side
            # streams come from the default pool) can land on a worker's stream
            self._streams = [torch.cuda.Stream(priority=-1) for _ in range(self.num_streams)]
        device = torch.cuda.current_device()
        out = [None] * len(self.disks)
        errors = []
        start = torch.cuda.current_stream()

        def worker(w):
            try:
                torch.cuda.set_device(device)
                st = self._streams[w]
                st.wait_stream(start)
                with torch.cuda.stream(st):
                    for i in range(w, len(self.disks), self.num_streams):
                        out[i] = fn(i)
            except BaseException as exc:  # re-raised on the calling thread
                errors.append(exc)

        threads = [threading.Thread(target=worker, args=(w,)) for w in range(self.num_streams)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for st in self._streams:
            start.wait_stream(st)
        if errors:
            raise errors[0]
        return out

    def forward(self, freeze=False, keep=False):
        """J of every disk (list of (mean accretion, mean torque))."""
        return self._each(lambda i: self.runs[i].forward(self.prims[i], self.disks[i].params, freeze=freeze,
                                                         keep=keep))

    def gradient(self, weights=(1.0, 0.0)):
        """(dJ/dprim0, dJ/d(q, e, nu, sink_rate)) of every disk, after
        forward(keep=True). The sweeps share the GPU, so the stage adjoints
        run in the longest segments (least total work); the library's default
        segment choice is restored afterwards."""
        lib = _capi.lib()
        _capi.check(lib.cbdiso_b200_set_adjoint_segment_rows(SHARED_SWEEP_ROWS), "set_adjoint_segment_rows")
        try:
            return self._each(lambda i: self.runs[i].gradient(weights))
        finally:
            lib.cbdiso_b200_set_adjoint_segment_rows(0)

    # ------------------------------------------------------------------
    # the whole batch's forward and adjoint as one CUDA graph

    def capture(self, weights=(1.0, 0.0)):
        """
        Capture the forward run and the reverse sweep of every disk into one
        CUDA graph: disk d's launches form branch d, on its own stream forked
        from the capturing one, so that all disks' kernels overlap on the
        device with no host work between them. Each replay starts every disk
        from its initial state and initial stepper record (device copies) with
        the frozen dt sequences; the results are read with results().
        Requires a forward(keep=True) with stored states and gradient(weights)
        before (they freeze the dt sequences and set up every buffer); this
        runs one more forward of every disk with its frozen dt sequence.
        """
        import torch

        lib = _capi.lib()
        # one more forward of every disk with its frozen dt sequence attached
        # to the stepper record that the graph starts from
        self.forward(keep=True)
        for r in self.runs:
            if r._fwd.get("trajectory") is None:
                raise ValueError("the captured batch needs stored states (store_states)")
        self._graph_inputs = []
        for r in self.runs:
            f = r._fwd
            s = f["solver"]
            w, jac = r._sweep_inputs(weights)
            sweep = r._sweep(s, 0, w)
            out4 = torch.zeros(4, dtype=torch.float64, device=s.device)
            self._graph_inputs.append(dict(run=r, solver=s, trajectory=f["trajectory"], history=f["history"],
                                           state0=f["trajectory"][0].clone(), record=s.last_stepper_record(),
                                           jac=jac, sweep=sweep, out4=out4))
        _capi.check(lib.cbdiso_b200_set_adjoint_segment_rows(SHARED_SWEEP_ROWS), "set_adjoint_segment_rows")
        try:
            self._graph = self._capture_branches(gradient=True)
            self._graph_forward = self._capture_branches(gradient=False)
        finally:
            lib.cbdiso_b200_set_adjoint_segment_rows(0)

    def _capture_branches(self, gradient):
        import torch

        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        graph = torch.cuda.CUDAGraph()
        branches = [torch.cuda.Stream() for _ in self.runs]
        with capture(graph, side):
            for g_in, st in zip(self._graph_inputs, branches):
                st.wait_stream(side)
                with torch.cuda.stream(st):
                    self._branch_launches(g_in, gradient)
            for st in branches:
                side.wait_stream(st)
        torch.cuda.current_stream().wait_stream(side)
        return graph

    def _branch_launches(self, g_in, gradient=True):
        """One disk's forward and (with `gradient`) reverse sweep, launches only."""
        import torch

        r, s, traj, sweep = g_in["run"], g_in["solver"], g_in["trajectory"], g_in["sweep"]
        traj[0].copy_(g_in["state0"])
        s.trajectory_launches(r.steps, traj, g_in["record"])
        if not gradient:
            return
        sweep.chain.zero_()
        sweep._lam3.zero_()
        sweep.run(g_in["history"], g_in["jac"], r.steps, states=traj)
        # the final reduction adds into its output
        g_in["out4"].zero_()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _capi.check(sweep.lib.cbdiso_b200_adjoint_chain_finish(ctypes.c_void_p(sweep.chain.data_ptr()), sweep.rows,
                                                               ctypes.c_void_p(g_in["out4"].data_ptr()), stream),
                    "chain_finish")

    def replay(self, gradient=True):
        """Run the captured batch (see capture) on the current stream: forward
        and adjoint, or (gradient=False) the forward runs alone."""
        (self._graph if gradient else self._graph_forward).replay()

    def results(self):
        """Per disk, after replay(): (J, dJ/dprim0, dJ/d(q, e, nu, sink_rate))
        with J = (mean accretion, mean torque), as forward() and gradient()
        return them."""
        out = []
        for g_in in self._graph_inputs:
            r, s = g_in["run"], g_in["solver"]
            rows = s.series_after_launches(r.steps)
            mdot = np.array([-(row[0] + row[1]) for row in rows])
            torque = np.array([row[2] for row in rows])
            wt = r.dts / r.dts.sum()
            J = np.array([np.dot(wt, mdot), np.dot(wt, torque)])
            grad_state = g_in["sweep"].lam[NG:-NG, NG:-NG].cpu().numpy()
            out.append((J, grad_state, g_in["out4"].cpu().numpy()))
        return out


def config4_disks(num=32, seed=4096, sizes=(256, 512)):
    """The batched adjoint workload: `num` disks, half of each size in
    `sizes` (seeded order), q ~ U[0.1, 1], e ~ U[0, 0.5], nu ~ logU[1e-4,
    1e-2], sink rate 10, Mach 10, on [-8, 8]^2 with the config-0 physics."""
    rng = np.random.default_rng(seed)
    order = rng.permutation(np.repeat(np.array(sizes), -(-num // len(sizes)))[:num])
    out = []
    for n in order:
        q = float(rng.uniform(0.1, 1.0))
        e = float(rng.uniform(0.0, 0.5))
        nu = float(10.0 ** rng.uniform(-4.0, -2.0))
        out.append(AdjointDisk(int(n), Params(q, e, nu, 10.0)))
    return out


# ---------------------------------------------------------------------------
# torch.autograd interface
# ---------------------------------------------------------------------------


def objective_function(run: AdjointRun, weights=(1.0, 0.0)):
    """
    A torch.autograd.Function computing J(sigma0, params) for `run`:
    sigma0 is the initial surface density (ni, nj) (velocities from the
    setup), params the tensor (q, e, nu, sink_rate); J is a 0-d tensor.
    """
    import torch

    class CircumbinaryObjective(torch.autograd.Function):
        @staticmethod
        def forward(ctx, sigma0, params):
            prim = run.initial_state(seed=0)
            prim[..., 0] = sigma0.detach().cpu().numpy()
            p = Params(*[float(v) for v in params.detach().cpu().tolist()])
            J = run.forward(prim, p, keep=True)
            return torch.tensor(float(weights[0] * J[0] + weights[1] * J[1]), dtype=torch.float64)

        @staticmethod
        def backward(ctx, gJ):
            grad_state, grad_params = run.gradient(weights)
            g = float(gJ)
            return (torch.from_numpy(grad_state[..., 0] * g), torch.from_numpy(grad_params * g))

    return CircumbinaryObjective


def main(argv=None):
    """One forward run and gradient on the device (a profiling / smoke case):
    python -m sailfish_b200.adjoint --resolution 512 --steps 20"""
    import argparse

    import torch

    p = argparse.ArgumentParser(description=main.__doc__)
    p.add_argument("--resolution", type=int, default=512)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--checkpoint-every", type=int, default=20)
    p.add_argument("--store-states", choices=["auto", "yes", "no"], default="auto")
    a = p.parse_args(argv)
    store = dict(auto=None, yes=True, no=False)[a.store_states]
    run = AdjointRun(resolution=a.resolution, steps=a.steps, checkpoint_every=a.checkpoint_every,
                     store_states=store)
    prim = run.initial_state(seed=0)
    params = Params(0.5, 0.1, 1e-3, 10.0)
    run.forward(prim, params, freeze=True, keep=True)
    J = run.forward(prim, params, keep=True)
    _, grad = run.gradient((1.0, 0.0))
    torch.cuda.synchronize()
    print("J", J, "dJ/d(q, e, nu, sink_rate)", grad)


if __name__ == "__main__":
    main()
