"""
Benchmark: zone-updates/s of the plain cbdiso_2d drop-in on one B200.

Workload (the headline throughput configuration): circumbinary disk on
[-8, 8]^2 at 4096^2 zones, FP64, equal-mass circular binary (softening 0.05,
sink radius 0.05, sink rate 10, torque-free sinks), Mach 10 locally
isothermal, nu = 1e-3, PLM theta 1.5, RK2, CFL 0.3, Keplerian buffer beyond
r = 7, with the accretion-rate and torque reductions every step. One "step"
is one driver iteration: dt from the CFL wavespeed, advance(dt), reductions().
Synthetic data: the setup's initial disk plus seeded 1e-3 noise on Sigma,
held in pinned host memory for the end-to-end (e2e) measurement, which
uploads it, runs the public driver loop and downloads the final state.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--size N]

Each state array is 403 MB at 4096^2, larger than the 126 MB L2, so no L2
flush is needed between steps. Rank 0 prints one JSON line.
"""

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_ZONE_UPDATE = 120.0  # RK2 x FP64 x 3 fields: 48 B stage 1 + 72 B stage 2
# DRAM bytes per zone and stage measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum of one step at 2048^2: the RK2 stage-1 launch reading
# the face cache, the stage-2 launch writing it and the stage-2 epilogue
# kernel, halved per stage); scaled by the zone count. It is above the
# algorithmic 60 B because of the cache's 48 B per zone and step and the
# epilogue's 24 B read-back.
NCU_TRAFFIC_PER_ZONE_LAUNCH = (316.53e6 + 62.18e6 + 220.12e6 + 249.12e6 + 100.89e6 + 3.63e6) / 2 / 2048 ** 2
# FP64 thread-instructions (DADD + DMUL + DFMA) per zone and stage, from the
# same three launches (ncu, the sum of
# smsp__sass_thread_inst_executed_op_{dadd,dmul,dfma}_pred_on.sum over zones;
# 2048^2 runs 19-row segments, 4096^2 37-row ones, which recompute fewer
# rows at segment tops: at 4096^2 this slightly overstates the count)
FP64_INST_PER_ZONE_LAUNCH = (318.2 + 509.8 + 114.8) / 2
GAM_FP64_INST_PER_ZONE_LAUNCH = (1224.8 + 1249.8) / 2
DIAGNOSTICS = [dict(quantity="time"), dict(quantity="mdot", which_mass=1, accretion=True),
               dict(quantity="mdot", which_mass=2, accretion=True),
               dict(quantity="torque", which_mass="both", gravity=True)]
SETUP_PARAMS = dict(domain_radius=8.0, mach_number=10.0, mass_ratio=1.0, eccentricity=0.0, sink_rate=10.0,
                    sink_radius=0.05, softening_length=0.05, nu=0.001)
THETA = 1.5
CFL = 0.3


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--size", type=int, default=4096)
    p.add_argument("--precision", default="exact", choices=["exact", "fma", "fast"])
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--tile", default=None, help="columns,rows,occupancy of the stage kernel (default: library)")
    p.add_argument("--no-face-cache", action="store_true",
                   help="recompute the face sound speeds and gravity factors in every stage")
    p.add_argument("--mode", default="auto", choices=["auto", "slab", "replicas"],
                   help="slab: one mesh split into N row slabs (guard rows exchanged over NCCL); replicas: N "
                        "independent runs; auto: slab for N > 1")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the batched-disk and adjoint measurements added to the line at N=1")
    return p.parse_args()


def fp64_peak():
    """FP64 issue rate of this GPU (thread-FMAs per second), measured with
    the library's probe: 8 CTAs of 256 threads per SM, eight independent FMA
    chains per thread, best of three launches timed with CUDA events."""
    import ctypes

    import torch

    from sailfish_b200 import _capi

    lib = _capi.lib()
    blocks = 8 * torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    iterations = 40000
    out = torch.zeros(blocks, dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for rep in range(4):
        start.record()
        _capi.check(lib.cbdiso_b200_fp64_probe(iterations, blocks, ctypes.c_void_p(out.data_ptr()), stream), "probe")
        stop.record()
        torch.cuda.synchronize()
        if rep:
            best = min(best, start.elapsed_time(stop) * 1e-3)
    return lib.cbdiso_b200_fp64_probe_fmas(iterations, blocks) / best


def fp64_roofline(inst_per_launch, kernel_s):
    """The stage kernel against the FP64 pipe: its FP64 thread-instructions
    per launch (ncu counts) over its CUDA-event launch time, against this
    GPU's measured FMA issue rate."""
    peak = fp64_peak()
    achieved = inst_per_launch / kernel_s
    return {"bound": "fp64", "achieved": round(achieved / 1e12, 3), "peak": round(peak / 1e12, 3),
            "unit": "T FP64 thread-instructions/s", "frac": round(achieved / peak, 4),
            "inst_per_launch": inst_per_launch,
            "inst_source": "ncu DADD + DMUL + DFMA thread-instructions per zone at 2048^2 scaled by zones",
            "peak_source": "measured: cbdiso_b200_fp64_probe, independent DFMA chains at full occupancy"}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def bench_config(n, precision):
    """The workload description both arms print for an n^2 run on one GPU."""
    state_mb = n * n * 3 * 8 / 1e6
    l2 = (f"state arrays ({state_mb:.0f} MB each at {n}^2) exceed the 126 MB L2; no flush" if state_mb > 126
          else f"state arrays ({state_mb:.0f} MB each at {n}^2) fit in L2; no flush")
    return {"workload": f"cbdiso_2d circumbinary disk {n}x{n} FP64 RK2 theta {THETA} CFL {CFL}, "
                        "per-step mdot/torque reductions", "zones": n * n, "precision": precision, "l2": l2,
            "parallelism": "single"}


def initial_state(n, seed):
    from sailfish_b200.cbdiso_2d import initial_condition
    from sailfish_b200.setups import CircumbinaryDisk

    setup = CircumbinaryDisk(**SETUP_PARAMS)
    mesh = setup.mesh(n)
    prim = initial_condition(setup, mesh, 0.0)
    rng = np.random.default_rng(seed)
    prim[..., 0] += 1e-3 * rng.uniform(-1.0, 1.0, size=(n, n))
    return setup, mesh, prim


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples (every PERIOD_MS) around
    the timed region. A timed region of a few dozen steps lasts tens of
    milliseconds, less than nvidia-smi needs to start, so the sampler is
    started first and waited for (its first sample), the caller keeps the GPU
    under the timed workload for LOAD_S before the timed region (`load`), and
    the summary keeps the samples from the start of that load to the end of
    the timed region: the clocks under exactly the timed steps."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 50
    LOAD_S = 0.6
    START_TIMEOUT_S = 20.0

    def __init__(self, device_index):
        self.device_index = device_index
        self.proc = None
        self.thread = None
        self.error = None
        self.samples = []  # (host time of arrival, line)
        self.t_load = self.t_stop = None

    def _read(self):
        for line in self.proc.stdout:
            if line.strip():
                self.samples.append((time.perf_counter(), line))

    def __enter__(self):
        import shutil
        import threading

        cmd = ["nvidia-smi", "-i", str(self.device_index), f"--query-gpu={self.FIELDS}",
               "--format=csv,noheader,nounits", "-lms", str(self.PERIOD_MS)]
        if shutil.which("stdbuf"):
            cmd = ["stdbuf", "-oL"] + cmd  # one line per sample as it is taken
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, bufsize=1)
        except (OSError, FileNotFoundError) as e:
            self.proc = None
            self.error = f"nvidia-smi could not be started: {e}"
            return self
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        deadline = time.perf_counter() + self.START_TIMEOUT_S
        while not self.samples and self.proc.poll() is None and time.perf_counter() < deadline:
            time.sleep(0.01)
        return self

    def load(self, step_fn, group_max=None):
        """Runs `step_fn` (some of the timed steps, synchronised) for about
        LOAD_S, so that samples fall under that load. The call count comes
        from the first call's duration; `group_max` makes it the same on all
        ranks where the steps hold collectives."""
        self.t_load = time.perf_counter()
        step_fn()
        once = time.perf_counter() - self.t_load
        n = max(0, math.ceil(self.LOAD_S / max(once, 1e-6)) - 1)
        if group_max is not None:
            n = group_max(n)
        for _ in range(n):
            step_fn()

    def stop(self):
        """Marks the end of the timed region (after its synchronize)."""
        self.t_stop = time.perf_counter()

    def __exit__(self, *exc):
        if self.proc is None:
            return
        if self.t_stop is None:
            self.stop()
        # the sample taken across the end of the timed region
        deadline = time.perf_counter() + 2.0 * self.PERIOD_MS * 1e-3
        while time.perf_counter() < deadline and not any(t > self.t_stop for t, _ in self.samples):
            time.sleep(0.005)
        self.proc.terminate()
        try:
            _, err = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            _, err = self.proc.communicate()
        self.thread.join(timeout=5)
        if not self.samples:
            self.error = ("nvidia-smi returned no samples (exit code "
                          f"{self.proc.returncode}): {(err or '').strip()[:200] or 'no message'}")

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0 = self.t_load if self.t_load is not None else -math.inf
        t1 = (self.t_stop if self.t_stop is not None else math.inf) + self.PERIOD_MS * 1e-3
        window = [line for t, line in self.samples if t0 <= t <= t1]
        for line in window:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            # never a silent null: say why there is no clock record
            why = self.error or f"no parsable samples among {len(window)} lines in the window"
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "unavailable": why}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "period_ms": self.PERIOD_MS,
                "window": f"{self.LOAD_S} s of the timed steps just before the timed region, and the timed region"}


def _max_over_ranks(n, tdist):
    import torch

    t = torch.tensor([int(n)], device="cuda", dtype=torch.int64)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return int(t.item())


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------


def stage_kernel_time(solver, repeats=20):
    """Average device time of one fused stage launch (alternating the two RK2
    stages on the resident state), measured with CUDA events on the launching
    stream."""
    import torch

    dt = solver.mesh.min_spacing() / solver.maximum_wavespeed() * CFL
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(2):
        solver.advance(dt)
    torch.cuda.synchronize()
    start.record()
    for _ in range(repeats):
        solver.advance(dt)
    stop.record()
    torch.cuda.synchronize()
    return start.elapsed_time(stop) * 1e-3 / (2 * repeats)


def slab_size(n, world):
    """Weak scaling: a square mesh with about n^2 zones per GPU (multiple of 64)."""
    return int(round(n * math.sqrt(world) / 64.0)) * 64


def run_slabs(args, rank, world):
    """N GPUs on one mesh of about N * n^2 zones, one row slab per rank
    (sailfish_b200.distributed): guard rows exchanged between stages, the
    wavespeed all-reduced each step."""
    import torch
    import torch.distributed as tdist

    from sailfish_b200 import pinned_empty
    from sailfish_b200.cbdiso_2d import initial_condition
    from sailfish_b200.distributed import DistributedSolver, subdivide
    from sailfish_b200.setups import CircumbinaryDisk

    n = slab_size(args.size, world)
    setup = CircumbinaryDisk(**SETUP_PARAMS)
    mesh = setup.mesh(n)
    physics = setup.physics
    physics["diagnostics"] = DIAGNOSTICS
    a, b = list(subdivide(n, world))[rank]
    prim = initial_condition(setup, mesh, 0.0, rows=(a, b))
    prim[..., 0] += 1e-3 * np.random.default_rng(args.seed + rank).uniform(-1.0, 1.0, size=(b - a, n))
    pinned = pinned_empty(prim.shape)  # the slab in pinned host memory, as in the one-GPU line
    pinned[...] = prim
    prim = pinned
    opts = dict(rk_order=2, plm_theta=THETA, precision=args.precision)
    solver = DistributedSolver(setup=setup, mesh=mesh, solution=prim, physics=physics, options=opts)
    solver.run(max(args.warmup, 3), cfl=CFL)
    tdist.barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clocks:
        # the same step count on every rank: the halo exchange is collective
        clocks.load(lambda: (solver.run(max(args.warmup, 3), cfl=CFL), torch.cuda.synchronize()),
                    group_max=lambda n: _max_over_ranks(n, tdist))
        tdist.barrier()
        torch.cuda.synchronize()
        start.record()
        rows = solver.run(args.steps, cfl=CFL)
        stop.record()
        torch.cuda.synchronize()
        clocks.stop()
    assert len(rows) == args.steps and all(np.isfinite(r[-1]) for r in rows)
    t = torch.tensor([start.elapsed_time(stop) * 1e-3], device="cuda", dtype=torch.float64)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    elapsed = float(t.item())
    value = n * n * args.steps / elapsed

    # end to end: host data in, the public driver loop, the whole state out
    e2e_steps = max(1, args.steps)
    tdist.barrier()
    t0 = time.perf_counter()
    s2 = DistributedSolver(setup=setup, mesh=mesh, solution=prim, physics=physics, options=opts)
    for _ in range(e2e_steps):
        s2.advance(mesh.min_spacing() / s2.maximum_wavespeed() * CFL)
        s2.reductions()
    final = s2.local.solution
    t1 = time.perf_counter()
    t = torch.tensor([t1 - t0], device="cuda", dtype=torch.float64)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    e2e_value = n * n * e2e_steps / float(t.item())
    # per step, summed over the ranks: the slab upload and download
    e2e_bytes = torch.tensor([float(prim.nbytes + final.nbytes)], device="cuda", dtype=torch.float64)
    tdist.all_reduce(e2e_bytes)
    del s2
    peak, peak_kind = measured_peaks()
    if rank != 0:
        return None
    return {
        "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"cbdiso_2d circumbinary disk {n}x{n} FP64 RK2 theta {THETA} CFL {CFL} "
                               f"split into {world} row slabs, per-step mdot/torque reductions",
                   "zones": n * n, "zones_per_gpu": n * n / world, "precision": args.precision,
                   "timed": "DistributedSolver.run: device dt / Kepler per rank, NCCL guard-row exchange "
                            "per stage, wavespeed all-reduce per step",
                   "l2": "state arrays exceed L2; no flush", "parallelism": f"slab{world}"},
        "e2e": {"value": e2e_value, "unit": "zone-updates/s",
                "h2d_bytes_per_step": int(float(e2e_bytes.item()) / 2 / e2e_steps),
                "d2h_bytes_per_step": int(float(e2e_bytes.item()) / 2 / e2e_steps), "steps": e2e_steps,
                "includes": "slab upload, public-API driver loop (host dt each step), slab download"},
        # per step: prologue, first stage (behind its face-cache fill pass when
        # the cache is on), second stage and its epilogue (wavespeed and sums);
        # plus the final series prologue
        "gpu_launches": (4 if args.no_face_cache else 5) * args.steps + 1,
        "roofline": {"bound": "hbm", "peak": peak, "unit": "GB/s", "peak_source": peak_kind,
                     "note": "per-kernel roofline is reported by the N = 1 line"},
        "clocks": clocks.summary(),
    }


def run_ours(args, rank, world):
    import torch

    from sailfish_b200 import make_solver, pinned_empty

    torch.cuda.set_device(rank % max(torch.cuda.device_count(), 1))
    n = args.size
    setup, mesh, prim = initial_state(n, args.seed + rank)
    # the initial state in pinned host memory, as a caller that feeds the
    # device keeps it (filled here, before any timing): the e2e upload is then
    # one direct host-to-device copy
    pinned = pinned_empty(prim.shape)
    pinned[...] = prim
    prim = pinned
    physics = setup.physics
    physics["diagnostics"] = DIAGNOSTICS
    zones = n * n

    def fresh():
        tile = tuple(int(v) for v in args.tile.split(",")) if args.tile else None
        return make_solver("cbdiso_2d", physics,
                           dict(rk_order=2, plm_theta=THETA, precision=args.precision, tile=tile,
                                face_cache=not args.no_face_cache),
                           setup=setup, mesh=mesh, solution=prim)

    solver = fresh()

    # value: the device-resident driver loop (dt, stage times and the Kepler
    # orbit on the device, CUDA-graph replay of 16-step groups), state in HBM
    solver.run(max(args.warmup, 16), cfl=CFL)
    dist = world > 1
    if dist:
        import torch.distributed as tdist
        tdist.barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h2d0, d2h0 = solver.h2d_bytes, solver.d2h_bytes
    with ClockSampler(torch.cuda.current_device()) as clocks:
        clocks.load(lambda: (solver.run(16, cfl=CFL), torch.cuda.synchronize()),
                    group_max=(lambda n: _max_over_ranks(n, tdist)) if dist else None)
        if dist:
            tdist.barrier()
        torch.cuda.synchronize()
        start.record()
        rows = solver.run(args.steps, cfl=CFL)
        stop.record()
        torch.cuda.synchronize()
        clocks.stop()
    assert len(rows) == args.steps and all(np.isfinite(r[-1]) for r in rows)
    elapsed = start.elapsed_time(stop) * 1e-3
    if dist:
        t = torch.tensor([elapsed], device="cuda", dtype=torch.float64)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        elapsed = float(t.item())
        tdist.barrier()
    h2d = (solver.h2d_bytes - h2d0) / args.steps
    d2h = (solver.d2h_bytes - d2h0) / args.steps
    value = zones * args.steps * world / elapsed

    # end-to-end through the public API, from host data: upload the initial
    # state, run the steps, download the final state (amortised per step)
    # the same number of steps as the device-timed loop: a run's fixed costs
    # (state upload, solver set-up, state download) are spread as in `value`.
    # The phases are timed separately too (synchronised at their
    # boundaries), so that the fixed cost and the per-step cost are known
    # whatever the step count.
    e2e_steps = max(1, args.steps)

    def e2e_once():
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s2 = fresh()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(e2e_steps):
            dt = mesh.min_spacing() / s2.maximum_wavespeed() * CFL
            s2.advance(dt)
            s2.reductions()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        final = s2.solution
        t3 = time.perf_counter()
        io = ((s2.h2d_bytes + prim.nbytes) / e2e_steps, (s2.d2h_bytes + final.nbytes) / e2e_steps)
        del s2, final
        return (t0, t1, t2, t3), io

    # one untimed repetition (the process's first download pins host memory
    # for its result, about 0.2 s at 4096^2, which later downloads reuse),
    # then three (the host's load moves the set-up and copies): the median by
    # total time is reported, all three are listed
    e2e_once()
    reps = [e2e_once() for _ in range(3)]
    reps.sort(key=lambda r: r[0][3] - r[0][0])
    (t0, t1, t2, t3), (e2e_h2d, e2e_d2h) = reps[1]
    e2e_elapsed = t3 - t0
    if dist:
        t = torch.tensor([e2e_elapsed], device="cuda", dtype=torch.float64)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        e2e_elapsed = float(t.item())
    e2e_value = zones * e2e_steps * world / e2e_elapsed  # host-driven loop: one dt round trip per step
    e2e_phases = {"setup_and_upload_ms": (t1 - t0) * 1e3, "steps_ms": (t2 - t1) * 1e3,
                  "download_ms": (t3 - t2) * 1e3, "fixed_ms": (t1 - t0 + t3 - t2) * 1e3,
                  "per_step_ms": (t2 - t1) * 1e3 / e2e_steps,
                  "repetitions_ms": [round((r[0][3] - r[0][0]) * 1e3, 2) for r in reps]}
    e2e_phases.update(transfer_floor(prim.nbytes))
    e2e_phases.update(host_copy_times(prim.nbytes))

    kernel_s = stage_kernel_time(solver)
    peak, peak_kind = measured_peaks()
    achieved = BYTES_PER_ZONE_UPDATE / 2 * zones / kernel_s / 1e9
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": round(NCU_TRAFFIC_PER_ZONE_LAUNCH * zones),
                "traffic_source": "ncu at 2048^2 scaled by zones",
                "traffic_note": "above the algorithmic bytes by design: the face cache writes and reads 48 B per "
                                "zone and step to save FP64 work, and the epilogue reads the new state back "
                                "(24 B per zone and step); HBM is about 85 % idle",
                "peak_source": peak_kind,
                "kernel": "one RK stage: stage_kernel (mean of the stage-1 reader and the stage-2 writer) with the "
                          "stage-2 epilogue kernel", "kernel_ms": round(kernel_s * 1e3, 4),
                "bytes_per_launch": BYTES_PER_ZONE_UPDATE / 2 * zones}

    fp64 = fp64_roofline(FP64_INST_PER_ZONE_LAUNCH * zones, kernel_s)

    line = {
        "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(bench_config(n, args.precision), **({"parallelism": "replicas"} if world > 1 else {})),
        "timed": {"loop": "Solver.run: device-side dt / Kepler, CUDA graph of 16-step groups",
                  "face_cache": not args.no_face_cache},
        "e2e": dict({"value": e2e_value, "unit": "zone-updates/s", "h2d_bytes_per_step": int(e2e_h2d),
                     "d2h_bytes_per_step": int(e2e_d2h), "steps": e2e_steps,
                     "includes": "solver set-up and initial-state upload from pinned host memory, public-API "
                                 "driver loop, final-state download (into pinned memory the caller owns); one "
                                 "untimed repetition first"}, **e2e_phases),
        "step_io": {"h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "note": "value loop: stepper record in, time series out, per step"},
        # per step: prologue, first stage (behind its face-cache fill pass when
        # the cache is on), second stage and its epilogue (wavespeed and sums);
        # plus the final series prologue
        "gpu_launches": (4 if args.no_face_cache else 5) * args.steps + 1,
        "roofline": roofline,
        "roofline_fp64": fp64,
        "clocks": clocks.summary(),
    }
    return line


def transfer_floor(nbytes, repeats=3):
    """Pinned host <-> device copy times of one state's bytes on this box
    (best of `repeats`, CUDA events): the least that an upload plus a download
    of the state can cost."""
    import torch

    host = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    dev = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = {}
    for name, (dst, src) in (("h2d", (dev, host)), ("d2h", (host, dev))):
        ms = float("inf")
        for _ in range(repeats):
            start.record()
            dst.copy_(src, non_blocking=True)
            stop.record()
            torch.cuda.synchronize()
            ms = min(ms, start.elapsed_time(stop))
        best[name] = ms
    del host, dev
    return {"pinned_h2d_ms": best["h2d"], "pinned_d2h_ms": best["d2h"],
            "pinned_h2d_gbs": nbytes / best["h2d"] / 1e6, "pinned_d2h_gbs": nbytes / best["d2h"] / 1e6,
            "transfer_floor_ms": best["h2d"] + best["d2h"]}


def host_copy_times(nbytes, repeats=3):
    """The host side of the state copies for a caller whose arrays are
    ordinary (pageable) numpy memory, with the solver's pool threads and row
    blocks (sailfish_b200/_hostio.py): one state's bytes from a numpy array
    into pinned memory (a staged upload's copy), and from pinned memory into
    a new numpy array, its first touch included (a download past the pinned
    hand-out limit); best of `repeats`. Both are bound by host memory
    bandwidth, which the device copies share: a staged upload moves 3
    state-sizes through host memory (copy read and write, device-copy read),
    a pageable download 4 (device-copy write, the new array's zero-fill on
    first touch, copy read and write). `pageable_traffic_floor_ms` is those
    7 state-sizes at the bandwidth the upload's copy reaches. The e2e figure
    itself starts from pinned memory and downloads into pinned memory: one
    state-size each way, the device copies alone (`transfer_floor_ms`)."""
    import torch

    from sailfish_b200 import _hostio

    n = nbytes // 8
    src = np.ones(n)
    pinned = torch.empty(n, dtype=torch.float64).pin_memory()
    staged = pinned.numpy()
    blocks = _hostio._blocks(n, 2 * _hostio._threads())
    pool = _hostio._get_pool()

    def parallel_copy(dst, frm):
        for job in [pool.submit(np.copyto, dst[a:b], frm[a:b]) for a, b in blocks]:
            job.result()

    copy_in = copy_out = float("inf")
    for _ in range(repeats):
        t0 = time.perf_counter()
        parallel_copy(staged, src)
        t1 = time.perf_counter()
        out = np.empty(n)
        parallel_copy(out, staged)
        t2 = time.perf_counter()
        del out
        copy_in, copy_out = min(copy_in, (t1 - t0) * 1e3), min(copy_out, (t2 - t1) * 1e3)
    del pinned, staged, src
    host_gbs = 2 * nbytes / copy_in / 1e6
    return {"host_copy_in_ms": copy_in, "host_copy_out_ms": copy_out, "host_copy_gbs": host_gbs,
            "pageable_traffic_floor_ms": 7 * nbytes / host_gbs / 1e6}


def sizes_extra(args, sizes=(1024, 2048), steps=100):
    """The other two grid sizes of the plain-solver throughput configuration:
    the same device-resident loop as `value` (face cache on, EXACT), and the
    stage kernel's launch time against the HBM copy bandwidth."""
    import torch

    from sailfish_b200 import make_solver

    out = {}
    peak, peak_kind = measured_peaks()
    for n in sizes:
        setup, mesh, prim = initial_state(n, args.seed)
        physics = setup.physics
        physics["diagnostics"] = DIAGNOSTICS
        s = make_solver("cbdiso_2d", physics, dict(rk_order=2, plm_theta=THETA, precision=args.precision),
                        setup=setup, mesh=mesh, solution=prim)
        s.run(16, cfl=CFL)
        reps = []
        for _ in range(3):
            torch.cuda.synchronize()
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            s.run(steps, cfl=CFL)
            stop.record()
            torch.cuda.synchronize()
            reps.append(start.elapsed_time(stop) / steps)
        ms = float(np.median(reps))
        kernel_s = stage_kernel_time(s)
        achieved = BYTES_PER_ZONE_UPDATE / 2 * n * n / kernel_s / 1e9
        out[str(n)] = {"value": n * n / (ms * 1e-3), "unit": "zone-updates/s", "ms_per_step": ms,
                       "repetitions_ms_per_step": [round(v, 4) for v in reps],
                       "steps": steps, "kernel_ms": round(kernel_s * 1e3, 4),
                       "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                                    "frac": round(achieved / peak, 4), "peak_source": peak_kind}}
        del s
    out["note"] = ("same workload and loop as `value` at the configuration's other grid sizes; "
                   "the median of three repetitions")
    return out


def precision_extra(args, steps=50):
    """The same 4096^2 device-resident loop in the two other arithmetic
    modes of the stage kernel: FMA (the EXACT source with FMA contraction, as
    nvcc builds the reference's own GPU path) and FAST (reciprocal multiplies
    and rsqrt-based gravity, within about an ulp per operation). Both pass the
    1e-12-per-step / 1e-10-after-1000-steps parity tests; the headline value
    stays EXACT, which reproduces the reference's CPU results bit for bit."""
    import torch

    from sailfish_b200 import make_solver

    setup, mesh, prim = initial_state(args.size, args.seed)
    physics = setup.physics
    physics["diagnostics"] = DIAGNOSTICS
    out = {}
    for precision in ("fma", "fast"):
        s = make_solver("cbdiso_2d", physics, dict(rk_order=2, plm_theta=THETA, precision=precision),
                        setup=setup, mesh=mesh, solution=prim)
        s.run(16, cfl=CFL)
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        s.run(steps, cfl=CFL)
        stop.record()
        torch.cuda.synchronize()
        ms = start.elapsed_time(stop) / steps
        out[precision] = {"value": args.size ** 2 / (ms * 1e-3), "ms_per_step": ms}
        del s
    out["note"] = "same workload and loop as `value`, other arithmetic modes; not the headline"
    return out


def batched_extra(plain_value):
    """Many-disk throughput: 64 seeded disks of 128^2 to 1024^2 (about 19.8 M
    zones), each with its own dt, q, e, Mach and nu, advanced together by the
    persistent tile-queue kernel; 48 timed steps after 16."""
    import torch

    from sailfish_b200.batched import BatchedSolver, config2_disks

    b = BatchedSolver(config2_disks(64, seed=2024), diagnostics=DIAGNOSTICS)
    b.run(16)
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    b.run(48)
    stop.record()
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop) / 48
    value = b.total_zones / (ms * 1e-3)
    return {"workload": "64 disks 128^2..1024^2, own dt / q / e / Mach / nu, RK2 FP64", "zones": b.total_zones,
            "value": value, "unit": "zone-updates/s", "ms_per_step": ms,
            "vs_single_disk_value": value / plain_value}


def _event_ms(fn):
    """Device time of fn() on the current stream, CUDA events around it."""
    import torch

    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    fn()
    stop.record()
    torch.cuda.synchronize()
    return start.elapsed_time(stop)


def adjoint_extra(cases=((512, 400), (2048, 100))):
    """Forward + gradient of the time-averaged accretion rate over RK2 steps
    (dt frozen), per step, against a plain device step of the same grid, in
    both sweep forms: `checkpointed` keeps one state every 20 steps and
    recomputes each segment in the reverse sweep (the configured form), and
    `stored` keeps every stage state of the forward run. 512^2 x 400 steps is
    the configured size; 2048^2 (100 steps) is where the plain step is
    throughput-bound. Timed with CUDA events on the launching stream."""
    import torch

    from sailfish_b200.adjoint import AdjointRun, Params

    params = Params(0.5, 0.1, 1e-3, 10.0)
    out = {"workload": "q 0.5, e 0.1, RK2, d(mean accretion)/d(Sigma_0, q, e, nu, sink rate), checkpoint every 20",
           "timing": "CUDA events on the launching stream"}
    for n, steps in cases:
        block = {"steps": steps}
        plain = None
        for form, store in (("checkpointed", False), ("stored", True)):
            run = AdjointRun(resolution=n, steps=steps, checkpoint_every=20, store_states=store)
            prim = run.initial_state(seed=0)
            run.forward(prim, params, freeze=True, keep=True)
            run.gradient((1.0, 0.0))
            # warm-up with the frozen dt sequence (records this form's CUDA graphs)
            run.forward(prim, params, keep=True)
            run.gradient((1.0, 0.0))
            fwd = _event_ms(lambda: run.forward(prim, params, keep=True)) / steps
            adj = _event_ms(lambda: run.gradient((1.0, 0.0))) / steps
            if plain is None:
                solver = run._solver(params, prim)
                solver.run(16, cfl=run.cfl)
                plain = _event_ms(lambda: solver.run(steps, cfl=run.cfl)) / steps
                del solver
            block[form] = {"forward_ms_per_step": fwd, "gradient_ms_per_step": adj,
                           "forward_plus_gradient_vs_plain": (fwd + adj) / plain,
                           "stored_states": run._fwd["trajectory"] is not None}
            del run
            torch.cuda.empty_cache()
        block["plain_ms_per_step"] = plain
        out[str(n)] = block
    return out


def batched_adjoint_extra(plain_value):
    """32 disks (half 256^2, half 512^2; own q, e, nu), 200 steps, stored
    states: the whole batch's forward and adjoint captured as one CUDA graph
    (one branch per disk) and replayed, against the batched forward of the
    same disks (the persistent tile-queue kernel) and the plain single-grid
    throughput; CUDA events. The eager forward and gradient (disks over 8
    streams and host threads) are timed beside it for the breakdown."""
    import torch

    from sailfish_b200.adjoint import BatchedAdjoint, config4_disks
    from sailfish_b200.batched import BatchedSolver, Disk

    disks = config4_disks(32)
    steps = 200
    batch = BatchedAdjoint(disks, steps=steps, streams=8, store_states=True)
    batch.forward(freeze=True, keep=True)
    batch.gradient((1.0, 0.0))
    fwd_eager = _event_ms(lambda: batch.forward(keep=True))
    grad_eager = _event_ms(lambda: batch.gradient((1.0, 0.0)))
    batch.capture((1.0, 0.0))
    batch.replay()
    graph_ms = min(_event_ms(batch.replay) for _ in range(3))
    batch.results()
    batch.replay(gradient=False)
    graph_fwd_ms = min(_event_ms(lambda: batch.replay(gradient=False)) for _ in range(3))
    members = []
    for d, r, p in zip(disks, batch.runs, batch.prims):
        setup = r.setup(d.params)
        members.append(Disk(setup, setup.mesh(d.resolution), p))
    b = BatchedSolver(members, diagnostics=[dict(quantity="mdot", which_mass=1, accretion=True),
                                            dict(quantity="mdot", which_mass=2, accretion=True),
                                            dict(quantity="torque", which_mass="both", gravity=True)])
    b.run(16)
    fwd_batched = _event_ms(lambda: b.run(steps))
    zones = sum(d.resolution ** 2 for d in disks)
    value = zones * steps / (graph_ms * 1e-3)
    del batch, b
    torch.cuda.empty_cache()
    return {"workload": "32 disks (16 x 256^2, 16 x 512^2), own q / e / nu, 200 RK2 steps, gradients of the "
                        "mean accretion rate, stored states",
            "forward_plus_gradient_graph_ms": graph_ms, "forward_graph_ms": graph_fwd_ms,
            "batched_forward_ms": fwd_batched,
            "forward_plus_gradient_vs_batched_forward": graph_ms / fwd_batched,
            "gradient_vs_batched_forward": (graph_ms - graph_fwd_ms) / fwd_batched,
            "eager_forward_ms": fwd_eager, "eager_gradient_ms": grad_eager,
            "zone_updates_per_s": value, "vs_plain_single_grid": value / plain_value,
            "timing": "CUDA events; forward + gradient as one captured graph with a branch per disk"}


GAM_SIZE = 2048
GAM_BYTES_PER_ZONE_STEP = 160  # stage 1: read 32 B + write 32 B; stage 2: read 2 x 32 B + write 32 B


def gamma_law_extra(steps=50, warmup=5):
    """The gamma-law solver (cbdgam_2d): a 2048^2 gamma-law circumbinary disk
    (alpha 0.1, buffer, constant softening, torque-free sinks, CFL 0.1), the
    reference's driver loop through the public API (dt from the wavespeed
    maximum every step), timed with CUDA events after warm-up; the stage
    kernel alone for its roofline; the reference's own gamma-law CPU kernels
    on a 512^2 sample beside it."""
    import ctypes

    import torch

    from sailfish_b200 import _capi, make_solver

    setup = _gamma_setup()
    mesh = setup.mesh(GAM_SIZE)
    s = make_solver("cbdgam_2d", setup.physics, {}, setup=setup, mesh=mesh)
    zones = GAM_SIZE * GAM_SIZE
    for _ in range(warmup):
        s.advance(mesh.min_spacing() / s.maximum_wavespeed() * 0.1)
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(steps):
        s.advance(mesh.min_spacing() / s.maximum_wavespeed() * 0.1)
    stop.record()
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop) / steps

    # the second-stage kernel alone (reads two states, writes one)
    lib, g = s._lib, s._grid
    stage = s._stage(s.time, 0.5, mesh.min_spacing() / s.maximum_wavespeed() * 0.1)
    out = torch.empty_like(s._buf[0])
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def launch():
        _capi.check(lib.cbdgam_b200_advance_stage(ctypes.byref(g), ctypes.byref(stage), s._ptr(s._buf[0]),
                                                  s._ptr(s._buf[1]), s._ptr(out), None, stream), "stage")

    for _ in range(3):
        launch()
    torch.cuda.synchronize()
    start.record()
    for _ in range(20):
        launch()
    stop.record()
    torch.cuda.synchronize()
    kernel_s = start.elapsed_time(stop) * 1e-3 / 20
    peak, peak_kind = measured_peaks()
    achieved = 96.0 * zones / kernel_s / 1e9
    line = {"workload": f"cbdgam_2d gamma-law circumbinary disk {GAM_SIZE}x{GAM_SIZE} FP64 RK2 theta 1.5 CFL 0.1, "
                        "alpha 0.1, buffer on", "zones": zones, "value": zones / (ms * 1e-3),
            "unit": "zone-updates/s", "ms_per_step": ms, "steps": steps, "warmup": warmup,
            "timed": "Solver.advance + maximum_wavespeed per step (one 8-byte read back), CUDA events",
            "roofline": {"bound": "fp64 issue (HBM shown for reference)", "kernel": "gam::stage_kernel (RK stage 2)",
                         "kernel_ms": round(kernel_s * 1e3, 4), "bytes_per_launch": 96 * zones,
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind},
            "roofline_fp64": fp64_roofline(GAM_FP64_INST_PER_ZONE_LAUNCH * zones, kernel_s)}
    del s, out
    try:
        line["cpu_baseline"] = gamma_cpu_baseline()
    except (FileNotFoundError, OSError) as e:
        line["cpu_baseline"] = {"unavailable": str(e)}
    return line


def _gamma_setup():
    from sailfish_b200.setups import CircumbinaryDisk

    return CircumbinaryDisk(eos="gamma-law")


def gamma_cpu_baseline(n=512, steps=3):
    """The reference's gamma-law kernels (oracle/_ref, OpenMP) driven as its
    solver adapter does (oracle/host_gam.py), on n^2 zones."""
    from oracle import host_gam as og
    from sailfish_b200.cbdgam_2d import initial_condition

    setup = _gamma_setup()
    mesh = setup.mesh(n)
    prim = initial_condition(setup, mesh, 0.0)
    onset = [0.0] * 4
    setup.primitive(0.0, [mesh.x1 - 0.1, 0.0], onset)
    from oracle import host as oh

    cfg = og.GamConfig(mesh.x0, mesh.x1, mesh.y0, mesh.y1, n, n, alpha=setup.alpha, buffer_is_enabled=True,
                       buffer_surface_density=onset[0], buffer_surface_pressure=onset[3],
                       masses=oh.binary_masses(1.0, 1.0, 1.0, 0.0, 0.05, "torque_free", 10.0, 0.05))
    kernels = og.GamKernels("ref", 1.5, threads="omp")
    solver = og.GamOracleSolver(cfg, prim, 0.0, kernels)
    solver.advance(og.driver_dt(solver, 0.1))
    t0 = time.perf_counter()
    for _ in range(steps):
        solver.advance(og.driver_dt(solver, 0.1))
    el = time.perf_counter() - t0
    return {"value": n * n * steps / el, "unit": "zone-updates/s",
            "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())), "kind": "reference",
            "sample": f"{steps} driver steps at {n}^2 (advance + wavespeed)"}


# ---------------------------------------------------------------------------
# the reference's CPU kernels (oracle/_ref) and the oracle port
# ---------------------------------------------------------------------------


def cpu_config(n):
    from oracle import host as oh

    return oh.Config(-8.0, 8.0, -8.0, 8.0, n, n, eos_type=2, mach_number=10.0, nu=1e-3, buffer_is_enabled=True,
                     buffer_driving_rate=100.0, buffer_onset_width=1.0, buffer_surface_density=1.0,
                     masses=oh.binary_masses(1.0, 1.0, 1.0, 0.0, 0.05, "torque_free", 10.0, 0.05),
                     plm_theta=THETA)


def cpu_kernels():
    from oracle import host as oh

    try:
        return oh.Kernels("ref", THETA, threads="omp"), "reference"
    except (FileNotFoundError, OSError):
        return oh.Kernels("oracle", THETA), "port"


def time_cpu(n, steps, warmup, seed):
    """Driver loop of the CPU kernels; returns zone-updates/s and the kind."""
    from oracle import host as oh

    _, _, prim = initial_state(n, seed)
    kernels, kind = cpu_kernels()
    solver = oh.OracleSolver(cpu_config(n), prim, 0.0, kernels)
    diags = [d for d in DIAGNOSTICS]
    for _ in range(warmup):
        solver.advance(oh.driver_dt(solver, CFL))
        solver.reductions(diags)
    t0 = time.perf_counter()
    for _ in range(steps):
        solver.advance(oh.driver_dt(solver, CFL))
        solver.reductions(diags)
    el = time.perf_counter() - t0
    return n * n * steps / el, kind, el


def run_reference(args, rank, world):
    if rank != 0:
        return None
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    n = args.size
    # each step is a full 4096^2 driver iteration; the count is capped so the
    # whole run stays within a few minutes
    per_step = 6.0 * (n / 4096.0) ** 2 * 8 / max(1, os.cpu_count())
    steps = max(1, min(args.steps, int(120.0 / max(per_step, 1e-3))))
    # the requested warm-up steps, up to three (about 1.2 s each at 4096^2)
    warmup = min(args.warmup, 3)
    value, kind, el = time_cpu(n, steps, warmup, args.seed)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))
    return {
        "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s", "n_gpus": world, "steps": steps,
        "warmup": warmup, "ms_per_step": el / steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": bench_config(n, "exact"),
        "cpu_baseline": {"value": value, "unit": "zone-updates/s", "cores": cores, "kind": kind,
                         "sample": f"{steps} full driver steps at {n}^2 (advance + wavespeed + reductions)"},
        "e2e": {"value": value, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    slabs = args.mode == "slab" or (args.mode == "auto" and world > 1)
    group = args.impl == "ours" and (world > 1 or slabs)
    if group:
        import datetime
        import socket

        import torch
        import torch.distributed as tdist

        if world == 1 and "MASTER_PORT" not in os.environ:
            with socket.socket() as sk:
                sk.bind(("127.0.0.1", 0))
                os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(sk.getsockname()[1]), RANK="0",
                                  WORLD_SIZE="1")
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    elif slabs:
        line = run_slabs(args, rank, world)
    else:
        line = run_ours(args, rank, world)
        if world == 1 and not args.no_extras:
            line["sizes"] = sizes_extra(args)
            line["precision_modes"] = precision_extra(args)
            line["batched"] = batched_extra(line["value"])
            line["adjoint"] = adjoint_extra()
            line["adjoint_batched"] = batched_adjoint_extra(line["value"])
            line["gamma_law"] = gamma_law_extra()
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            n = args.size
            v, kind, el = time_cpu(n, 2 if n >= 2048 else 5, 1, args.seed)
            line["cpu_baseline"] = {"value": v, "unit": "zone-updates/s",
                                    "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())), "kind": kind,
                                    "sample": f"{2 if n >= 2048 else 5} driver steps at {n}^2"}
    if group:
        import torch.distributed as tdist

        tdist.destroy_process_group()
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
