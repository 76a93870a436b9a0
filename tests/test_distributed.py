"""
The multi-GPU solver's host logic as gloo ranks on CPU (world sizes 2 and 3),
with the oracle patch engine in place of the B200 kernels: patch split,
guard-row exchange between stages, wavespeed all-reduce and patch-ordered
sums. Checked against the same patches advanced serially in one process
(the reference's multi-patch scheme: bit for bit) and the single-grid
oracle.
"""

import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import host as oh
from sailfish_b200.distributed import subdivide

DIAGS = [dict(quantity="time"), dict(quantity="mdot", which_mass=1, accretion=True),
         dict(quantity="mdot", which_mass=2, accretion=True), dict(quantity="torque", which_mass="both", gravity=True)]


def _problem(ni, nj, seed):
    from sailfish_b200.cbdiso_2d import initial_condition
    from sailfish_b200.mesh import PlanarCartesian2DMesh
    from sailfish_b200.setups import CircumbinaryDisk

    setup = CircumbinaryDisk(domain_radius=6.0, mass_ratio=0.6, eccentricity=0.2, nu=0.002)
    mesh = PlanarCartesian2DMesh(-6.0, -6.0, 6.0, 6.0, ni, nj)
    prim = initial_condition(setup, mesh, 0.0)
    prim[..., 0] += 1e-3 * np.random.default_rng(seed).uniform(-1.0, 1.0, size=(ni, nj))
    physics = setup.physics
    physics["diagnostics"] = DIAGS
    return setup, mesh, prim, physics


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, ni, nj, rk, steps, out_dir):
    import torch.distributed as dist

    from patch_engine import OraclePatch
    from sailfish_b200.distributed import DistributedSolver

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        setup, mesh, prim, physics = _problem(ni, nj, 3)
        s = DistributedSolver(setup=setup, mesh=mesh, solution=prim, physics=physics,
                              options=dict(rk_order=rk, plm_theta=1.8), engine=OraclePatch)
        dts, series, speeds = [], [], []
        for _ in range(steps):
            ws = s.maximum_wavespeed()
            dt = mesh.min_spacing() / ws * 0.3
            s.advance(dt)
            dts.append(dt)
            speeds.append(ws)
            series.append(s.reductions())
        sol = s.solution
        if rank == 0:
            np.savez(os.path.join(out_dir, "out.npz"), solution=sol, dts=np.array(dts), speeds=np.array(speeds),
                     series=np.array(series, dtype=complex), time=s.time)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world, ni, nj, rk", [(2, 20, 18, 2), (3, 17, 12, 3)])
def test_patch_ranks_match_serial_patches_and_one_grid(world, ni, nj, rk):
    from patch_engine import SerialPatches

    steps = 4
    with tempfile.TemporaryDirectory() as out:
        mp.spawn(_rank, args=(world, _free_port(), ni, nj, rk, steps, out), nprocs=world, join=True)
        got = dict(np.load(os.path.join(out, "out.npz")))
    setup, mesh, prim, physics = _problem(ni, nj, 3)

    serial = SerialPatches(setup, mesh, prim, physics, dict(rk_order=rk, plm_theta=1.8), world)
    for n in range(steps):
        ws = serial.maximum_wavespeed()
        assert ws == got["speeds"][n]
        dt = mesh.min_spacing() / ws * 0.3
        assert dt == got["dts"][n]
        serial.advance(dt)
    np.testing.assert_array_equal(got["solution"], serial.solution)

    # the whole grid as one patch: the same states up to the patches' edge rounding
    cfg = serial.p[0].o.cfg._replace(x0=mesh.x0, x1=mesh.x1, ni=ni)
    one = oh.OracleSolver(cfg, prim)
    for dt in got["dts"]:
        one.advance(dt)
    np.testing.assert_allclose(got["solution"], one.solution, rtol=1e-12, atol=1e-14)
    want = one.reductions(DIAGS, num_patches=world)
    scale = one.reductions(DIAGS, num_patches=world, absolute=True)
    for k in range(1, len(DIAGS)):
        assert abs(got["series"][-1][k] - want[k]) <= 1e-12 * abs(scale[k]) + 1e-300, (k, got["series"][-1][k], want[k])
    assert got["time"] == one.time


def test_subdivide_matches_the_reference_partition():
    """subdivide.py:35-60: the first (n mod parts) patches one row longer."""
    assert list(subdivide(10, 3)) == [(0, 4), (4, 7), (7, 10)]
    assert list(subdivide(4096, 8))[-1] == (3584, 4096)
    assert sum(b - a for a, b in subdivide(17, 5)) == 17


def test_thread_ranks_match_gloo_ranks():
    """The in-process thread ranks (used by the single-GPU test of the real
    kernels) give the same run as separate gloo processes."""
    from patch_engine import OraclePatch, SerialPatches
    from sailfish_b200.distributed import DistributedSolver
    from thread_comm import ThreadComm

    ni, nj, world = 15, 11, 3
    setup, mesh, prim, physics = _problem(ni, nj, 5)
    comm = ThreadComm(world)

    def rank(r):
        s = DistributedSolver(setup=setup, mesh=mesh, solution=prim, physics=physics,
                              options=dict(rk_order=2, plm_theta=1.8), engine=OraclePatch, comm=comm)
        for _ in range(3):
            s.advance(mesh.min_spacing() / s.maximum_wavespeed() * 0.3)
        return s.solution, s.reductions()

    out = comm.run(rank)
    serial = SerialPatches(setup, mesh, prim, physics, dict(rk_order=2, plm_theta=1.8), world)
    for _ in range(3):
        serial.advance(mesh.min_spacing() / serial.maximum_wavespeed() * 0.3)
    for sol, red in out:
        np.testing.assert_array_equal(sol, serial.solution)
        assert red == out[0][1]


# ---------------------------------------------------------------------------
# the gamma-law solver's patches, against the reference's own two-patch run
# (tests/golden/gam_n48_cool_p2.npz: 48^2, cooling, eccentric q = 0.5 binary)
# ---------------------------------------------------------------------------


def _gam_problem():
    from cases import diagnostics, gam_initial_state, load
    from sailfish_b200.mesh import PlanarCartesian2DMesh
    from sailfish_b200.setups import CircumbinaryDisk

    d = load("gam_n48_cool_p2")
    meta = d["meta"]
    x0, y0, x1, y1, ni, nj = meta["mesh"]
    setup = CircumbinaryDisk(**meta["params"])
    mesh = PlanarCartesian2DMesh(x0, y0, x1, y1, int(ni), int(nj))
    physics = setup.physics
    physics["diagnostics"] = diagnostics(meta)
    return d, setup, mesh, gam_initial_state(d), physics


def _gam_rank(rank, world, port, out_dir):
    import torch.distributed as dist

    from patch_engine import GamOraclePatch
    from sailfish_b200.distributed import DistributedSolver

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        d, setup, mesh, prim, physics = _gam_problem()
        s = DistributedSolver(setup=setup, mesh=mesh, solution=prim, physics=physics, engine=GamOraclePatch)
        dts, series = [], []
        for _ in range(d["meta"]["steps"]):
            dt = mesh.min_spacing() / s.maximum_wavespeed() * d["meta"]["cfl"]
            s.advance(dt)
            dts.append(dt)
            series.append(s.reductions())
        sol = s.solution
        if rank == 0:
            np.savez(os.path.join(out_dir, "out.npz"), solution=sol, dts=np.array(dts),
                     series=np.array(series, dtype=complex), time=s.time)
    finally:
        dist.destroy_process_group()


def test_gamma_patch_ranks_reproduce_the_reference_two_patch_run():
    """Two gloo ranks, one gamma-law patch each (oracle kernels), against
    the reference solver run with num_patches=2: dts and states bit for
    bit, the time series to rounding (the sums are regrouped per patch)."""
    with tempfile.TemporaryDirectory() as out:
        mp.spawn(_gam_rank, args=(2, _free_port(), out), nprocs=2, join=True)
        got = dict(np.load(os.path.join(out, "out.npz")))
    d = _gam_problem()[0]
    assert d["meta"]["patches"] == 2
    np.testing.assert_array_equal(got["dts"], d["dts"])
    np.testing.assert_array_equal(got["solution"], d["last"])
    assert float(got["time"]) == float(d["time"])
    want = d["series"]
    scale = np.maximum(np.abs(want).max(axis=0), 1e-300)
    assert (np.abs(got["series"] - want).max(axis=0) / scale).max() <= 1e-12


def test_default_engine_follows_the_equation_of_state():
    """A gamma-law physics dict makes the distributed solver's patches
    cbdgam_2d patches; it is checked by the engine it picks, without a GPU."""
    from sailfish_b200.distributed import DistributedSolver
    from thread_comm import ThreadComm

    d, setup, mesh, prim, physics = _gam_problem()
    picked = []

    class Probe:
        def __init__(self, **kwargs):
            raise RuntimeError("stop")

    import sailfish_b200.cbdgam_2d as gam

    real = gam.Solver
    try:
        gam.Solver = lambda **kw: picked.append("cbdgam_2d") or Probe(**kw)
        comm = ThreadComm(1)
        with pytest.raises(RuntimeError, match="stop"):
            comm.run(lambda r: DistributedSolver(setup=setup, mesh=mesh, solution=prim, physics=physics,
                                                 comm=comm))
    finally:
        gam.Solver = real
    assert picked == ["cbdgam_2d"]
