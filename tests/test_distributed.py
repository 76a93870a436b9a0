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
