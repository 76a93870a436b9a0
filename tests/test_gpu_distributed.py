"""
The multi-GPU solver with its real patch kernels, on the one GPU of this
test: ranks are host threads (thread_comm.ThreadComm), each advancing its
patch with the B200 stage kernel and exchanging guard rows through host-side
copies between stages; compared with the same patches advanced serially on
the oracle (the reference's multi-patch scheme). One NCCL rank runs the
torch.distributed path itself.
"""

import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from patch_engine import SerialPatches  # noqa: E402
from sailfish_b200.distributed import DistributedSolver  # noqa: E402
from test_distributed import DIAGS, _problem  # noqa: E402
from thread_comm import ThreadComm  # noqa: E402


@pytest.mark.parametrize("world, ni, nj, rk", [(2, 40, 36, 2), (3, 33, 24, 2), (4, 29, 20, 3)])
def test_patch_kernels_match_serial_patches(world, ni, nj, rk):
    setup, mesh, prim, physics = _problem(ni, nj, 7)
    opts = dict(rk_order=rk, plm_theta=1.8, precision="exact")
    comm = ThreadComm(world)
    steps = 5

    def rank(r):
        torch.cuda.set_device(0)
        s = DistributedSolver(setup=setup, mesh=mesh, solution=prim, physics=physics, options=opts, comm=comm)
        speeds, series = [], []
        for _ in range(steps):
            ws = s.maximum_wavespeed()
            s.advance(mesh.min_spacing() / ws * 0.3)
            speeds.append(ws)
            series.append(s.reductions())
        return s.solution, speeds, series

    out = comm.run(rank)
    # every rank saw the same all-reduced wavespeeds, sums and whole state
    for sol, speeds, series in out[1:]:
        np.testing.assert_array_equal(sol, out[0][0])
        assert speeds == out[0][1] and series == out[0][2]
    # the serial oracle patches, driven by the same dt sequence: EXACT
    # precision agrees with the CPU build to an ulp where CUDA's pow / exp
    # round differently from glibc's
    serial = SerialPatches(setup, mesh, prim, physics, opts, world)
    for n in range(steps):
        ws = serial.maximum_wavespeed()
        assert abs(out[0][1][n] - ws) <= 1e-14 * ws, (n, ws, out[0][1][n])
        serial.advance(mesh.min_spacing() / out[0][1][n] * 0.3)
    want = serial.solution
    err = np.abs(out[0][0] - want).max(axis=(0, 1)) / np.abs(want).max(axis=(0, 1))
    assert err.max() <= 1e-13, err


def test_device_resident_run_matches_advance():
    """DistributedSolver.run (device dt, Kepler orbit, all-reduced wavespeed)
    equals the host-driven advance loop on the same thread ranks."""
    setup, mesh, prim, physics = _problem(36, 30, 8)
    opts = dict(rk_order=2, plm_theta=1.5, precision="exact")

    def go(use_run):
        comm = ThreadComm(2)

        def rank(r):
            torch.cuda.set_device(0)
            s = DistributedSolver(setup=setup, mesh=mesh, solution=prim, physics=physics, options=opts, comm=comm)
            if use_run:
                rows = s.run(6, cfl=0.3)
                return s.solution, [r[-1] for r in rows], rows[-1][:-1]
            dts = []
            for _ in range(6):
                dts.append(mesh.min_spacing() / s.maximum_wavespeed() * 0.3)
                s.advance(dts[-1])
            return s.solution, dts, s.reductions()

        return comm.run(rank)

    a, b = go(True), go(False)
    for (sa, da, ra), (sb, db, rb) in zip(a, b):
        np.testing.assert_array_equal(sa, sb)
        assert da == db
        np.testing.assert_allclose(np.array(ra[1:], dtype=complex), np.array(rb[1:], dtype=complex), rtol=1e-12)


def test_one_nccl_rank():
    import torch.distributed as dist

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        setup, mesh, prim, physics = _problem(32, 32, 9)
        s = DistributedSolver(setup=setup, mesh=mesh, solution=prim, physics=physics,
                              options=dict(rk_order=2, plm_theta=1.8))
        rows = s.run(4, cfl=0.3)
        assert len(rows) == 4 and s.solution.shape == (32, 32, 3)
        serial = SerialPatches(setup, mesh, prim, physics, dict(rk_order=2, plm_theta=1.8), 1)
        for r in rows:
            serial.advance(r[-1])
        want = serial.solution
        err = np.abs(s.solution - want).max(axis=(0, 1)) / np.abs(want).max(axis=(0, 1))
        assert err.max() <= 1e-13, err
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gamma_patch_kernels_against_the_reference_two_patch_run(world):
    """The gamma-law solver as thread ranks with its real stage kernels on
    the reference's two-patch fixture (48^2, cooling): with two ranks the
    patches are the reference's own, with three they differ only in the
    patches' edge rounding; dts to 1e-13, states to 1e-12 of each field's
    maximum, every rank's view identical."""
    from test_distributed import _gam_problem

    d, setup, mesh, prim, physics = _gam_problem()
    comm = ThreadComm(world)
    meta = d["meta"]

    def rank(r):
        torch.cuda.set_device(0)
        s = DistributedSolver(setup=setup, mesh=mesh, solution=prim, physics=physics, comm=comm)
        dts, series = [], []
        for _ in range(meta["steps"]):
            dt = mesh.min_spacing() / s.maximum_wavespeed() * meta["cfl"]
            s.advance(dt)
            dts.append(dt)
            series.append(s.reductions())
        return s.solution, dts, series, type(s.local).__module__

    out = comm.run(rank)
    for sol, dts, series, module in out:
        assert module == "sailfish_b200.cbdgam_2d"
        np.testing.assert_array_equal(sol, out[0][0])
        assert dts == out[0][1] and series == out[0][2]
    sol, dts = out[0][0], np.array(out[0][1])
    np.testing.assert_allclose(dts, d["dts"], rtol=1e-13, atol=0)
    want = d["last"]
    err = np.abs(sol - want).max(axis=(0, 1)) / np.abs(want).max(axis=(0, 1))
    assert err.max() <= 1e-12, err
