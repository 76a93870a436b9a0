"""
Batched many-disk stepping: one persistent launch per RK stage over every
disk's tiles. Each disk must match the same disk run alone (bit for bit in
state; reductions equal with the same tile shape), with its own dt sequence.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sailfish_b200 import make_solver  # noqa: E402
from sailfish_b200.batched import BatchedSolver, Disk, config2_disks  # noqa: E402

DIAGS = [dict(quantity="time"), dict(quantity="mdot", which_mass=1, accretion=True),
         dict(quantity="mdot", which_mass=2, accretion=True),
         dict(quantity="torque", which_mass="both", gravity=True)]


def _alone(disk, steps, tile):
    physics = disk.setup.physics
    physics["diagnostics"] = DIAGS
    s = make_solver("cbdiso_2d", physics, dict(rk_order=2, plm_theta=1.5, tile=tile), setup=disk.setup,
                    mesh=disk.mesh, solution=disk.solution)
    rows = s.run(steps, cfl=0.3, graph=False)
    return s, rows


@pytest.mark.parametrize("graph", [False, True])
def test_batched_disks_match_single_disk_runs(graph):
    disks = config2_disks(num=6, seed=11, sizes=(64, 96, 128, 200))
    tiles = {(n, n): (128 if n > 96 else 64, 16) for n in (64, 96, 128, 200)}
    b = BatchedSolver(disks, diagnostics=DIAGS, tiles=tiles)
    series = b.run(10, cfl=0.3, graph=graph, steps_per_graph=5)
    for i, d in enumerate(disks):
        n = d.mesh.shape[0]
        w, r = tiles[(n, n)]
        s, rows = _alone(d, 10, (w, r, 6 if w == 128 else 12))
        assert np.array_equal(b.solution(i), s.solution), f"disk {i} ({n}^2)"
        assert np.array_equal(np.array(series[i], dtype=complex), np.array(rows, dtype=complex)), f"disk {i}"
        assert b.times[i] == s.time


def test_batched_each_disk_has_its_own_time_step():
    disks = config2_disks(num=4, seed=3, sizes=(64, 128))
    b = BatchedSolver(disks, diagnostics=DIAGS)
    series = b.run(3, cfl=0.3)
    dts = [row[-1] for rows in series for row in rows[:1]]
    assert len(set(dts)) > 1


def test_batched_tiles_from_autotuner(tmp_path, monkeypatch):
    monkeypatch.setenv("SAILFISH_B200_TILE_CACHE", str(tmp_path / "tiles.json"))
    from sailfish_b200.autotune import tuned_tiles

    t = tuned_tiles([(96, 96)], "exact")
    assert (96, 96) in t and t[(96, 96)][0] in (64, 128)
    assert (tmp_path / "tiles.json").exists()
    assert tuned_tiles([(96, 96)], "exact") == t  # served from the cache


def test_batched_face_cache_is_bit_identical():
    disks = config2_disks(num=5, seed=7, sizes=(64, 96, 128))
    on = BatchedSolver(disks, diagnostics=DIAGS)
    off = BatchedSolver(disks, diagnostics=DIAGS, options=dict(face_cache=False))
    assert on._fcache is not None and off._fcache is None
    a = on.run(12, cfl=0.3, graph=True, steps_per_graph=4)
    b = off.run(12, cfl=0.3, graph=True, steps_per_graph=4)
    assert a == b
    for i in range(len(disks)):
        assert np.array_equal(on.solution(i), off.solution(i))
    torch.cuda.synchronize()
    assert float(on._fcache[0]) == 20261204.5  # the first disk's key was written
