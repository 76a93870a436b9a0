"""
Tile-shape autotuner for the stage kernels.

For a grid size it times candidate tile shapes on a synthetic circumbinary
disk of that size (the config-0 physics) with CUDA events and keeps the
fastest. Results are cached in a JSON file keyed by GPU name, precision,
kernel kind and size, by default ~/.cache/sailfish_b200/tiles.json
(override with SAILFISH_B200_TILE_CACHE).

  * batched kernel: (strip_width, rows) per disk size, measured through a
    one-disk BatchedSolver (the exact code path of a batch);
  * single-grid kernel: (columns, rows, occupancy) for Solver's `tile` option.
"""

from __future__ import annotations

import json
import os

BATCHED_CANDIDATES = [(w, r) for w in (128, 64) for r in (8, 16, 32, 64)]
PLAIN_CANDIDATES = [(128, r, 6) for r in (8, 16, 32, 64)] + [(128, r, 5) for r in (16, 32)] + \
    [(64, r, 12) for r in (16, 32)]


def cache_path():
    return os.environ.get("SAILFISH_B200_TILE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "sailfish_b200", "tiles.json"))


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(cache):
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path + ".tmp", "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(path + ".tmp", path)
    except OSError:
        pass


def _key(kind, precision, ni, nj):
    import torch

    return f"{torch.cuda.get_device_name()}|{precision}|{kind}|{ni}x{nj}"


def _disk(ni, nj, seed=7):
    import numpy as np

    from .cbdiso_2d import initial_condition
    from .mesh import PlanarCartesian2DMesh
    from .setups import CircumbinaryDisk

    setup = CircumbinaryDisk(domain_radius=8.0, nu=1e-3)
    mesh = PlanarCartesian2DMesh(-8.0, -8.0, 8.0, 8.0, ni, nj)
    prim = initial_condition(setup, mesh, 0.0)
    prim[..., 0] += 1e-3 * np.random.default_rng(seed).uniform(-1.0, 1.0, size=(ni, nj))
    return setup, mesh, prim


def _time(fn, repeats):
    import torch

    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(repeats):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / repeats


def tune_batched(ni, nj, precision="exact", candidates=BATCHED_CANDIDATES, steps=4, fill_zones=1 << 23):
    """
    Fastest (strip_width, rows) of the batched kernel for ni x nj disks, timed
    in a batch of copies holding about `fill_zones` zones, so the GPU is as
    full as in a real batch and the tile's own cost decides.
    """
    from .batched import BatchedSolver, Disk

    setup, mesh, prim = _disk(ni, nj)
    disk = Disk(setup, mesh, prim)
    copies = max(1, fill_zones // (ni * nj))
    best, best_ms = None, float("inf")
    for width, rows in candidates:
        if width > 64 and nj <= 64:
            continue
        b = BatchedSolver([disk] * copies, precision=precision, tiles={(ni, nj): (width, rows)})
        ms = _time(lambda: b.run(steps, graph=False), 2)
        del b
        if ms < best_ms:
            best, best_ms = (width, rows), ms
    return best


def tune_plain(ni, nj, precision="exact", candidates=PLAIN_CANDIDATES, steps=4):
    """Fastest (columns, rows, occupancy) of the single-grid stage kernel."""
    from . import make_solver

    setup, mesh, prim = _disk(ni, nj)
    best, best_ms = None, float("inf")
    for tile in candidates:
        s = make_solver("cbdiso_2d", setup.physics, dict(precision=precision, tile=tile, plm_theta=1.5),
                        setup=setup, mesh=mesh, solution=prim)
        dt = mesh.min_spacing() / s.maximum_wavespeed() * 0.3

        def go():
            for _ in range(steps):
                s.advance(dt)

        ms = _time(go, 2)
        del s
        if ms < best_ms:
            best, best_ms = tuple(tile), ms
    return best


def tuned_tiles(sizes, precision="exact"):
    """{(ni, nj): (strip_width, rows)} for the batched kernel, from the cache or measured."""
    cache = _load()
    out = {}
    dirty = False
    for ni, nj in sizes:
        key = _key("batched", precision, ni, nj)
        if key not in cache:
            cache[key] = list(tune_batched(ni, nj, precision))
            dirty = True
        out[(ni, nj)] = tuple(cache[key])
    if dirty:
        _store(cache)
    return out


def tuned_plain_tile(ni, nj, precision="exact"):
    """(columns, rows, occupancy) for Solver's `tile` option, cached."""
    cache = _load()
    key = _key("plain", precision, ni, nj)
    if key not in cache:
        cache[key] = list(tune_plain(ni, nj, precision))
        _store(cache)
    return tuple(cache[key])
