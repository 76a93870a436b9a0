"""
Whole-state copies between host numpy arrays and device tensors.

A state at 4096^2 is 403 MB. Copied directly between pageable numpy memory
and the device, it moves at about 2-10 GB/s: the driver stages pageable
copies through its own buffer, and a new numpy array's pages are first
touched (faulted in and zeroed) by the single copying thread. These helpers
instead go through one pinned staging buffer kept for the process (the
device copy then runs at PCIe speed) and copy between it and the numpy array
with several host threads (numpy releases the GIL while copying), so the
page faults and the memcpy run in parallel, block by block behind the device
copies. Measured on the B200 host at 4096^2 before the pipelining: download
186 -> 21 ms, upload 37 -> 13 ms.

The staging buffer is allocated on first use (pinning is itself slow: about
0.2 s for 403 MB) and grows to the largest state copied; `release_staging()`
frees it. Copies are serialised by a lock, so threads may share it.
"""

from __future__ import annotations

import os
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

SMALL = 8 << 20  # below this many bytes a plain copy is as fast
_lock = threading.Lock()
_staging = None
_pool = None


def _threads():
    # the copies into a new array are bound by its page faults, which scale
    # with the threads taking them
    return max(1, min(16, os.cpu_count() or 1))


def _get_pool():
    global _pool
    if _pool is None:
        _pool = ThreadPoolExecutor(_threads(), thread_name_prefix="sailfish_b200_hostio")
    return _pool


def _staging_view(nbytes, shape):
    """A pinned float64 tensor of `shape` over the process's staging buffer."""
    import torch

    global _staging
    if _staging is None or _staging.numel() < nbytes:
        _staging = None
        size = max(nbytes, 64 << 20)
        _staging = torch.empty(size, dtype=torch.uint8, pin_memory=True)
    return _staging[:nbytes].view(torch.float64).view(shape)


def release_staging():
    """Free the pinned staging buffer (it is allocated again when needed)."""
    global _staging
    with _lock:
        _staging = None


def _blocks(n, k):
    k = max(1, min(k, n))
    return [(a * n // k, (a + 1) * n // k) for a in range(k)]


def download(tensor):
    """A new numpy array equal to a float64 device tensor (any strides).

    Pipelined in row blocks: each block's device-to-pinned copy is followed,
    as soon as it has landed, by its copy into the numpy array on a pool
    thread, while the next blocks are still in flight."""
    import torch

    nbytes = tensor.numel() * 8
    if nbytes < SMALL or tensor.dim() == 0:
        return tensor.cpu().numpy()
    src = tensor.contiguous()
    out = np.empty(tuple(src.shape), dtype=np.float64)
    with _lock:
        stage = _staging_view(nbytes, tuple(src.shape))
        host = stage.numpy()
        stream = torch.cuda.current_stream(src.device)
        events = []
        for a, b in _blocks(src.shape[0], 2 * _threads()):
            stage[a:b].copy_(src[a:b], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
            events.append((a, b, ev))
        pool = _get_pool()
        jobs = []
        for a, b, ev in events:
            ev.synchronize()
            jobs.append(pool.submit(np.copyto, out[a:b], host[a:b]))
        for j in jobs:
            j.result()
    return out


def upload(array, target):
    """Copy a float64 numpy array into a device tensor view of its shape
    (any strides); returns after the copy has completed.

    Pipelined in row blocks: pool threads copy the blocks into pinned memory
    and each block goes to the device as soon as it is staged."""
    import torch

    array = np.asarray(array, dtype=np.float64)
    if tuple(array.shape) != tuple(target.shape):
        raise ValueError(f"shape {array.shape} does not match the device view's {tuple(target.shape)}")
    nbytes = array.size * 8
    if nbytes < SMALL or array.ndim == 0:
        target.copy_(torch.from_numpy(np.ascontiguousarray(array)))
        return
    with _lock:
        stage = _staging_view(nbytes, tuple(array.shape))
        host = stage.numpy()
        pool = _get_pool()
        blocks = _blocks(array.shape[0], 2 * _threads())
        jobs = [pool.submit(np.copyto, host[a:b], array[a:b]) for a, b in blocks]
        for (a, b), j in zip(blocks, jobs):
            j.result()
            target[a:b].copy_(stage[a:b], non_blocking=True)  # on the target device's current stream
        torch.cuda.current_stream(target.device).synchronize()
