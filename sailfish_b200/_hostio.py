"""
Whole-state copies between host numpy arrays and device tensors.

A state at 4096^2 is 403 MB. The device reaches page-locked (pinned) host
memory at PCIe speed (about 55 GB/s each way on the B200 host); pageable
memory it reaches only through the driver's own staging, at 2-10 GB/s, and
a new numpy array's pages are first touched (faulted in and zeroed) by the
single copying thread. So:

* `upload` of an array that already lives in pinned memory (one from
  `pinned_empty`, or one that `download` returned) is one direct copy.
  Any other array goes through one pinned staging buffer kept for the
  process: the pool's threads copy it in row blocks, every thread on the
  same block, so the first blocks are staged early and each goes to the
  device as soon as it is staged while the next ones are copied.
* `download` returns an array in pinned memory of its own: one direct
  copy, and the caller's later `upload` of it is direct too. Freed, such an
  array's memory goes back to torch's pinned-memory cache, where the next
  download finds it, so pinning (about 0.2 s for 403 MB) is paid once per
  size and process. While more than `PINNED_HANDOUT_LIMIT` bytes of
  returned arrays are alive, further downloads return pageable arrays
  copied through the staging buffer instead, so that a caller keeping many
  states does not pin an unbounded amount of host memory.

The staging buffer is allocated on first use and grows to the largest
state staged; `release_staging()` frees it. Staged copies are serialised by
a lock, so threads may share this module.
"""

from __future__ import annotations

import collections
import os
import threading
import warnings
import weakref
from concurrent.futures import ThreadPoolExecutor

import numpy as np

SMALL = 8 << 20  # below this many bytes a plain copy is as fast
PINNED_HANDOUT_LIMIT = 16 << 30  # bytes of live pinned arrays returned by `download`
_lock = threading.Lock()
_handout_lock = threading.Lock()
_handout_bytes = 0
_released = collections.deque()  # byte counts of freed hand-outs, not yet subtracted
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


def pinned_empty(shape):
    """An uninitialised float64 numpy array of `shape` in pinned host memory:
    the form of host data that `upload` sends to the device in one direct
    copy. The memory returns to torch's pinned-memory cache when the array
    and its views are freed."""
    import torch

    return torch.empty(tuple(shape), dtype=torch.float64, pin_memory=True).numpy()


def is_pinned(array):
    """Whether a numpy array's memory is page-locked host memory that the
    device can copy from directly."""
    import torch

    if not isinstance(array, np.ndarray) or array.size == 0 or not torch.cuda.is_available():
        return False
    try:
        return bool(_as_tensor(array).is_pinned())
    except (TypeError, ValueError, RuntimeError):
        return False


def _as_tensor(array):
    """A CPU tensor over the array's memory (read-only arrays included:
    torch only warns that it could write to them, and nothing here does)."""
    import torch

    with warnings.catch_warnings():
        warnings.simplefilter("ignore", UserWarning)
        return torch.from_numpy(array)


def _blocks(n, k):
    k = max(1, min(k, n))
    return [(a * n // k, (a + 1) * n // k) for a in range(k)]


def _release_handout(nbytes):
    # Runs in whichever thread frees the array, possibly in the middle of this
    # module's own critical section (a garbage collection there): so no lock,
    # only a thread-safe append that the next count takes off.
    _released.append(nbytes)


def _drain_released():
    """Subtract the freed hand-outs from the count; the caller holds
    _handout_lock."""
    global _handout_bytes
    while True:
        try:
            nbytes = _released.popleft()
        except IndexError:
            return _handout_bytes
        _handout_bytes -= nbytes


def handout_bytes():
    """Bytes of pinned arrays returned by `download` and still alive."""
    with _handout_lock:
        return _drain_released()


def _pinned_handout(shape, nbytes):
    """A pinned float64 tensor for a download, counted against the limit;
    None when the limit would be passed. The caller hands its memory out
    through `_counted_numpy`."""
    import torch

    global _handout_bytes
    with _handout_lock:
        if _drain_released() + nbytes > PINNED_HANDOUT_LIMIT:
            return None
        _handout_bytes += nbytes
    try:
        return torch.empty(shape, dtype=torch.float64, pin_memory=True)
    except RuntimeError:
        _release_handout(nbytes)
        return None


def _counted_numpy(out, nbytes):
    """The numpy array over a hand-out tensor. The count drops when the
    object that owns the memory for numpy (the array's base, which the
    array and all its views keep alive; not `out` itself, a separate
    wrapper) is freed."""
    arr = out.numpy()
    weakref.finalize(arr.base if arr.base is not None else arr, _release_handout, nbytes)
    return arr


def download(tensor):
    """A new numpy array equal to a float64 device tensor (any strides).

    Normally in pinned memory of its own, filled by one device-to-host copy.
    Past the pinned hand-out limit: a pageable array, pipelined in row
    blocks (each block's device-to-pinned copy is followed, as soon as it
    has landed, by its copy into the array on a pool thread, while the next
    blocks are still in flight)."""
    import torch

    nbytes = tensor.numel() * 8
    if nbytes < SMALL or tensor.dim() == 0:
        return tensor.cpu().numpy()
    out = _pinned_handout(tuple(tensor.shape), nbytes)
    if out is not None:
        try:
            out.copy_(tensor, non_blocking=True)
            torch.cuda.current_stream(tensor.device).synchronize()
        except BaseException:
            _release_handout(nbytes)
            raise
        return _counted_numpy(out, nbytes)
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

    From pinned memory: one direct copy. Otherwise staged in row blocks: all
    pool threads copy block 0 into pinned memory (each its own rows), then
    block 1, and so on, and each block goes to the device as soon as its
    rows are staged."""
    import torch

    array = np.asarray(array, dtype=np.float64)
    if tuple(array.shape) != tuple(target.shape):
        raise ValueError(f"shape {array.shape} does not match the device view's {tuple(target.shape)}")
    nbytes = array.size * 8
    if nbytes < SMALL or array.ndim == 0:
        target.copy_(torch.from_numpy(np.ascontiguousarray(array)))
        return
    stream = torch.cuda.current_stream(target.device)
    if array.flags.c_contiguous and is_pinned(array):
        target.copy_(_as_tensor(array), non_blocking=True)
        stream.synchronize()
        return
    with _lock:
        stage = _staging_view(nbytes, tuple(array.shape))
        host = stage.numpy()
        nthreads = _threads()
        blocks = _blocks(array.shape[0], 2 * nthreads)
        left = [nthreads] * len(blocks)
        staged = [threading.Event() for _ in blocks]
        count_lock = threading.Lock()

        def stage_rows(w):
            # worker w: its share of every block's rows, block by block.
            # Every block is counted even after a failed copy, so that no
            # wait below is left hanging; the job's result raises the error.
            error = None
            for k, (a, b) in enumerate(blocks):
                lo, hi = a + (b - a) * w // nthreads, a + (b - a) * (w + 1) // nthreads
                if error is None and hi > lo:
                    try:
                        np.copyto(host[lo:hi], array[lo:hi])
                    except BaseException as e:  # noqa: BLE001
                        error = e
                with count_lock:
                    left[k] -= 1
                    if left[k] == 0:
                        staged[k].set()
            if error is not None:
                raise error

        jobs = [_get_pool().submit(stage_rows, w) for w in range(nthreads)]
        for k, (a, b) in enumerate(blocks):
            staged[k].wait()
            target[a:b].copy_(stage[a:b], non_blocking=True)  # on the target device's current stream
        for j in jobs:
            j.result()
        stream.synchronize()
