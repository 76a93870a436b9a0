"""
Host-side logic of the whole-state copies (sailfish_b200/_hostio.py), run
without a GPU: the row blocks of the staged copies, the staged upload's
block-major worker pipeline (with CPU tensors standing in for the device
buffer and the pinned staging memory), pageable arrays reported as such,
and the live-byte count of pinned hand-outs, which falls when the last view
of a returned array is freed.
"""

import gc
import types

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from sailfish_b200 import _hostio  # noqa: E402


def test_blocks_cover_the_rows_once():
    for n in (1, 7, 100, 4096):
        for k in (1, 3, 32, 5000):
            blocks = _hostio._blocks(n, k)
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(a < b for a, b in blocks)
            assert all(b0 == a1 for (_, b0), (a1, _) in zip(blocks, blocks[1:]))


def test_pageable_arrays_are_not_pinned():
    assert not _hostio.is_pinned(np.zeros((4, 4, 3)))
    assert not _hostio.is_pinned(np.zeros(0))
    assert not _hostio.is_pinned([1.0, 2.0])


@pytest.fixture
def cpu_standins(monkeypatch):
    """The staged upload's device pieces as CPU tensors (a stream that needs
    no synchronisation, staging memory that is not pinned)."""
    monkeypatch.setattr(torch.cuda, "current_stream", lambda device=None: types.SimpleNamespace(
        synchronize=lambda: None))

    def staging(nbytes, shape):
        buf = torch.empty(max(nbytes, 64 << 20), dtype=torch.uint8)
        return buf[:nbytes].view(torch.float64).view(shape)

    monkeypatch.setattr(_hostio, "_staging_view", staging)


@pytest.mark.parametrize("n", [33, 700, 1100])
def test_staged_upload_fills_a_strided_view_exactly(cpu_standins, n):
    host = np.random.default_rng(n).standard_normal((n, n + 3, 3))
    buf = torch.full((n + 4, n + 7, 3), float("nan"), dtype=torch.float64)
    _hostio.upload(host, buf[2:-2, 2:-2])
    np.testing.assert_array_equal(buf[2:-2, 2:-2].numpy(), host)
    assert torch.isnan(buf[:2]).all() and torch.isnan(buf[:, -2:]).all()


def test_staged_upload_raises_a_worker_error_without_hanging(cpu_standins, monkeypatch):
    n = 1100
    host = np.zeros((n, n, 3))
    buf = torch.zeros((n, n, 3), dtype=torch.float64)
    calls = []
    real = np.copyto

    def failing_copy(dst, src):
        calls.append(1)
        if len(calls) == 3:
            raise MemoryError("planted")
        real(dst, src)

    monkeypatch.setattr(_hostio.np, "copyto", failing_copy)
    with pytest.raises(MemoryError, match="planted"):
        _hostio.upload(host, buf)


def test_handout_count_follows_the_arrays(monkeypatch):
    real_empty = torch.empty

    def unpinned_empty(*args, **kw):
        kw.pop("pin_memory", None)
        return real_empty(*args, **kw)

    monkeypatch.setattr(torch, "empty", unpinned_empty)
    gc.collect()
    before = _hostio.handout_bytes()
    out = _hostio._pinned_handout((100, 3), 2400)
    arr = _hostio._counted_numpy(out, 2400)
    del out
    gc.collect()
    assert _hostio.handout_bytes() == before + 2400
    view = arr[10:20]
    del arr
    gc.collect()
    assert _hostio.handout_bytes() == before + 2400  # a view keeps the memory
    del view
    gc.collect()
    assert _hostio.handout_bytes() == before
    monkeypatch.setattr(_hostio, "PINNED_HANDOUT_LIMIT", before + 1000)
    assert _hostio._pinned_handout((100, 3), 2400) is None
    assert _hostio.handout_bytes() == before
