"""
Whole-state host <-> device copies (sailfish_b200/_hostio.py): bit-exact
round trips for strided device views above and below the staging threshold,
from pageable and from pinned host arrays, downloads into pinned arrays of
their own and past the pinned hand-out limit, and concurrent callers. Also
the FP64 issue-rate probe the benchmark's FP64 roofline divides by.
"""

import gc
import threading
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sailfish_b200 import _hostio  # noqa: E402


@pytest.mark.parametrize("n", [40, 1100])
def test_round_trip_through_strided_views(n):
    rng = np.random.default_rng(n)
    host = rng.standard_normal((n, n + 3, 3))
    buf = torch.full((n + 4, n + 7, 3), float("nan"), dtype=torch.float64, device="cuda")
    view = buf[2:-2, 2:-2]
    _hostio.upload(host, view)
    assert torch.isnan(buf[:2]).all() and torch.isnan(buf[:, -2:]).all()  # guards untouched
    back = _hostio.download(view)
    assert back.shape == host.shape and back.dtype == np.float64
    np.testing.assert_array_equal(back, host)
    # the returned array is the caller's own: a later download does not touch it
    _hostio.upload(host * 2.0, view)
    np.testing.assert_array_equal(back, host)
    np.testing.assert_array_equal(_hostio.download(view), host * 2.0)


def _strided_view(n):
    buf = torch.full((n + 4, n + 7, 3), float("nan"), dtype=torch.float64, device="cuda")
    return buf, buf[2:-2, 2:-2]


def test_downloads_are_pinned_and_pinned_arrays_upload_directly():
    n = 1100
    host = np.random.default_rng(1).standard_normal((n, n + 3, 3))
    buf, view = _strided_view(n)
    assert not _hostio.is_pinned(host)
    _hostio.upload(host, view)  # staged: pageable source
    back = _hostio.download(view)
    assert _hostio.is_pinned(back) and back.flags.c_contiguous and back.flags.writeable
    np.testing.assert_array_equal(back, host)
    # a pinned array goes straight to the device, read-only ones included
    p = _hostio.pinned_empty(host.shape)
    assert _hostio.is_pinned(p)
    p[...] = host * 3.0
    p.flags.writeable = False
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        _hostio.upload(p, view)
    assert torch.isnan(buf[:2]).all() and torch.isnan(buf[:, -2:]).all()  # guards untouched
    np.testing.assert_array_equal(_hostio.download(view), host * 3.0)
    # the first download is the caller's own: the later copies did not touch it
    np.testing.assert_array_equal(back, host)
    # and uploads directly as well
    _hostio.upload(back, view)
    np.testing.assert_array_equal(_hostio.download(view), host)


def test_pinned_handout_limit(monkeypatch):
    n = 1100
    host = np.random.default_rng(2).standard_normal((n, n + 3, 3))
    _, view = _strided_view(n)
    _hostio.upload(host, view)
    gc.collect()
    before = _hostio.handout_bytes()
    arrays = [_hostio.download(view) for _ in range(2)]
    assert _hostio.handout_bytes() == before + 2 * host.nbytes
    del arrays
    gc.collect()
    assert _hostio.handout_bytes() == before
    # past the limit: a pageable array, the same values
    monkeypatch.setattr(_hostio, "PINNED_HANDOUT_LIMIT", 0)
    back = _hostio.download(view)
    assert not _hostio.is_pinned(back)
    np.testing.assert_array_equal(back, host)
    assert _hostio.handout_bytes() == before


def test_shape_mismatch_raises():
    buf = torch.zeros((10, 10, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        _hostio.upload(np.zeros((9, 10, 3)), buf)


def test_concurrent_callers_and_release():
    n = 1024
    arrays = [np.full((n, n, 3), float(k)) for k in range(4)]
    bufs = [torch.empty((n, n, 3), dtype=torch.float64, device="cuda") for _ in range(4)]
    errors = []

    def work(k):
        try:
            for _ in range(3):
                _hostio.upload(arrays[k], bufs[k])
                got = _hostio.download(bufs[k])
                assert np.array_equal(got, arrays[k])
        except Exception as e:  # noqa: BLE001
            errors.append(e)

    threads = [threading.Thread(target=work, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors
    _hostio.release_staging()
    np.testing.assert_array_equal(_hostio.download(bufs[1]), arrays[1])


def test_fp64_probe_measures_a_plausible_rate():
    """The FP64 issue-rate probe behind the bench's FP64 roofline runs and
    reports a rate between 1 and 100 T thread-FMAs/s."""
    import ctypes

    from sailfish_b200 import _capi

    lib = _capi.lib()
    blocks = 8 * torch.cuda.get_device_properties(0).multi_processor_count
    out = torch.zeros(blocks, dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    assert lib.cbdiso_b200_fp64_probe(1000, blocks, ctypes.c_void_p(out.data_ptr()), stream) == 0
    start.record()
    assert lib.cbdiso_b200_fp64_probe(20000, blocks, ctypes.c_void_p(out.data_ptr()), stream) == 0
    stop.record()
    torch.cuda.synchronize()
    rate = lib.cbdiso_b200_fp64_probe_fmas(20000, blocks) / (start.elapsed_time(stop) * 1e-3)
    assert 1e12 < rate < 1e14
    assert not out.any()  # the guard store never fires
    assert lib.cbdiso_b200_fp64_probe(0, blocks, ctypes.c_void_p(out.data_ptr()), stream) == 1
