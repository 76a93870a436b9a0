"""
The correctly rounded arithmetic of the EXACT stencil, checked on the device:
Markstein-corrected division against IEEE division, the double-double
x^-1.5 and x^4 against correctly rounded values computed with Python's
decimal module, and the PLM slope against the reference's formula.
"""

import ctypes
from decimal import Decimal, getcontext

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sailfish_b200 import _capi  # noqa: E402


def _eval(a, b):
    da = torch.from_numpy(a).cuda()
    db = torch.from_numpy(b).cuda()
    out = torch.empty(4 * a.size, dtype=torch.float64, device="cuda")
    st = _capi.lib().cbdiso_b200_eval_primitives(a.size, ctypes.c_void_p(da.data_ptr()),
                                                 ctypes.c_void_p(db.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    return out.cpu().numpy().reshape(-1, 4)


def _random(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    mant = rng.uniform(1.0, 2.0, n)
    exp = rng.integers(lo, hi + 1, n)
    sign = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    return sign * np.ldexp(mant, exp)


def test_division_is_ieee():
    a = _random(4_000_000, -40, 40, 1)
    b = _random(4_000_000, -40, 40, 2)
    b[::3] = 16.0 / 4096.0 * (1 + np.arange(b[::3].size) % 7)
    out = _eval(a, b)
    assert np.array_equal(out[:, 0], a / b)


def _cr(v):
    return float(v)


def test_powers_are_correctly_rounded():
    getcontext().prec = 60
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.uniform(0.0025, 200.0, 20000), np.ldexp(rng.uniform(1, 2, 5000),
                                                                    rng.integers(-20, 20, 5000))])
    out = _eval(x, np.ones_like(x))
    want15 = np.array([_cr(Decimal(float(v)) ** Decimal(-1.5)) for v in x])
    want4 = np.array([_cr(Decimal(float(v)) ** 4) for v in x])
    assert np.array_equal(out[:, 1], want15)
    assert np.array_equal(out[:, 2], want4)


def test_plm_slope_matches_reference_formula():
    a = _random(200000, -5, 5, 4)
    b = _random(200000, -5, 5, 5)
    a[::7] = 0.0
    out = _eval(a, b)
    yl, y0, yr, th = a, b, a + b, 1.5
    x = (y0 - yl) * th
    y = (yr - yl) * 0.5
    z = (yr - y0) * th
    m = np.minimum(np.abs(x), np.minimum(np.abs(y), np.abs(z)))
    want = 0.25 * np.abs(np.copysign(1, x) + np.copysign(1, y)) * (np.copysign(1, x) + np.copysign(1, z)) * m
    assert np.array_equal(out[:, 3], want)
