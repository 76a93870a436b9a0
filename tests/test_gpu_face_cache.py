"""
The face cache (cbdiso_b200_advance_stage_cached): the stage at t0 + dt stores
the face sound speeds and zone gravity factors for its point masses, and the
next step's first stage loads them (after a fill pass when the key does not
match its masses). In EXACT precision states, dts and reductions must be
bit-identical to recomputing them in every stage.
"""

import ctypes

import numpy as np
import pytest

from cases import load
from test_gpu_parity import field_error, product_solver

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

CASES = ["cbd_t15_n64", "cbd_t18_48x40_ecc", "kitp_t15_n56_rk1_forcefree", "kitp_t18_n64_rk3_p2",
         "bondi_t18_64x32", "explosion_t15_n40", "cbd_t18_n48_inactive"]


def _host_loop(s, steps):
    dts, red = [], []
    for _ in range(steps):
        dt = s.mesh.min_spacing() / s.maximum_wavespeed() * 0.3
        s.advance(dt)
        dts.append(dt)
        red.append(s.reductions())
    return dts, red


@pytest.mark.parametrize("name", CASES)
def test_host_loop_bit_identical_with_and_without_cache(name):
    d = load(name)
    on = product_solver(d, "exact", face_cache=True)
    off = product_solver(d, "exact", face_cache=False)
    assert on._fcache is not None and off._fcache is None
    a = _host_loop(on, 12)
    b = _host_loop(off, 12)
    assert a[0] == b[0]
    assert a[1] == b[1]
    assert np.array_equal(on.solution, off.solution)


@pytest.mark.parametrize("name", ["cbd_t15_n64", "kitp_t18_n64_rk3_p2", "bondi_t18_64x32"])
@pytest.mark.parametrize("precision", ["fma", "fast"])
def test_host_loop_with_and_without_cache_contracted(name, precision):
    """The FMA and FAST builds let the compiler contract a * b + c freely,
    and it may contract the kernel's cached and uncached code paths
    differently: the two agree to rounding, not bit for bit."""
    d = load(name)
    on = product_solver(d, precision, face_cache=True)
    off = product_solver(d, precision, face_cache=False)
    a = _host_loop(on, 12)
    b = _host_loop(off, 12)
    np.testing.assert_allclose(a[0], b[0], rtol=1e-13, atol=0)
    assert field_error(on.solution, off.solution) <= 1e-13


@pytest.mark.parametrize("name", ["cbd_t15_n64", "kitp_t18_n64_rk3_p2", "kitp_t15_n56_rk1_forcefree"])
def test_device_loop_bit_identical_with_and_without_cache(name):
    d = load(name)
    on = product_solver(d, "exact", face_cache=True)
    off = product_solver(d, "exact", face_cache=False)
    ra = on.run(20, cfl=0.3, graph=True, steps_per_graph=5)
    rb = off.run(20, cfl=0.3, graph=True, steps_per_graph=5)
    assert ra == rb
    assert np.array_equal(on.solution, off.solution)


def _face_values(s, time):
    """cs^2 at the x-faces (numpy, the reference's operation order) for the
    locally isothermal EOS, with the point masses at `time`."""
    g = s._grid
    ni, nj = g.ni, g.nj
    dx, dy = (g.xr - g.xl) / ni, (g.yr - g.yl) / nj
    i = np.arange(ni + 1, dtype=np.float64)[:, None]
    j = np.arange(nj, dtype=np.float64)[None, :]
    x = g.xl + i * dx
    y = g.yl + (j + 0.5) * dy
    phi = np.zeros((ni + 1, nj))
    for m in s._point_masses(time):
        if m.mass > 0.0:
            dxm, dym = x - m.position_x, y - m.position_y
            r2 = dxm * dxm + dym * dym
            phi -= m.mass / np.sqrt(r2 + m.softening_length * m.softening_length)
    return -phi / g.mach2


def test_cache_holds_the_end_of_step_face_sound_speeds():
    d = load("cbd_t15_n64")
    s = product_solver(d, "exact", face_cache=True)
    s.advance(s.mesh.min_spacing() / s.maximum_wavespeed() * 0.3)
    torch.cuda.synchronize()
    c = s._fcache.cpu().numpy()
    assert c[0] == 20261204.5  # the key's format tag: the last stage recorded its masses
    g = s._grid
    ni, nj = g.ni, g.nj
    pairs = c[32:32 + 2 * (ni + 1) * nj].reshape(ni + 1, nj, 2)
    want = _face_values(s, s.time)
    assert np.array_equal(pairs[..., 0], want)
    assert np.array_equal(pairs[..., 1], np.sqrt(want))


def test_fill_pass_holds_the_stage_values():
    """A reader's fill pass computes the face sound speeds for the stage's
    masses when the key does not match them (here: a new cache)."""
    from sailfish_b200 import _capi

    d = load("cbd_t15_n64")
    s = product_solver(d, "exact", face_cache=True)
    lib, g = s._lib, s._grid
    st = _capi.Stage()
    m1, m2 = s._point_masses(0.25)
    from sailfish_b200.cbdiso_2d import _mass_struct

    _mass_struct(m1, st.mass[0])
    _mass_struct(m2, st.mass[1])
    st.a, st.dt, st.buffer_central_mass = 0.0, 1e-4, m1.mass + m2.mass
    out = torch.empty_like(s._buf[1])
    assert lib.cbdiso_b200_advance_stage_cached(ctypes.byref(g), ctypes.byref(st), None, s._ptr(s._buf[0]), None,
                                                s._ptr(out), None, None, None, s._ptr(s._fcache), 2,
                                                s._stream()) == 0
    torch.cuda.synchronize()
    c = s._fcache.cpu().numpy()
    ni, nj = g.ni, g.nj
    assert c[0] == 20261204.5  # the reader recorded the key
    pairs = c[32:32 + 2 * (ni + 1) * nj].reshape(ni + 1, nj, 2)
    want = _face_values(s, 0.25)
    assert np.array_equal(pairs[..., 0], want)
    assert np.array_equal(pairs[..., 1], np.sqrt(want))


def test_cache_after_reset():
    d = load("cbd_t18_48x40_ecc")
    on = product_solver(d, "exact", face_cache=True)
    off = product_solver(d, "exact", face_cache=False)
    start, t0 = on.solution.copy(), on.time
    # back to an earlier time: the cached key no longer matches
    _host_loop(on, 5)
    on.reset(start, t0)
    assert _host_loop(on, 6) == _host_loop(off, 6)
    assert np.array_equal(on.solution, off.solution)
    # another state at the cached time: the key matches, the values still apply
    t1 = on.time
    on.reset(start, t1)
    off.reset(start, t1)
    assert _host_loop(on, 4) == _host_loop(off, 4)
    assert np.array_equal(on.solution, off.solution)


def test_cached_entry_rejects_a_misaligned_cache():
    from sailfish_b200 import _capi

    d = load("cbd_t15_n64")
    s = product_solver(d, "exact", face_cache=True)
    st = _capi.Stage()
    args = (ctypes.byref(s._grid), ctypes.byref(st), None, s._ptr(s._buf[0]), None, s._ptr(s._buf[1]), None,
            None, None)
    lib = s._lib
    assert lib.cbdiso_b200_advance_stage_cached(*args, ctypes.c_void_p(s._fcache.data_ptr() + 8), 2,
                                                s._stream()) == 1  # invalid argument
    assert lib.cbdiso_b200_advance_stage_cached(*args, s._ptr(s._fcache), 3, s._stream()) == 1
    assert int(s._lib.cbdiso_b200_face_cache_bytes(ctypes.byref(s._grid))) == \
        8 * (32 + 2 * (65 * 64 + 64 * 65 + 64 * 64))


@pytest.mark.parametrize("name", ["gam_n64", "gam_n40_soft_inviscid", "gam_n48_cool_p2", "gam_n256"])
def test_gamma_law_bit_identical_with_and_without_cache(name):
    """The gamma-law solver's cache (scale-height geometry at faces and
    centres, gravity factors with constant softening) changes no bit."""
    from cases import gam_names
    from test_gpu_gamma import gam_solver

    assert name in gam_names()
    d = load(name)
    on, off = gam_solver(d, face_cache=True), gam_solver(d, face_cache=False)
    assert on._fcache is not None and off._fcache is None
    cfl = d["meta"]["cfl"]
    for _ in range(10):
        dt = on.mesh.min_spacing() / on.maximum_wavespeed() * cfl
        assert dt == off.mesh.min_spacing() / off.maximum_wavespeed() * cfl
        on.advance(dt)
        off.advance(dt)
        assert on.reductions() == off.reductions()
    assert np.array_equal(on.solution, off.solution)
    torch.cuda.synchronize()
    assert float(on._fcache[0]) == 20260102.5  # the second stages wrote their values

