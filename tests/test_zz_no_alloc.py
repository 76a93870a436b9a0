"""
The no-allocation stage entry point, cbdiso_b200_advance_stage_noalloc.

Some callers cannot allocate device memory: a binding written against the
reference's kernel interface passes only the arrays its solver owns and has
no scratch buffer to offer, and applications that route all device memory
through their own pool do not let a library call cudaMalloc. This entry point
keeps the epilogue's reductions scratch in a fixed 5 MiB array inside the
library. Here it is called through the C-ABI twice in a row and compared with
the existing entry point (caller-provided scratch) on the same inputs, within
the tolerance of the other parity tests; grids beyond its capacity are
rejected before any launch.

This file is named to be collected last, so a run that stops at the first
failure has run every other test first. It also passes on its own in a fresh
process.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from oracle import host as oh  # noqa: E402
from sailfish_b200 import _capi  # noqa: E402

CAPACITY_ERROR = 6  # CBD_ERR_CAPACITY


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _mass(m, out):
    out.x, out.y, out.vx, out.vy, out.mass = m.x, m.y, m.vx, m.vy, m.mass
    out.softening_length, out.sink_rate, out.sink_radius, out.sink_model = 0.05, m.sink_rate, m.sink_radius, 2


def _problem(ni=300, nj=260):
    g = _capi.Grid()
    g.ni, g.nj = ni, nj
    g.xl, g.xr, g.yl, g.yr = -8.0, 8.0, -7.0, 7.0
    g.plm_theta, g.eos_type, g.precision = 1.5, 2, 0
    g.cs2, g.mach2, g.nu = 1.0, 100.0, 1e-3
    g.velocity_ceiling, g.density_floor = 1e12, 1e-12
    g.buffer_is_enabled, g.buffer_surface_density = 1, 1.0
    g.buffer_driving_rate, g.buffer_outer_radius, g.buffer_onset_width = 100.0, 8.0, 1.0
    masses = oh.binary_masses(1.0, 1.0, 0.7, 0.2)
    st = _capi.Stage()
    m1, m2 = masses(0.3)
    _mass(m1, st.mass[0])
    _mass(m2, st.mass[1])
    st.a, st.dt, st.buffer_central_mass = 0.0, 2e-3, m1.mass + m2.mass
    ep = _capi.Epilogue()
    e1, e2 = masses(0.302)
    _mass(e1, ep.mass[0])
    _mass(e2, ep.mass[1])
    ep.want_wavespeed = 1
    diags = [(1, 1, 0, 1), (1, 2, 0, 1), (4, 3, 1, 0)]  # mdot m1, mdot m2 (accretion), torque both (gravity)
    ep.num_diag = len(diags)
    for k, (q, w, grav, acc) in enumerate(diags):
        ep.diag[k].quantity, ep.diag[k].which_mass, ep.diag[k].gravity, ep.diag[k].accretion = q, w, grav, acc
    cfg = oh.Config(g.xl, g.xr, g.yl, g.yr, ni, nj)
    x, y = oh.cell_centres(cfg)
    prim = oh.circumbinary_disk_primitive(x, y)
    prim[..., 0] += oh.seeded_noise(ni, nj, 5)
    dev = torch.zeros((ni + 4, nj + 4, 3), dtype=torch.float64, device="cuda")
    dev[2:-2, 2:-2] = torch.from_numpy(prim).cuda()
    return g, st, ep, dev


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def test_noalloc_stage_matches_the_allocating_entry_point_on_two_calls():
    lib = _capi.lib()
    g, st, ep, p = _problem()
    assert lib.cbdiso_b200_fill_guards(ctypes.byref(g), _ptr(p), _stream()) == 0

    # existing entry point, with caller-allocated scratch
    scratch = torch.zeros(lib.cbdiso_b200_scratch_bytes(ctypes.byref(g)) // 8 + 8, dtype=torch.float64,
                          device="cuda")
    want_p = torch.zeros_like(p)
    want_r = torch.zeros(33, dtype=torch.float64, device="cuda")
    assert lib.cbdiso_b200_advance_stage(ctypes.byref(g), ctypes.byref(st), None, _ptr(p), None, _ptr(want_p),
                                         ctypes.byref(ep), _ptr(scratch), _ptr(want_r), _stream()) == 0
    want_p, want_r = want_p.cpu().numpy(), want_r.cpu().numpy()[:7]

    for call in range(2):
        got_p = torch.zeros_like(p)
        got_r = torch.full((33,), np.nan, dtype=torch.float64, device="cuda")
        status = lib.cbdiso_b200_advance_stage_noalloc(ctypes.byref(g), ctypes.byref(st), None, _ptr(p), None,
                                                       _ptr(got_p), ctypes.byref(ep), _ptr(got_r), _stream())
        assert status == 0, f"call {call}: status {status}"
        got_p, got_r = got_p.cpu().numpy(), got_r.cpu().numpy()[:7]
        for q in range(3):
            scale = np.abs(want_p[..., q]).max()
            assert np.abs(got_p[..., q] - want_p[..., q]).max() <= 1e-12 * scale, f"call {call}, field {q}"
        assert got_r[0] == pytest.approx(want_r[0], rel=1e-14)
        assert np.all(np.abs(got_r[1:] - want_r[1:]) <= 1e-12 * np.maximum(np.abs(want_r[1:]), 1e-300) + 1e-300)


def test_noalloc_rejects_grids_beyond_its_capacity():
    lib = _capi.lib()
    g, st, ep, _ = _problem(16, 16)
    g.ni = g.nj = 8192
    assert lib.cbdiso_b200_scratch_bytes(ctypes.byref(g)) > (5 << 20)
    status = lib.cbdiso_b200_advance_stage_noalloc(ctypes.byref(g), ctypes.byref(st), None, None, None, None,
                                                   ctypes.byref(ep), None, None)
    assert status == CAPACITY_ERROR
    assert lib.cbdiso_b200_status_string(status) == b"request exceeds library capacity"


def test_noalloc_stage_without_epilogue_has_no_size_limit():
    """A stage with no epilogue uses no scratch: an 8192^2 grid, beyond the
    array's capacity with an epilogue, runs and equals the allocating entry
    point's result bit for bit (the same kernel on the same inputs)."""
    lib = _capi.lib()
    g, st, _, small = _problem(16, 16)
    n = 8192
    g.ni = g.nj = n
    g.xl, g.xr, g.yl, g.yr = -8.0, 8.0, -8.0, 8.0
    cfg = oh.Config(g.xl, g.xr, g.yl, g.yr, n, n)
    x, y = oh.cell_centres(cfg)
    p = torch.zeros((n + 4, n + 4, 3), dtype=torch.float64, device="cuda")
    p[2:-2, 2:-2] = torch.from_numpy(oh.circumbinary_disk_primitive(x, y)).cuda()
    del x, y
    assert lib.cbdiso_b200_fill_guards(ctypes.byref(g), _ptr(p), _stream()) == 0
    got = torch.zeros_like(p)
    status = lib.cbdiso_b200_advance_stage_noalloc(ctypes.byref(g), ctypes.byref(st), None, _ptr(p), None,
                                                   _ptr(got), None, None, _stream())
    assert status == 0
    want = torch.zeros_like(p)
    assert lib.cbdiso_b200_advance_stage(ctypes.byref(g), ctypes.byref(st), None, _ptr(p), None, _ptr(want),
                                         None, None, None, _stream()) == 0
    assert torch.equal(got, want)
