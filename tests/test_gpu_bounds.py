"""
Bounds canaries and awkward grid sizes for every kernel family of both
solvers: each device array of a launch sits inside a larger buffer whose
margins (1 MiB on each side) hold a sentinel bit pattern, and after the
launch the margins must be untouched. Sizes include a single zone, sizes below
one tile and odd sizes that fill no tile (257 x 130, 130 x 257); at 257 x 130
the stage results are also compared with the oracles.
"""

import ctypes

import numpy as np
import pytest

from oracle import host as oh
from oracle import host_gam as og

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sailfish_b200 import _capi  # noqa: E402

MARGIN = 1 << 17  # doubles
SENTINEL = -1.2345678901234567e300
SIZES = [(1, 1), (2, 3), (5, 130), (130, 5), (257, 130), (130, 257)]


class Padded:
    """A device float64 array of `shape` inside sentinel margins."""

    def __init__(self, shape, fill=0.0):
        self.shape = tuple(shape)
        self.n = int(np.prod(self.shape))
        self.whole = torch.full((self.n + 2 * MARGIN,), SENTINEL, dtype=torch.float64, device="cuda")
        self.view = self.whole[MARGIN:MARGIN + self.n].view(self.shape)
        self.view.fill_(fill)

    @property
    def ptr(self):
        return ctypes.c_void_p(self.view.data_ptr())

    def intact(self):
        sentinel = torch.tensor(SENTINEL, dtype=torch.float64).view(torch.int64).item()
        bits = self.whole.view(torch.int64)
        return bool((bits[:MARGIN] == sentinel).all()) and bool((bits[MARGIN + self.n:] == sentinel).all())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _iso_state(ni, nj, seed=3):
    cfg = oh.Config(-8.0, 8.0, -7.0, 7.0, ni, nj, eos_type=2, mach_number=10.0, nu=1e-3, buffer_is_enabled=True,
                    buffer_driving_rate=100.0, buffer_onset_width=1.0, buffer_surface_density=1.0,
                    masses=oh.binary_masses(1.0, 1.0, 0.7, 0.2), plm_theta=1.5)
    x, y = oh.cell_centres(cfg)
    prim = oh.circumbinary_disk_primitive(x, y)
    prim[..., 0] += oh.seeded_noise(ni, nj, seed)
    s = oh.OracleSolver(cfg, prim, 0.3, oh.Kernels("oracle", 1.5))
    s._set_bc()
    return cfg, s


def _mass(m, out):
    (out.x, out.y, out.vx, out.vy, out.mass, out.softening_length, out.sink_rate, out.sink_radius,
     out.sink_model) = m.args()


@pytest.mark.parametrize("ni, nj", SIZES)
def test_isothermal_kernels_stay_in_bounds(ni, nj):
    cfg, s = _iso_state(ni, nj)
    lib = _capi.lib()
    lib.cbdiso_b200_set_stream(_stream())
    assert lib.cbdiso_b200_set_plm_theta(1.5) == 0
    shape = s.p1.shape
    prd = Padded(shape)
    prd.view.copy_(torch.from_numpy(s.p1))
    u0 = Padded(shape)
    assert lib.cbdiso_2d_primitive_to_conserved(ni, nj, prd.ptr, u0.ptr) == 0
    wr = Padded(shape)
    m1, m2 = cfg.point_masses(s.time)
    buf = (cfg.buffer_surface_density, m1.mass + m2.mass, cfg.buffer_driving_rate, s.buffer_outer_radius,
           cfg.buffer_onset_width, int(cfg.buffer_is_enabled))
    dt = 0.5 * oh.driver_dt(s, 0.3)
    assert lib.cbdiso_2d_advance_rk(ni, nj, s.xl, s.xr, s.yl, s.yr, u0.ptr, prd.ptr, wr.ptr, *buf, *m1.args(),
                                    *m2.args(), cfg.sound_speed ** 2, cfg.mach_number ** 2, cfg.eos_type, cfg.nu,
                                    0.5, dt, cfg.velocity_ceiling, cfg.density_floor) == 0
    ws = Padded(shape[:2])
    assert lib.cbdiso_2d_wavespeed(ni, nj, s.xl, s.xr, s.yl, s.yr, cfg.sound_speed ** 2, cfg.mach_number ** 2,
                                   cfg.eos_type, *m1.args(), *m2.args(), prd.ptr, ws.ptr) == 0
    rate = Padded(shape)
    assert lib.cbdiso_2d_point_mass_source_term(ni, nj, s.xl, s.xr, s.yl, s.yr, *m1.args(), prd.ptr,
                                                rate.ptr) == 0

    # the product stage with its epilogue, scratch and result in margins too
    g = _capi.Grid()
    g.ni, g.nj = ni, nj
    g.xl, g.xr, g.yl, g.yr = s.xl, s.xr, s.yl, s.yr
    g.plm_theta, g.eos_type, g.precision = 1.5, 2, 0
    g.cs2, g.mach2, g.nu = 1.0, 100.0, 1e-3
    g.velocity_ceiling, g.density_floor = cfg.velocity_ceiling, cfg.density_floor
    g.buffer_is_enabled, g.buffer_surface_density = 1, 1.0
    g.buffer_driving_rate, g.buffer_outer_radius, g.buffer_onset_width = 100.0, s.buffer_outer_radius, 1.0
    st = _capi.Stage()
    _mass(m1, st.mass[0])
    _mass(m2, st.mass[1])
    st.a, st.dt, st.buffer_central_mass = 0.5, dt, m1.mass + m2.mass
    ep = _capi.Epilogue()
    _mass(m1, ep.mass[0])
    _mass(m2, ep.mass[1])
    ep.want_wavespeed, ep.num_diag = 1, 2
    ep.diag[0].quantity, ep.diag[0].which_mass, ep.diag[0].accretion = 1, 3, 1
    ep.diag[1].quantity, ep.diag[1].which_mass, ep.diag[1].gravity = 4, 3, 1
    scratch = Padded((int(lib.cbdiso_b200_scratch_bytes(ctypes.byref(g))) // 8 + 8,))
    result = Padded((33,))
    out = Padded(shape)
    assert lib.cbdiso_b200_advance_stage(ctypes.byref(g), ctypes.byref(st), None, prd.ptr, prd.ptr, out.ptr,
                                         ctypes.byref(ep), scratch.ptr, result.ptr, _stream()) == 0
    assert lib.cbdiso_b200_fill_guards(ctypes.byref(g), out.ptr, _stream()) == 0
    assert lib.cbdiso_b200_reduce(ctypes.byref(g), ctypes.byref(ep), out.ptr, scratch.ptr, result.ptr,
                                  _stream()) == 0
    torch.cuda.synchronize()
    for a in (prd, u0, wr, ws, rate, scratch, result, out):
        assert a.intact()
    interior = out.view[2:-2, 2:-2].cpu().numpy()
    assert np.isfinite(interior).all() and np.isfinite(result.view[:5].cpu().numpy()).all()
    if (ni, nj) == (257, 130):
        want = np.zeros_like(s.p1)
        s.k.advance_rk(ni, nj, s.xl, s.xr, s.yl, s.yr, u0.view.cpu().numpy(), s.p1, want, buf, m1, m2,
                       cfg.sound_speed ** 2, cfg.mach_number ** 2, cfg.eos_type, cfg.nu, 0.5, dt,
                       cfg.velocity_ceiling, cfg.density_floor)
        got = wr.view.cpu().numpy()
        for q in range(3):
            scale = np.abs(want[2:-2, 2:-2, q]).max()
            assert np.abs(got[2:-2, 2:-2, q] - want[2:-2, 2:-2, q]).max() <= 1e-13 * scale


def _gam_state(ni, nj, seed=4):
    masses = oh.binary_masses(1.0, 1.0, 0.7, 0.2)
    cfg = og.GamConfig(-6.0, 6.0, -5.0, 5.0, ni, nj, alpha=0.1, cooling_coefficient=1.0, buffer_is_enabled=True,
                       buffer_surface_density=0.3, buffer_surface_pressure=3e-3, masses=masses)
    prim = np.empty((ni, nj, 4))
    for i in range(ni):
        for j in range(nj):
            prim[i, j] = og.gamma_disk_primitive(cfg.x0 + (i + 0.5) * cfg.dx, cfg.y0 + (j + 0.5) * cfg.dy)
    prim[..., 0] *= 1.0 + oh.seeded_noise(ni, nj, seed)
    s = og.GamOracleSolver(cfg, prim, 0.2)
    s._set_bc()
    return cfg, s


@pytest.mark.parametrize("ni, nj", SIZES)
def test_gamma_law_kernels_stay_in_bounds(ni, nj):
    cfg, s = _gam_state(ni, nj)
    lib = _capi.lib()
    lib.cbdiso_b200_set_stream(_stream())
    assert lib.cbdgam_b200_set_plm_theta(1.5) == 0
    gamma = cfg.gamma_law_index
    shape = s.p1.shape
    prd = Padded(shape)
    prd.view.copy_(torch.from_numpy(s.p1))
    u0 = Padded(shape)
    assert lib.cbdgam_2d_primitive_to_conserved(ni, nj, prd.ptr, u0.ptr, gamma) == 0
    wr = Padded(shape)
    m1, m2 = cfg.point_masses(s.time)
    buf = (cfg.buffer_surface_density, cfg.buffer_surface_pressure, m1.mass + m2.mass, cfg.buffer_driving_rate,
           s.buffer_outer_radius, cfg.buffer_onset_width, int(cfg.buffer_is_enabled))
    dt = 0.5 * og.driver_dt(s, 0.1)
    tail = (cfg.alpha, 0.5, dt, cfg.velocity_ceiling, cfg.cooling_coefficient, cfg.mach_ceiling,
            cfg.density_floor, cfg.pressure_floor, int(cfg.constant_softening))
    assert lib.cbdgam_2d_advance_rk(ni, nj, s.xl, s.xr, s.yl, s.yr, u0.ptr, prd.ptr, wr.ptr, gamma, *buf,
                                    *m1.args(), *m2.args(), *tail) == 0
    ws = Padded(shape[:2])
    assert lib.cbdgam_2d_wavespeed(ni, nj, prd.ptr, ws.ptr, gamma) == 0
    rate = Padded(shape)
    assert lib.cbdgam_2d_point_mass_source_term(ni, nj, s.xl, s.xr, s.yl, s.yr, *m1.args(), *m2.args(), 2,
                                                prd.ptr, rate.ptr, int(cfg.constant_softening), gamma) == 0

    g = _capi.GamGrid()
    g.ni, g.nj = ni, nj
    g.xl, g.xr, g.yl, g.yr = s.xl, s.xr, s.yl, s.yr
    g.plm_theta, g.gamma_law_index, g.alpha, g.cooling_coefficient = 1.5, gamma, cfg.alpha, 1.0
    g.mach_ceiling, g.velocity_ceiling = cfg.mach_ceiling, cfg.velocity_ceiling
    g.density_floor, g.pressure_floor, g.constant_softening = cfg.density_floor, cfg.pressure_floor, 1
    g.buffer_is_enabled, g.buffer_surface_density, g.buffer_surface_pressure = 1, 0.3, 3e-3
    g.buffer_driving_rate, g.buffer_outer_radius, g.buffer_onset_width = 1000.0, s.buffer_outer_radius, 0.1
    st = _capi.GamStage()
    _mass(m1, st.mass[0])
    _mass(m2, st.mass[1])
    st.buffer_central_mass, st.a, st.dt = m1.mass + m2.mass, 0.5, dt
    out = Padded(shape)
    wsmax = Padded((1,))
    assert lib.cbdgam_b200_advance_stage(ctypes.byref(g), ctypes.byref(st), prd.ptr, prd.ptr, out.ptr,
                                         wsmax.ptr, _stream()) == 0
    assert lib.cbdgam_b200_fill_guards(ctypes.byref(g), out.ptr, _stream()) == 0
    masses = (_capi.Mass * 2)()
    _mass(m1, masses[0])
    _mass(m2, masses[1])
    diags = (_capi.Diag * 2)()
    diags[0].quantity, diags[0].which_mass, diags[0].accretion = 1, 3, 1
    diags[1].quantity, diags[1].which_mass, diags[1].gravity = 4, 3, 1
    scratch = Padded((int(lib.cbdgam_b200_scratch_bytes(ctypes.byref(g))) // 8 + 8,))
    result = Padded((9,))
    assert lib.cbdgam_b200_reduce(ctypes.byref(g), masses, diags, 2, out.ptr, scratch.ptr, result.ptr,
                                  _stream()) == 0
    torch.cuda.synchronize()
    for a in (prd, u0, wr, ws, rate, out, wsmax, scratch, result):
        assert a.intact()
    assert np.isfinite(out.view[2:-2, 2:-2].cpu().numpy()).all()
    assert float(result.view[0].item()) == float(wsmax.view[0].item())
    if (ni, nj) == (257, 130):
        want = np.zeros_like(s.p1)
        s.k.advance_rk(cfg, s.xl, s.xr, s.yl, s.yr, u0.view.cpu().numpy(), s.p1, want, buf, m1, m2, 0.5, dt)
        got = wr.view.cpu().numpy()
        for q in range(4):
            scale = np.abs(want[2:-2, 2:-2, q]).max()
            assert np.abs(got[2:-2, 2:-2, q] - want[2:-2, 2:-2, q]).max() <= 1e-13 * scale
