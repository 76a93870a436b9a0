"""
The C-ABI library loads without a GPU, exports every entry point declared in
include/cbdiso_b200.h, and its struct layouts match the ctypes binding.
"""

import ctypes
import os
import re

from sailfish_b200 import _capi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "cbdiso_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:int|long|void|size_t|char)\s*\*?\s*(\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_binding_list():
    assert declared_functions() == sorted(_capi.exported_symbols())


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_capi.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_struct_layouts_match():
    c_sizes, py_sizes = _capi.abi_sizes()
    assert c_sizes == py_sizes


def test_host_only_entry_points():
    lib = _capi.lib()
    assert lib.cbdiso_b200_version() == 1
    assert lib.cbdiso_b200_status_string(1) == b"invalid argument"
    assert lib.cbdiso_b200_set_plm_theta(1.5) == 0
    assert lib.cbdiso_b200_set_plm_theta(3.0) == 1
    assert lib.cbdiso_b200_set_plm_theta(1.8) == 0
    assert lib.cbdiso_b200_set_precision(7) == 1
    g = _capi.Grid(ni=0, nj=4)
    assert lib.cbdiso_b200_scratch_bytes(ctypes.byref(g)) == 0
    assert lib.cbdiso_b200_fill_guards(ctypes.byref(g), None, None) == 1
    # drop-in kernels reject bad sizes before touching the device
    assert lib.cbdiso_2d_primitive_to_conserved(0, 4, None, None) == 1


def test_face_cache_and_adjoint_settings_host_checks():
    """Host-side checks of the face-cache and adjoint-segment entry points
    (nothing is launched)."""
    lib = _capi.lib()
    g = _capi.Grid(ni=8, nj=6, xl=-1.0, xr=1.0, yl=-1.0, yr=1.0, eos_type=2, mach2=100.0, plm_theta=1.5)
    # header, (cs^2, cs) pairs of every x- and y-face and (g_1, g_2) of every zone
    assert lib.cbdiso_b200_face_cache_bytes(ctypes.byref(g)) == 8 * (32 + 2 * (9 * 6 + 8 * 7 + 8 * 6))
    assert lib.cbdiso_b200_face_cache_bytes(ctypes.byref(_capi.Grid(ni=0, nj=6))) == 0
    st = _capi.Stage()
    a, b = ctypes.c_void_p(0x1000), ctypes.c_void_p(0x2000)
    args = (ctypes.byref(g), ctypes.byref(st), None, a, None, b, None, None, None)
    assert lib.cbdiso_b200_advance_stage_cached(*args, None, 2, None) == 1            # no cache
    assert lib.cbdiso_b200_advance_stage_cached(*args, ctypes.c_void_p(0x1008), 2, None) == 1  # not 16-byte aligned
    assert lib.cbdiso_b200_advance_stage_cached(*args, ctypes.c_void_p(0x3000), 3, None) == 1  # unknown role
    # disk records take an even, non-negative cache offset
    rec = (ctypes.c_char * int(lib.cbdiso_b200_batch_disk_bytes()))()
    assert lib.cbdiso_b200_batch_disk_set_face_cache(rec, -2) == 1
    assert lib.cbdiso_b200_batch_disk_set_face_cache(rec, 3) == 1
    assert lib.cbdiso_b200_batch_disk_set_face_cache(rec, 4096) == 0
    assert lib.cbdiso_b200_batch_disk_set_face_cache(None, 0) == 1
    # adjoint segment rows: 0 (the library's choice) or 4 .. 32
    assert lib.cbdiso_b200_set_adjoint_segment_rows(3) == 1
    assert lib.cbdiso_b200_set_adjoint_segment_rows(33) == 1
    assert lib.cbdiso_b200_set_adjoint_segment_rows(8) == 0
    assert lib.cbdiso_b200_set_adjoint_segment_rows(0) == 0
    # the gamma-law cache: header, zone (sqrt(w2), g_1) pairs and g_2, x- and y-faces
    gg = _capi.GamGrid(ni=8, nj=6, xl=-1.0, xr=1.0, yl=-1.0, yr=1.0, gamma_law_index=5.0 / 3.0, plm_theta=1.5)
    assert lib.cbdgam_b200_face_cache_bytes(ctypes.byref(gg)) == 8 * (32 + 3 * 48 + 9 * 6 + 8 * 7)
    gst = _capi.GamStage()
    assert lib.cbdgam_b200_advance_stage_cached(ctypes.byref(gg), ctypes.byref(gst), a, None, b, None,
                                                ctypes.c_void_p(0x1008), 2, None) == 1


def test_epilogue_rates_only_query():
    """The host query behind the batched stage's epilogue form: source rates
    of the masses without a radial cut qualify, anything else does not."""
    lib = _capi.lib()
    ep = _capi.Epilogue(want_wavespeed=1, num_diag=2)
    ep.diag[0] = _capi.Diag(quantity=1, which_mass=1, accretion=1)  # mdot of mass 1
    ep.diag[1] = _capi.Diag(quantity=4, which_mass=3, gravity=1)  # torque of both
    assert lib.cbdiso_b200_epilogue_rates_only(ctypes.byref(ep)) == 1
    ep.diag[1].has_cut = 1
    ep.diag[1].r0, ep.diag[1].r1 = 0.5, 2.0
    assert lib.cbdiso_b200_epilogue_rates_only(ctypes.byref(ep)) == 0
    ep.diag[1] = _capi.Diag(quantity=8, which_mass=1)  # total mass: not a rate
    assert lib.cbdiso_b200_epilogue_rates_only(ctypes.byref(ep)) == 0
    ep.num_diag = 0
    assert lib.cbdiso_b200_epilogue_rates_only(ctypes.byref(ep)) == 1
    ep.num_diag = _capi.MAX_DIAG + 1
    assert lib.cbdiso_b200_epilogue_rates_only(ctypes.byref(ep)) == -1
    ep.num_diag = 1
    ep.diag[0] = _capi.Diag(quantity=99, which_mass=1)
    assert lib.cbdiso_b200_epilogue_rates_only(ctypes.byref(ep)) == -1
    assert lib.cbdiso_b200_epilogue_rates_only(None) == -1
