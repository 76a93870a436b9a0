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
