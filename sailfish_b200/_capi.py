"""
ctypes binding of libcbdiso_b200.so (include/cbdiso_b200.h).

The library is loaded from the package directory, where
`python -m sailfish_b200._build` (or __graft_entry__.build()) puts it. There is
no fallback: if the library is missing, `lib()` raises.
"""

import ctypes
import os
from ctypes import POINTER, Structure, c_double, c_int, c_size_t, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcbdiso_b200.so")

CBD_OK = 0
NONFINITE = 3  # CBD_ERR_NONFINITE
STATUS = {
    0: "success",
    1: "invalid argument",
    2: "CUDA runtime error",
    3: "non-finite value",
    4: "device wait timed out",
    5: "Kepler solve did not converge",
    6: "request exceeds library capacity",
}
PRECISION = {"exact": 0, "fma": 1, "fast": 2}
MAX_DIAG = 16
MAX_FUSED = 4
QUANTITY = dict(mdot=1, fx=2, fy=3, torque=4, sigma_m1=5, eccentricity_vector=6, angular_momentum=7, mass=8,
                power=9)


class CbdError(RuntimeError):
    """A libcbdiso_b200 entry point returned a non-zero status."""

    def __init__(self, status, where=""):
        self.status = status
        super().__init__(f"{where}: {STATUS.get(status, 'unknown status')} (status {status})")


class Mass(Structure):
    _fields_ = [("x", c_double), ("y", c_double), ("vx", c_double), ("vy", c_double), ("mass", c_double),
                ("softening_length", c_double), ("sink_rate", c_double), ("sink_radius", c_double),
                ("sink_model", c_int), ("_pad0", c_int)]


class Grid(Structure):
    _fields_ = [("ni", c_int), ("nj", c_int), ("xl", c_double), ("xr", c_double), ("yl", c_double),
                ("yr", c_double), ("plm_theta", c_double), ("eos_type", c_int), ("precision", c_int),
                ("cs2", c_double), ("mach2", c_double), ("nu", c_double), ("velocity_ceiling", c_double),
                ("density_floor", c_double), ("buffer_is_enabled", c_int), ("tile_columns", c_int),
                ("tile_rows", c_int), ("tile_occupancy", c_int), ("buffer_surface_density", c_double),
                ("buffer_driving_rate", c_double), ("buffer_outer_radius", c_double),
                ("buffer_onset_width", c_double)]


class Stage(Structure):
    _fields_ = [("mass", Mass * 2), ("a", c_double), ("dt", c_double), ("buffer_central_mass", c_double)]


class Diag(Structure):
    _fields_ = [("quantity", c_int), ("which_mass", c_int), ("gravity", c_int), ("accretion", c_int),
                ("has_cut", c_int), ("_pad", c_int), ("r0", c_double), ("r1", c_double)]


class Orbit(Structure):
    _fields_ = [("semimajor_axis", c_double), ("total_mass", c_double), ("mass_ratio", c_double),
                ("eccentricity", c_double), ("softening_length", c_double), ("sink_rate", c_double),
                ("sink_radius", c_double), ("sink_model", c_int), ("has_x_offset", c_int), ("x_offset", c_double)]


class Epilogue(Structure):
    _fields_ = [("mass", Mass * 2), ("want_wavespeed", c_int), ("num_diag", c_int), ("diag", Diag * MAX_DIAG)]


class GamGrid(Structure):
    """cbdgam_grid_t: a gamma-law run's mesh, physics and options."""

    _fields_ = [("ni", c_int), ("nj", c_int), ("xl", c_double), ("xr", c_double), ("yl", c_double),
                ("yr", c_double), ("plm_theta", c_double), ("gamma_law_index", c_double), ("alpha", c_double),
                ("cooling_coefficient", c_double), ("mach_ceiling", c_double), ("velocity_ceiling", c_double),
                ("density_floor", c_double), ("pressure_floor", c_double), ("constant_softening", c_int),
                ("buffer_is_enabled", c_int), ("buffer_surface_density", c_double),
                ("buffer_surface_pressure", c_double), ("buffer_driving_rate", c_double),
                ("buffer_outer_radius", c_double), ("buffer_onset_width", c_double)]


class GamStage(Structure):
    """cbdgam_stage_t: what changes per gamma-law RK stage."""

    _fields_ = [("mass", Mass * 2), ("buffer_central_mass", c_double), ("a", c_double), ("dt", c_double)]


GAM_MAX_DIAG = 4


_lib = None
_DP = POINTER(c_double)


def _declare(lib):
    I, D, P, V = c_int, c_double, c_void_p, c_void_p
    m9 = [D] * 8 + [I]
    sig = {
        "cbdiso_2d_advance_rk": [I, I, D, D, D, D, P, P, P, D, D, D, D, D, I] + m9 + m9 + [D, D, I, D, D, D, D, D],
        "cbdiso_2d_primitive_to_conserved": [I, I, P, P],
        "cbdiso_2d_point_mass_source_term": [I, I, D, D, D, D] + m9 + [P, P],
        "cbdiso_2d_wavespeed": [I, I, D, D, D, D, D, D, I] + m9 + m9 + [P, P],
        "cbdiso_b200_set_stream": [V],
        "cbdiso_b200_set_plm_theta": [D],
        "cbdiso_b200_set_precision": [I],
        "cbdiso_b200_version": [],
        "cbdiso_b200_fill_guards": [POINTER(Grid), P, V],
        "cbdiso_b200_advance_stage": [POINTER(Grid), POINTER(Stage), P, P, P, P, POINTER(Epilogue), P, P, V],
        "cbdiso_b200_advance_stage_noalloc": [POINTER(Grid), POINTER(Stage), P, P, P, P, POINTER(Epilogue), P, V],
        "cbdiso_b200_advance_stage_cached": [POINTER(Grid), POINTER(Stage), P, P, P, P, POINTER(Epilogue), P, P, P,
                                             I, V],
        "cbdiso_b200_reduce": [POINTER(Grid), POINTER(Epilogue), P, P, P, V],
        "cbdiso_b200_epilogue_rates_only": [POINTER(Epilogue)],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = c_int
    lib.cbdiso_b200_scratch_bytes.argtypes = [POINTER(Grid)]
    lib.cbdiso_b200_scratch_bytes.restype = c_size_t
    lib.cbdiso_b200_face_cache_bytes.argtypes = [POINTER(Grid)]
    lib.cbdiso_b200_face_cache_bytes.restype = c_size_t
    lib.cbdiso_b200_stage_record_bytes.argtypes = []
    lib.cbdiso_b200_stage_record_bytes.restype = c_size_t
    lib.cbdiso_b200_stage_record.argtypes = [POINTER(Grid), POINTER(Stage), POINTER(Epilogue), c_void_p]
    lib.cbdiso_b200_stage_record.restype = c_int
    lib.cbdiso_b200_eval_primitives.argtypes = [ctypes.c_long, c_void_p, c_void_p, c_void_p, c_void_p]
    lib.cbdiso_b200_eval_primitives.restype = c_int
    lib.cbdiso_b200_stepper_bytes.argtypes = []
    lib.cbdiso_b200_stepper_bytes.restype = c_size_t
    lib.cbdiso_b200_stepper_init.argtypes = [POINTER(Grid), POINTER(Orbit), c_int, c_double, c_double, c_double,
                                             c_double, c_int, c_void_p]
    lib.cbdiso_b200_stepper_init.restype = c_int
    lib.cbdiso_b200_stepper_attach.argtypes = [c_void_p, c_void_p, c_int, c_void_p, c_int]
    lib.cbdiso_b200_stepper_attach.restype = c_int
    lib.cbdiso_b200_step_prologue.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p]
    lib.cbdiso_b200_step_prologue.restype = c_int
    lib.cbdiso_b200_batch_disk_bytes.argtypes = []
    lib.cbdiso_b200_batch_disk_bytes.restype = c_size_t
    lib.cbdiso_b200_batch_disk_record.argtypes = [POINTER(Grid), POINTER(Epilogue), c_int, c_int,
                                                  ctypes.c_longlong, c_int, POINTER(c_int), c_void_p]
    lib.cbdiso_b200_batch_disk_record.restype = c_int
    lib.cbdiso_b200_batched_stage.argtypes = [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                              c_int, c_int, c_int, c_void_p, c_void_p, c_int, c_void_p]
    lib.cbdiso_b200_batched_stage.restype = c_int
    lib.cbdiso_b200_batched_stage_cached.argtypes = [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p,
                                                     c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_int,
                                                     c_void_p, c_int, c_void_p]
    lib.cbdiso_b200_batched_stage_cached.restype = c_int
    lib.cbdiso_b200_batch_disk_set_face_cache.argtypes = [c_void_p, ctypes.c_longlong]
    lib.cbdiso_b200_batch_disk_set_face_cache.restype = c_int
    lib.cbdiso_b200_batched_finalize.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_int, c_void_p]
    lib.cbdiso_b200_batched_finalize.restype = c_int
    lib.cbdiso_b200_batched_prologue.argtypes = [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p, c_int,
                                                 c_int, c_void_p]
    lib.cbdiso_b200_batched_prologue.restype = c_int
    lib.cbdiso_b200_adjoint_workspace_bytes.argtypes = [POINTER(Grid)]
    lib.cbdiso_b200_adjoint_workspace_bytes.restype = c_size_t
    lib.cbdiso_b200_set_adjoint_variant.argtypes = [c_int]
    lib.cbdiso_b200_set_adjoint_variant.restype = c_int
    lib.cbdiso_b200_set_adjoint_segment_rows.argtypes = [c_int]
    lib.cbdiso_b200_set_adjoint_segment_rows.restype = c_int
    lib.cbdiso_b200_adjoint_chain_blocks.argtypes = [POINTER(Grid)]
    lib.cbdiso_b200_adjoint_chain_blocks.restype = c_size_t
    V = c_void_p
    D = c_double
    for name, args in {
        "cbdiso_b200_stage_record_branches": [POINTER(Grid), V, V, V, V, V],
        "cbdiso_b200_stage_tangent": [POINTER(Grid), V, V, D, D, V, V, V, V, V, V, V],
        "cbdiso_b200_stage_adjoint": [POINTER(Grid), V, V, V, V, V, V, V, V, V, V, V],
        "cbdiso_b200_objective_tangent": [POINTER(Grid), V, V, D, V, V, D, D, V, c_int, V],
        "cbdiso_b200_objective_adjoint": [POINTER(Grid), V, V, D, D, V, V, V, V],
        "cbdiso_b200_stage_adjoint_chained": [POINTER(Grid), V, V, V, V, V, V, V, V, V, V, V],
        "cbdiso_b200_objective_adjoint_chained": [POINTER(Grid), V, V, D, D, V, V, V, V, V],
        "cbdiso_b200_adjoint_chain_finish": [V, c_int, V, V],
    }.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = c_int
    m9 = [D] * 8 + [I]
    for name, args in {
        "cbdgam_2d_advance_rk": [I, I, D, D, D, D, V, V, V, D, D, D, D, D, D, D, I] + m9 + m9
        + [D, D, D, D, D, D, D, D, I],
        "cbdgam_2d_wavespeed": [I, I, V, V, D],
        "cbdgam_2d_primitive_to_conserved": [I, I, V, V, D],
        "cbdgam_2d_point_mass_source_term": [I, I, D, D, D, D] + m9 + m9 + [I, V, V, I, D],
        "cbdgam_b200_set_plm_theta": [D],
        "cbdgam_b200_advance_stage": [POINTER(GamGrid), POINTER(GamStage), V, V, V, V, V],
        "cbdgam_b200_advance_stage_cached": [POINTER(GamGrid), POINTER(GamStage), V, V, V, V, V, I, V],
        "cbdgam_b200_fill_guards": [POINTER(GamGrid), V, V],
        "cbdgam_b200_reduce": [POINTER(GamGrid), POINTER(Mass), POINTER(Diag), c_int, V, V, V, V],
        "cbdgam_b200_eval_powers": [ctypes.c_long, V, V, V],
    }.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = c_int
    lib.cbdiso_b200_fp64_probe.argtypes = [ctypes.c_long, c_int, c_void_p, c_void_p]
    lib.cbdiso_b200_fp64_probe.restype = c_int
    lib.cbdiso_b200_fp64_probe_fmas.argtypes = [ctypes.c_long, c_int]
    lib.cbdiso_b200_fp64_probe_fmas.restype = ctypes.c_long
    lib.cbdgam_b200_disk_primitive.argtypes = [ctypes.c_long, c_void_p, c_void_p, c_double, c_double, c_double,
                                               c_void_p]
    lib.cbdgam_b200_disk_primitive.restype = None
    lib.cbdgam_b200_scratch_bytes.argtypes = [POINTER(GamGrid)]
    lib.cbdgam_b200_scratch_bytes.restype = c_size_t
    lib.cbdgam_b200_face_cache_bytes.argtypes = [POINTER(GamGrid)]
    lib.cbdgam_b200_face_cache_bytes.restype = c_size_t
    lib.cbdgam_b200_abi_sizes.argtypes = [POINTER(c_size_t)]
    lib.cbdgam_b200_abi_sizes.restype = None
    lib.cbdiso_b200_abi_sizes.argtypes = [POINTER(c_size_t)]
    lib.cbdiso_b200_abi_sizes.restype = None
    lib.cbdiso_b200_status_string.argtypes = [c_int]
    lib.cbdiso_b200_status_string.restype = ctypes.c_char_p
    return lib


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m sailfish_b200._build` "
                "(there is no CPU fallback)")
        _lib = _declare(ctypes.CDLL(LIB_PATH))
    return _lib


def check(status, where=""):
    if status != CBD_OK:
        raise CbdError(status, where)


def exported_symbols():
    """Names declared in include/cbdiso_b200.h (for the export test)."""
    return [
        "cbdiso_2d_advance_rk", "cbdiso_2d_primitive_to_conserved", "cbdiso_2d_point_mass_source_term",
        "cbdiso_2d_wavespeed", "cbdiso_b200_set_stream", "cbdiso_b200_set_plm_theta", "cbdiso_b200_set_precision",
        "cbdiso_b200_status_string", "cbdiso_b200_version", "cbdiso_b200_scratch_bytes", "cbdiso_b200_fill_guards",
        "cbdiso_b200_advance_stage", "cbdiso_b200_reduce", "cbdiso_b200_abi_sizes",
        "cbdiso_b200_stage_record_bytes", "cbdiso_b200_stage_record", "cbdiso_b200_eval_primitives",
        "cbdiso_b200_advance_stage_noalloc", "cbdiso_b200_face_cache_bytes", "cbdiso_b200_advance_stage_cached",
        "cbdiso_b200_stepper_bytes", "cbdiso_b200_stepper_init",
        "cbdiso_b200_step_prologue", "cbdiso_b200_batch_disk_bytes", "cbdiso_b200_batch_disk_record",
        "cbdiso_b200_batched_stage", "cbdiso_b200_batched_finalize", "cbdiso_b200_batched_prologue",
        "cbdiso_b200_batched_stage_cached", "cbdiso_b200_batch_disk_set_face_cache", "cbdiso_b200_epilogue_rates_only",
        "cbdiso_b200_adjoint_workspace_bytes", "cbdiso_b200_stage_record_branches", "cbdiso_b200_stage_tangent",
        "cbdiso_b200_stage_adjoint", "cbdiso_b200_objective_tangent", "cbdiso_b200_objective_adjoint",
        "cbdiso_b200_stepper_attach", "cbdiso_b200_stage_adjoint_chained", "cbdiso_b200_objective_adjoint_chained",
        "cbdiso_b200_adjoint_chain_finish", "cbdiso_b200_adjoint_chain_blocks",
        "cbdiso_b200_set_adjoint_variant", "cbdiso_b200_set_adjoint_segment_rows",
        "cbdgam_2d_advance_rk", "cbdgam_2d_wavespeed", "cbdgam_2d_primitive_to_conserved",
        "cbdgam_2d_point_mass_source_term", "cbdgam_b200_set_plm_theta", "cbdgam_b200_advance_stage",
        "cbdgam_b200_face_cache_bytes", "cbdgam_b200_advance_stage_cached",
        "cbdgam_b200_fill_guards", "cbdgam_b200_scratch_bytes", "cbdgam_b200_reduce", "cbdgam_b200_abi_sizes",
        "cbdgam_b200_eval_powers", "cbdiso_b200_fp64_probe", "cbdiso_b200_fp64_probe_fmas",
        "cbdgam_b200_disk_primitive",
    ]


def abi_sizes():
    """(C sizes, ctypes sizes) of the public structs: cbd_mass_t,
    cbd_grid_t, cbd_stage_t, cbd_epilogue_t, cbdgam_grid_t, cbdgam_stage_t."""
    out = (c_size_t * 4)()
    lib().cbdiso_b200_abi_sizes(out)
    gam = (c_size_t * 2)()
    lib().cbdgam_b200_abi_sizes(gam)
    return list(out) + list(gam), [ctypes.sizeof(t) for t in (Mass, Grid, Stage, Epilogue, GamGrid, GamStage)]
