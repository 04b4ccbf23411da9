"""ctypes binding of the product library libhc_b200.so (C ABI: include/hc_abi.h).

The library is built in-tree by heliocubed_b200.build.  There is no fallback:
if the library is missing or CUDA is unavailable every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhc_b200.so")

_D = C.POINTER(C.c_double)
_VP = C.c_void_p

HC_OK = 0
ERRORS = {-1: "HC_ERR_ARG", -2: "HC_ERR_CUDA", -3: "HC_ERR_UNSUPPORTED", -4: "HC_ERR_INVALID_STATE", -5: "HC_ERR_NOMEM"}

# Every function hc_abi.h declares, with its ctypes signature.
SIGNATURES = {
    "hc_last_error": (C.c_char_p, []),
    "hc_ctx_create": (C.c_int, [_VP, C.c_int, C.POINTER(_VP)]),
    "hc_ctx_destroy": (C.c_int, [_VP]),
    "hc_level_state_size": (C.c_size_t, [_VP]),
    "hc_level_primitive_size": (C.c_size_t, [_VP]),
    "hc_box_rhs": (C.c_int, [_VP, _VP, _VP, _VP, C.c_double, _VP, _VP, _VP]),
    "hc_box_gravity": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "hc_box_rhs_o4": (C.c_int, [_VP, _VP, _VP, C.c_double, _VP, _VP, _VP]),
    "hc_box_gravity_o4": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "hc_o4_batch_create": (C.c_int, [_VP, _VP, C.c_int, C.c_double, _VP]),
    "hc_o4_batch_rhs": (C.c_int, [_VP, _VP, _VP]),
    "hc_o4_batch_destroy": (C.c_int, [_VP]),
    "hc_ensemble_create": (C.c_int, [_VP, C.c_int, C.POINTER(_VP)]),
    "hc_ensemble_advance_cfl": (C.c_int, [_VP, _VP, C.c_int, _VP, _VP, _VP]),
    "hc_ensemble_destroy": (C.c_int, [_VP]),
    "hc_level_prepare": (C.c_int, [_VP, _VP, _VP, C.c_double, _VP]),
    "hc_level_rhs": (C.c_int, [_VP, _VP, _VP, _VP]),
    "hc_level_rk4_step": (C.c_int, [_VP, _VP, C.c_double, C.c_double, _VP]),
    "hc_level_rk4_stage": (C.c_int, [_VP, _VP, C.c_int, C.c_double, C.c_double, _VP, _VP, _VP]),
    "hc_level_set_radial_window": (C.c_int, [_VP, C.c_int, C.c_int]),
    "hc_level_stage_state": (C.c_int, [_VP, _VP, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_long),
                                       C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "hc_level_rk4_step_noalloc": (C.c_int, [_VP, _VP, C.c_double, C.c_double, _VP]),
    "hc_level_advance_cfl": (C.c_int, [_VP, _VP, C.c_int, _VP, _VP, _VP]),
    "hc_level_dt_cfl": (C.c_int, [_VP, _VP, _VP, _VP]),
    "hc_level_valid": (C.c_int, [_VP, _VP, _VP, _VP]),
    "hc_level_init": (C.c_int, [_VP, _VP, _VP, _VP]),
    "hc_geometry_export": (C.c_long, [_VP, C.c_int, _VP]),
    "hc_cone_prepare": (C.c_int, [_VP, C.c_double, _VP]),
    "hc_stage_tiles": (C.c_int, [_VP, C.c_int]),
    "hc_ctx_autotune": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "hc_ctx_set_tiles": (C.c_int, [_VP, C.c_int, C.c_int]),
    "hc_o4_variants": (C.c_int, [_VP, C.c_int]),
    "hc_amr_plan_create": (C.c_int, [_VP, _VP, C.c_int, _VP, C.c_int, _VP]),
    "hc_amr_plan_destroy": (C.c_int, [_VP]),
    "hc_amr_rk_stage": (C.c_int, [_VP, _VP, C.c_int, C.c_int, C.c_double, _VP]),
    "hc_amr_restrict": (C.c_int, [_VP, _VP, C.c_int, C.c_int, _VP]),
    "hc_amr_plan_set_reflux": (C.c_int, [_VP, _VP, C.c_int]),
    "hc_amr_reflux": (C.c_int, [_VP, _VP, C.c_int, C.c_int, _VP]),
    "hc_amr_cf_weights": (C.c_int, [C.c_int, C.c_int, _VP]),
    "hc_amr_plan_set_cf_interp": (C.c_int, [_VP, _VP, C.c_int]),
    "hc_amr_cf_interpolate": (C.c_int, [_VP, _VP, C.c_int, C.c_int, _VP]),
    "hc_amr_plan_set_cf_fine": (C.c_int, [_VP, _VP, C.c_int]),
    "hc_amr_plan_set_copies": (C.c_int, [_VP, _VP, C.c_int]),
    "hc_amr_copy": (C.c_int, [_VP, _VP, C.c_int, C.c_int, _VP]),
    "hc_amr_cf_mapped": (C.c_int, [_VP, _VP, C.c_int, C.c_int, _VP]),
    "hc_amr_cf_quotient": (C.c_int, [_VP, _VP, C.c_int, C.c_int, _VP]),
    "hc_amr_plan_set_native": (C.c_int, [_VP, _VP, C.c_int]),
    "hc_level_cartesian_size": (C.c_size_t, [_VP]),
    "hc_level_prepare_cartesian": (C.c_int, [_VP, _VP, _VP, _VP, C.c_double, _VP]),
    "hc_level_rhs_fluxes": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "hc_amr_native": (C.c_int, [_VP, _VP, C.c_int, C.c_int, C.c_double, _VP]),
    "hc_ctx_set_o4_variants": (C.c_int, [_VP, _VP]),
    "hc_level_insert_cone": (C.c_int, [_VP, _VP, C.c_double, _VP, _VP, _VP]),
    "hc_cone_event": (C.c_int, [_VP, _VP]),
    "hc_level_set_cme_schedule": (C.c_int, [_VP, _VP, C.c_int, _VP]),
    "hc_level_set_inlet": (C.c_int, [_VP, _VP, C.c_int, _VP]),
}


class HcParams(C.Structure):
    """hc_params of include/hc_abi.h (option semantics of src/Inputs_Parsing.H)."""
    _fields_ = [
        ("spatial_order", C.c_int), ("limiter", C.c_int), ("riemann_solver", C.c_int),
        ("divergence_cleaning", C.c_int), ("sun_gravity", C.c_int),
        ("init_condition_type", C.c_int), ("temporal_order", C.c_int),
        ("nr", C.c_int), ("na", C.c_int), ("spatial_operator", C.c_int), ("berta_detector_type", C.c_int),
        ("berta_fallback_type", C.c_int), ("autotune", C.c_int),
        ("radial_offset", C.c_int), ("radial_cells", C.c_int), ("reserved_i", C.c_int * 1),
        ("gamma", C.c_double), ("entropy_fix_coeff", C.c_double), ("cfl", C.c_double),
        ("inner_radius", C.c_double), ("outer_radius", C.c_double),
        ("radial_stretch", C.c_double), ("strength", C.c_double), ("berta_eta_d", C.c_double),
        ("reserved_d", C.c_double * 6),
    ]


class HcBox(C.Structure):
    _fields_ = [("lo", C.c_int * 3), ("hi", C.c_int * 3), ("ghost", C.c_int), ("block", C.c_int)]


class HcInit(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("pulse_block", C.c_int), ("pulse_i", C.c_int), ("pulse_j", C.c_int),
        ("pulse_k", C.c_int), ("reserved_i", C.c_int * 3),
        ("rho0", C.c_double), ("p0", C.c_double), ("vr", C.c_double), ("b0", C.c_double),
        ("r_ref", C.c_double), ("pulse_amp", C.c_double), ("pulse_width", C.c_double),
        ("reserved_d", C.c_double * 4),
    ]


class HcBoxWork(C.Structure):
    """Mirror of hc_box_work in include/hc_abi.h."""
    _fields_ = [("box", HcBox), ("usph", C.c_void_p), ("rhs", C.c_void_p), ("flux", C.c_void_p * 3)]


_CONE_SPEC = ("lat_deg", "lon_deg", "half_angle_deg", "apex_speed", "wind_speed", "drag_gamma",
              "reference_height", "reference_time", "density", "temperature")
_CONE = ("radius", "entry_shift", "entry_time", "speed", "end_time", "insertion_time", "density", "temperature")


class HcConeSpec(C.Structure):
    """Mirror of hc_cone_spec in include/hc_abi.h."""
    _fields_ = [(n, C.c_double) for n in _CONE_SPEC] + [("reserved", C.c_double * 6)]


class HcCone(C.Structure):
    """Mirror of hc_cone in include/hc_abi.h."""
    _fields_ = [("axis", C.c_double * 3)] + [(n, C.c_double) for n in _CONE] + [("reserved", C.c_double * 6)]


class HcRkBox(C.Structure):
    """Mirror of hc_rk_box in include/hc_abi.h."""
    _fields_ = [("ncells", C.c_longlong), ("state", C.c_void_p), ("stage", C.c_void_p), ("rk", C.c_void_p * 4)]


class HcRestrictBox(C.Structure):
    """Mirror of hc_restrict_box in include/hc_abi.h."""
    _fields_ = [("fine", C.c_void_p), ("coarse", C.c_void_p), ("fine_lo", C.c_int * 3), ("fine_n", C.c_int * 3),
                ("coarse_lo", C.c_int * 3), ("coarse_n", C.c_int * 3), ("lo", C.c_int * 3), ("hi", C.c_int * 3),
                ("ratio", C.c_int * 3), ("reserved", C.c_int)]


class HcRefluxBox(C.Structure):
    """Mirror of hc_reflux_box in include/hc_abi.h."""
    _fields_ = [("fine_flux", C.c_void_p), ("coarse_flux", C.c_void_p), ("rhs", C.c_void_p),
                ("fine_lo", C.c_int * 3), ("fine_n", C.c_int * 3), ("coarse_lo", C.c_int * 3),
                ("coarse_n", C.c_int * 3), ("rhs_lo", C.c_int * 3), ("rhs_n", C.c_int * 3), ("lo", C.c_int * 3),
                ("hi", C.c_int * 3), ("ratio", C.c_int * 3), ("dir", C.c_int), ("fine_side", C.c_int),
                ("reserved", C.c_int), ("scale", C.c_double)]


class HcCfBox(C.Structure):
    """Mirror of hc_cf_box in include/hc_abi.h."""
    _fields_ = [("coarse", C.c_void_p), ("fine", C.c_void_p), ("coarse_lo", C.c_int * 3), ("coarse_n", C.c_int * 3),
                ("fine_lo", C.c_int * 3), ("fine_n", C.c_int * 3), ("valid_lo", C.c_int * 3),
                ("valid_hi", C.c_int * 3), ("ratio", C.c_int * 3), ("ncomp", C.c_int)]


class HcCopyBox(C.Structure):
    """Mirror of hc_copy_box in include/hc_abi.h."""
    _fields_ = [("src", C.c_void_p), ("dst", C.c_void_p), ("src_lo", C.c_int * 3), ("src_n", C.c_int * 3),
                ("dst_lo", C.c_int * 3), ("dst_n", C.c_int * 3), ("lo", C.c_int * 3), ("hi", C.c_int * 3),
                ("perm", C.c_int * 3), ("sign", C.c_int * 3), ("shift", C.c_int * 3), ("ncomp", C.c_int)]


class HcCfFineBox(C.Structure):
    """Mirror of hc_cf_fine_box in include/hc_abi.h."""
    _fields_ = [("jac", C.c_void_p), ("donor", C.c_void_p), ("state", C.c_void_p), ("mapped", C.c_void_p),
                ("out", C.c_void_p), ("jac_lo", C.c_int * 3), ("jac_n", C.c_int * 3), ("donor_lo", C.c_int * 3),
                ("donor_n", C.c_int * 3), ("state_lo", C.c_int * 3), ("state_n", C.c_int * 3),
                ("mapped_lo", C.c_int * 3), ("mapped_n", C.c_int * 3), ("out_lo", C.c_int * 3),
                ("out_n", C.c_int * 3), ("valid_lo", C.c_int * 3), ("valid_hi", C.c_int * 3),
                ("block_lo", C.c_int * 3), ("block_hi", C.c_int * 3)]


class HcNativeBox(C.Structure):
    """Mirror of hc_native_box in include/hc_abi.h."""
    _fields_ = [("cart", C.c_void_p), ("usph", C.c_void_p), ("cart_lo", C.c_int * 3), ("cart_n", C.c_int * 3),
                ("usph_lo", C.c_int * 3), ("usph_n", C.c_int * 3), ("block", C.c_int)]


class HcCmeEvent(C.Structure):
    """Mirror of hc_cme_event in include/hc_abi.h."""
    _fields_ = [("insertion_time", C.c_double), ("feeding_end", C.c_double), ("boundary", C.c_int),
                ("reserved", C.c_int)]


class HcError(RuntimeError):
    pass


_lib = None


def lib() -> C.CDLL:
    """Load libhc_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise HcError(f"{LIB_PATH} is missing: build it with `python -m heliocubed_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str) -> None:
    if rc != HC_OK:
        msg = lib().hc_last_error().decode(errors="replace")
        raise HcError(f"{what} failed: {ERRORS.get(rc, rc)}: {msg}")
