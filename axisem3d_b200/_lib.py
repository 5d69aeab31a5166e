"""ctypes binding of the engine's C ABI (include/axg.h).

The shared library is built in-tree (axisem3d_b200/libaxg.so) by
``axisem3d_b200.build``; importing this module never falls back to anything
else: a missing library raises immediately.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaxg.so")

AXG_OK = 0
AXG_E_ARG, AXG_E_STATE, AXG_E_CUDA, AXG_E_UNSTABLE, AXG_E_NOMEM, AXG_E_UNSUPPORTED = -1, -2, -3, -4, -5, -6
AXG_FP64, AXG_FP32, AXG_MIXED = 0, 1, 2
AXG_ISO, AXG_TISO, AXG_ANISO = 0, 1, 2
AXG_ATT_NONE, AXG_ATT_FULL, AXG_ATT_CG4 = 0, 1, 2
AXG_FIELD_STIFF, AXG_FIELD_DISPL, AXG_FIELD_VELOC, AXG_FIELD_ACCEL = 0, 1, 2, 3
AXG_MAP_LINEAR, AXG_MAP_SPHERICAL, AXG_MAP_SEMI_SPHERICAL = 0, 1, 2
AXG_MAX_SLS = 8

PRECISIONS = {"fp64": AXG_FP64, "fp32": AXG_FP32, "mixed": AXG_MIXED}

P_i32 = C.POINTER(C.c_int32)
P_i64 = C.POINTER(C.c_int64)
P_u8 = C.POINTER(C.c_uint8)
P_f64 = C.POINTER(C.c_double)


class axg_config(C.Structure):
    _fields_ = [("precision", C.c_int32), ("device", C.c_int32), ("dt", C.c_double),
                ("t0", C.c_double), ("nsls", C.c_int32),
                ("att_alpha", C.c_double * AXG_MAX_SLS), ("att_beta", C.c_double * AXG_MAX_SLS),
                ("att_gamma", C.c_double * AXG_MAX_SLS), ("stability_interval", C.c_int32),
                ("deterministic", C.c_int32), ("compensated", C.c_int32), ("plain", C.c_int32),
                ("autotune", C.c_int32), ("nwave", C.c_int32)]


class axg_solid_points(C.Structure):
    _fields_ = [("count", C.c_int32), ("nr", P_i32), ("mass_nr", P_i32), ("mass_offset", P_i64),
                ("mass", P_f64), ("axial", P_u8)]


class axg_fluid_points(C.Structure):
    _fields_ = [("count", C.c_int32), ("nr", P_i32), ("mass_nr", P_i32), ("mass_offset", P_i64),
                ("mass", P_f64), ("axial", P_u8), ("surface", P_u8)]


class axg_solid_elements(C.Structure):
    _fields_ = [("count", C.c_int32), ("nr", P_i32), ("points", P_i32), ("axial", P_u8),
                ("geometry", P_f64), ("rtz", P_u8), ("theta", P_f64), ("rheology", P_i32),
                ("is3d", P_u8), ("mat_offset", P_i64), ("moduli", P_f64), ("attenuation", P_i32),
                ("att_offset", P_i64), ("att_moduli", P_f64)]


class axg_fluid_elements(C.Structure):
    _fields_ = [("count", C.c_int32), ("nr", P_i32), ("points", P_i32), ("axial", P_u8),
                ("geometry", P_f64), ("is3d", P_u8), ("mat_offset", P_i64), ("moduli", P_f64)]


class axg_solid_fluid(C.Structure):
    _fields_ = [("count", C.c_int32), ("solid_point", P_i32), ("fluid_point", P_i32),
                ("ns_unassembled", P_f64), ("nz_unassembled", P_f64), ("ns_assembled", P_f64),
                ("nz_assembled", P_f64), ("mass_fluid", P_f64)]


class axg_stf(C.Structure):
    _fields_ = [("half_duration", C.c_double), ("decay_factor", C.c_double),
                ("time_shift", C.c_double), ("derivative_order", C.c_int32)]


class axg_moment_sources(C.Structure):
    _fields_ = [("count", C.c_int32), ("element", P_i32), ("nu", P_i32), ("pattern_offset", P_i64),
                ("pattern", P_f64), ("stf", C.POINTER(axg_stf)), ("wavefield", P_i32)]


class axg_force_sources(C.Structure):
    _fields_ = [("count", C.c_int32), ("element", P_i32), ("nu", P_i32), ("pattern_offset", P_i64),
                ("pattern", P_f64), ("stf", C.POINTER(axg_stf)), ("wavefield", P_i32)]


class axg_pressure_sources(C.Structure):
    _fields_ = [("count", C.c_int32), ("element", P_i32), ("nu", P_i32), ("pattern_offset", P_i64),
                ("pattern", P_f64), ("stf", C.POINTER(axg_stf)), ("wavefield", P_i32)]


class axg_stations(C.Structure):
    _fields_ = [("count", C.c_int32), ("element", P_i32), ("weights", P_f64), ("phi", P_f64)]


class axg_clayton(C.Structure):
    _fields_ = [("count", C.c_int32), ("point", P_i32), ("rho_vp", P_f64), ("rho_vs", P_f64),
                ("area", P_f64), ("theta", P_f64)]


class axg_clayton3d(C.Structure):
    _fields_ = [("count", C.c_int32), ("point", P_i32), ("offset", P_i64), ("nvalues", C.c_int64),
                ("rho_vp", P_f64), ("rho_vs", P_f64), ("area", P_f64), ("normal", P_f64)]


class axg_scanning(C.Structure):
    _fields_ = [("tol_fourier_h1", C.c_double), ("rel_tol_h1", C.c_double), ("abs_tol_h1", C.c_double),
                ("max_num_peaks", C.c_int32), ("interval", C.c_int32), ("n_solid", C.c_int32),
                ("solid_points", P_i32), ("n_fluid", C.c_int32), ("fluid_points", P_i32)]


AXG_SCAN_MAX_PEAKS = 32

# name -> (restype, argtypes) of every entry point declared in include/axg.h
H = C.c_void_p
SIGNATURES = {
    "axg_create": (C.c_int, [C.POINTER(axg_config), C.POINTER(H)]),
    "axg_destroy": (C.c_int, [H]),
    "axg_last_error": (C.c_char_p, [H]),
    "axg_version": (C.c_char_p, []),
    "axg_set_solid_points": (C.c_int, [H, C.POINTER(axg_solid_points)]),
    "axg_set_fluid_points": (C.c_int, [H, C.POINTER(axg_fluid_points)]),
    "axg_set_solid_elements": (C.c_int, [H, C.POINTER(axg_solid_elements)]),
    "axg_set_fluid_elements": (C.c_int, [H, C.POINTER(axg_fluid_elements)]),
    "axg_set_solid_fluid": (C.c_int, [H, C.POINTER(axg_solid_fluid)]),
    "axg_set_moment_sources": (C.c_int, [H, C.POINTER(axg_moment_sources)]),
    "axg_set_force_sources": (C.c_int, [H, C.POINTER(axg_force_sources)]),
    "axg_set_pressure_sources": (C.c_int, [H, C.POINTER(axg_pressure_sources)]),
    "axg_set_solid_fluid3d": (C.c_int, [H, C.c_int32, P_i32, P_i32, P_i64, C.c_int64, P_f64, P_f64, P_f64]),
    "axg_set_stf_table": (C.c_int, [H, C.c_int32, C.c_int32, C.c_int32, P_f64, P_f64, C.c_int32, C.c_double,
                                     C.c_double, C.c_int32]),
    "axg_set_stations": (C.c_int, [H, C.POINTER(axg_stations), C.c_int32]),
    "axg_set_clayton": (C.c_int, [H, C.c_int32, C.POINTER(axg_clayton)]),
    "axg_set_sponge": (C.c_int, [H, C.c_int32, C.c_int32, P_i32, P_f64]),
    "axg_set_ocean_load": (C.c_int, [H, C.c_int32, P_i32, P_f64, P_f64]),
    "axg_set_ocean_load3d": (C.c_int, [H, C.c_int32, P_i32, P_i64, C.c_int64, P_f64, P_f64]),
    "axg_set_clayton3d": (C.c_int, [H, C.c_int32, C.POINTER(axg_clayton3d)]),
    "axg_set_scanning": (C.c_int, [H, C.POINTER(axg_scanning)]),
    "axg_set_prt": (C.c_int, [H, C.c_int32, P_i32, P_i64, P_u8, C.c_int64, P_f64]),
    "axg_set_prt_fluid": (C.c_int, [H, C.c_int32, P_i32, P_i64, P_u8, C.c_int64, P_f64, P_f64]),
    "axg_scanning_nr": (C.c_int, [H, P_i32, P_i32]),
    "axg_set_sponge3d": (C.c_int, [H, C.c_int32, C.c_int32, P_i32, P_i64, C.c_int64, P_f64]),
    "axg_finalize": (C.c_int, [H]),
    "axg_apply_sources": (C.c_int, [H, C.c_int32]),
    "axg_compute_stiffness": (C.c_int, [H]),
    "axg_compute_stiffness_noalloc": (C.c_int, [H, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "axg_set_adjoint_slices": (C.c_int, [H, C.c_int32]),
    "axg_get_adjoint_slices": (C.c_int, [H, P_f64, P_f64]),
    "axg_gather_stiffness": (C.c_int, [H, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p]),
    "axg_set_element_parts": (C.c_int, [H, C.c_void_p, C.c_void_p]),
    "axg_compute_stiffness_part": (C.c_int, [H, C.c_int32]),
    "axg_scatter_add_stiffness": (C.c_int, [H, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p]),
    "axg_apply_bc_before_assembly": (C.c_int, [H]),
    "axg_apply_bc_after_assembly": (C.c_int, [H]),
    "axg_stiff_to_accel": (C.c_int, [H]),
    "axg_newmark_update": (C.c_int, [H]),
    "axg_record_stations": (C.c_int, [H, C.c_int32]),
    "axg_run": (C.c_int, [H, C.c_int32, C.c_int32]),
    "axg_current_step": (C.c_int, [H, P_i32]),
    "axg_get_field": (C.c_int, [H, C.c_int32, C.c_int32, P_f64]),
    "axg_set_field": (C.c_int, [H, C.c_int32, C.c_int32, P_f64]),
    "axg_field_size": (C.c_int, [H, C.c_int32, P_i64]),
    "axg_get_seismograms": (C.c_int, [H, P_f64, P_i32]),
    "axg_get_station_gradients": (C.c_int, [H, P_f64, P_i32]),
    "axg_set_station_gradient": (C.c_int, [H, C.c_int32]),
    "axg_forward_checkpointed": (C.c_int, [H, C.c_int32, C.c_int32]),
    "axg_adjoint_run": (C.c_int, [H, P_f64, P_f64, P_f64, P_f64, P_f64]),
    "axg_field_raw_bytes": (C.c_int, [H, C.c_int32, C.c_int32, P_i64]),
    "axg_set_field_raw": (C.c_int, [H, C.c_int32, C.c_int32, C.c_void_p, C.c_int64]),
    "axg_get_field_raw": (C.c_int, [H, C.c_int32, C.c_int32, C.c_void_p, C.c_int64]),
    "axg_set_element_record": (C.c_int, [H, C.c_int32, P_i32, P_i32, P_i32, C.c_int32, C.c_int32]),
    "axg_element_record_words": (C.c_int, [H, P_i64]),
    "axg_get_element_records": (C.c_int, [H, C.c_int32, C.c_int32, P_f64]),
    "axg_synchronize": (C.c_int, [H]),
    "axg_launch_count": (C.c_int, [H, P_i64]),
    "axg_set_timing": (C.c_int, [H, C.c_int32]),
    "axg_stiffness_time_ms": (C.c_int, [H, P_f64, P_i64]),
    "axg_stiffness_cost": (C.c_int, [H, P_f64, P_f64]),
    "axg_point_cost": (C.c_int, [H, P_f64]),
    "axg_set_stream": (C.c_int, [H, C.c_void_p]),
    "axg_set_team_size": (C.c_int, [H, C.c_int32, C.c_int32]),
    "axg_spectral_tables": (C.c_int, [P_f64] * 6),
    "axg_quad_geometry": (C.c_int, [C.c_int32, P_f64, C.c_int32, P_f64, P_f64]),
    "axg_quad_geometry_batch": (C.c_int, [C.c_int32, C.c_int32, P_f64, P_u8, P_f64, P_f64]),
    "axg_quad_map": (C.c_int, [C.c_int32, P_f64, C.c_double, C.c_double, P_f64]),
    "axg_quad_dt": (C.c_int, [P_f64, C.c_double, P_f64]),
    "axg_att_alpha_beta_gamma": (C.c_int, [C.c_int32, P_f64, P_f64, C.c_double, P_f64, P_f64, P_f64]),
    "axg_att_moduli": (C.c_int, [C.c_int32, P_f64, P_f64, C.c_double, C.c_double, C.c_double,
                                 C.c_int32, P_f64, P_f64, P_f64, P_f64, P_f64, P_f64]),
}

_lib = None


def lib():
    """The loaded engine library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("axisem3d_b200: %s is missing; run `python -m axisem3d_b200.build` "
                               "(the engine has no fallback path)" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def ptr(a, ctype):
    """Pointer to a contiguous numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))
