"""ctypes binding of libkrakenb200.so (the C ABI in include/krakenb200.h).

The library is loaded from this directory only.  If it is missing or cannot
be loaded, every entry point raises: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libkrakenb200.so"

KB_OK = 0
KB_ERR_ARG = -1
KB_ERR_UNSUPPORTED = -2
KB_ERR_CUDA = -3
KB_ERR_TIMEOUT = -4
KB_ERR_NONFINITE = -5
KB_ERR_NOMEM = -6

KB_F64, KB_F32, KB_F32_DEV, KB_F16_DEV, KB_BF16_DEV = 0, 1, 2, 3, 4
KB_F16_DEV_SR, KB_BF16_DEV_SR = 5, 6   # same format, stochastic rounding on store

_vp, _cvp, _u8p = C.c_void_p, C.c_void_p, C.c_void_p
_i, _d, _sz = C.c_int, C.c_double, C.c_size_t
_dp = C.POINTER(C.c_double)

# name -> argtypes (restype is int unless listed in _RESTYPES)
SIGNATURES: dict[str, list] = {
    "kb_version": [],
    "kb_last_error": [],
    "kb_sync": [_vp],
    "kb_stream_2d": [_vp, _cvp, _i, _i, _i, _vp],
    "kb_collide_2d": [_vp, _u8p, _i, _i, _d, _i, _vp],
    "kb_apply_zou_he_north_2d": [_vp, _d, _i, _i, _i, _vp],
    "kb_apply_zou_he_south_2d": [_vp, _d, _i, _i, _i, _vp],
    "kb_apply_zou_he_west_2d": [_vp, _d, _i, _i, _i, _vp],
    "kb_apply_zou_he_pressure_east_2d": [_vp, _i, _i, _d, _i, _vp],
    "kb_apply_zou_he_pressure_west_2d": [_vp, _i, _i, _d, _i, _vp],
    "kb_apply_extrapolate_east_2d": [_vp, _i, _i, _i, _vp],
    "kb_apply_bounce_back_wall_2d": [_vp, _i, _i, _i, _i, _vp],
    "kb_compute_macroscopic_2d": [_vp, _vp, _vp, _cvp, _i, _i, _i, _vp],
    "kb_init_equilibrium_2d": [_vp, _cvp, _cvp, _cvp, _i, _i, _i, _i, _vp],
    "kb_fused_bgk_step": [_vp, _cvp, _vp, _vp, _vp, _u8p, _i, _i, _d, _i, _vp],
    "kb_trt_rates": [_d, _d, _dp, _dp],
    "kb_fused_trt_step": [_vp, _cvp, _vp, _vp, _vp, _u8p, _i, _i, _d, _d, _i, _vp],
    "kb_compute_macroscopic_forced_2d": [_vp, _vp, _vp, _cvp, _i, _i, _d, _d, _i, _vp],
    "kb_compute_macroscopic_forced_3d": [_vp, _vp, _vp, _vp, _cvp, _i, _i, _i, _d, _d, _d, _i,
                                         _vp],
    "kb_compute_macroscopic_forced_field_3d": [_vp, _vp, _vp, _vp, _cvp, _cvp, _cvp, _cvp, _i, _i,
                                               _i, _i, _vp],
    "kb_stream_periodic_xz_wall_y_3d": [_vp, _cvp, _i, _i, _i, _i, _vp],
    "kb_slab_fill_ghosts_3d": [_vp, _i, _i, _i, _i, _i, _i, _vp],
    "kb_collide_guo_2d": [_vp, _u8p, _i, _i, _d, _d, _d, _i, _vp],
    "kb_collide_guo_field_2d": [_vp, _u8p, _cvp, _cvp, _i, _i, _d, _i, _vp],
    "kb_collide_guo_3d": [_vp, _u8p, _i, _i, _i, _d, _d, _d, _d, _i, _vp],
    "kb_collide_guo_field_3d": [_vp, _u8p, _cvp, _cvp, _cvp, _i, _i, _i, _d, _i, _vp],
    "kb_fused_trt_libb_step": [_vp, _cvp, _vp, _vp, _vp, _u8p, _cvp, _cvp, _cvp, _i, _i, _d, _d,
                               _i, _vp],
    "kb_fused_trt_libb_step_3d": [_vp, _cvp, _vp, _vp, _vp, _vp, _u8p, _cvp, _cvp, _cvp, _cvp, _i,
                                  _i, _i, _d, _d, _i, _i, _vp],
    "kb_libb_links_create": [_vp, _u8p, _cvp, _cvp, _cvp, _cvp, _i, _i, _i, _i, _vp],
    "kb_libb_links_destroy": [_vp],
    "kb_libb_links_info": [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_int)],
    "kb_fused_trt_libb_links_step_3d": [_vp, _cvp, _vp, _vp, _vp, _vp, _vp, _d, _d, _i, _i, _vp],
    "kb_aa_stream_step_2d": [_vp, _vp, _vp, _vp, _u8p, _i, _i, _d, _i, _vp],
    "kb_aa_local_step_2d": [_vp, _vp, _vp, _vp, _u8p, _i, _i, _d, _i, _vp],
    "kb_collide_mrt_2d": [_vp, _u8p, _i, _i, _d, _d, _d, _d, _i, _vp],
    "kb_stream_fully_periodic_2d": [_vp, _cvp, _i, _i, _i, _vp],
    "kb_stream_periodic_x_wall_y_2d": [_vp, _cvp, _i, _i, _i, _vp],
    "kb_cavity_step_2d": [_vp, _cvp, _vp, _vp, _vp, _u8p, _i, _i, _d, _d, _i, _vp],
    "kb_cavity_mrt_init_step_2d": [_vp, _cvp, _cvp, _cvp, _i, _u8p, _i, _i, _d, _d, _d, _d, _d,
                                   _i, _vp],
    "kb_cavity_movingwall_step_2d": [_vp, _cvp, _vp, _vp, _vp, _u8p, _i, _i, _d, _d, _i, _vp],
    "kb_cavity_mrt_step_2d": [_vp, _cvp, _vp, _vp, _vp, _u8p, _i, _i, _d, _d, _d, _d, _d, _i,
                              _vp],
    "kb_fused_natconv_step": [_vp, _cvp, _vp, _cvp, _vp, _i, _i, _d, _d, _d, _d, _d, _d, _i, _vp],
    "kb_fused_natconv_vt_step": [_vp, _cvp, _vp, _cvp, _vp, _i, _i, _d, _d, _d, _d, _d, _d, _d,
                                 _d, _i, _vp],
    "kb_compute_temperature_2d": [_vp, _cvp, _i, _i, _i, _vp],
    "kb_collide_thermal_2d": [_vp, _cvp, _cvp, _i, _i, _d, _i, _vp],
    "kb_collide_thermal_masked_2d": [_vp, _cvp, _cvp, _u8p, _i, _i, _d, _i, _vp],
    "kb_apply_fixed_temp_face_2d": [_vp, _i, _i, _i, _d, _d, _d, _i, _i, _i, _vp],
    "kb_apply_fixed_temp_2d": [_vp, _i, _i, C.c_uint, _dp, _i, _vp],
    "kb_collide_boussinesq_2d": [_vp, _cvp, _u8p, _i, _i, _d, _d, _d, _i, _vp],
    "kb_collide_boussinesq_vt_2d": [_vp, _cvp, _u8p, _i, _i, _d, _d, _d, _d, _i, _vp],
    "kb_collide_boussinesq_vt_modified_2d": [_vp, _cvp, _u8p, _i, _i, _d, _d, _d, _d, _d, _i,
                                             _vp],
    "kb_collide_thermal_3d": [_vp, _cvp, _cvp, _cvp, _i, _i, _i, _d, _i, _vp],
    "kb_compute_temperature_3d": [_vp, _cvp, _i, _i, _i, _i, _vp],
    "kb_apply_fixed_temp_face_3d": [_vp, _i, _i, _i, _i, _d, _dp, C.c_uint, _i, _vp],
    "kb_apply_fixed_temp_3d": [_vp, _i, _i, _i, C.c_uint, _dp, _i, _vp],
    "kb_collide_boussinesq_3d": [_vp, _cvp, _u8p, _i, _i, _i, _d, _d, _d, _i, _vp],
    "kb_stream_3d": [_vp, _cvp, _i, _i, _i, _i, _vp],
    "kb_collide_3d": [_vp, _u8p, _i, _i, _i, _d, _i, _vp],
    "kb_apply_zou_he_velocity_3d": [_vp, _i, _i, _i, _i, _d, _d, _d, _i, _vp],
    "kb_apply_zou_he_top_3d": [_vp, _d, _i, _i, _i, _i, _vp],
    "kb_apply_zou_he_pressure_3d": [_vp, _i, _i, _i, _i, _d, _i, _vp],
    "kb_compute_macroscopic_3d": [_vp, _vp, _vp, _vp, _cvp, _i, _i, _i, _i, _vp],
    "kb_fused_trt_step_3d": [_vp, _cvp, _vp, _vp, _vp, _vp, _u8p, _i, _i, _i, _d, _d, _i, _i,
                             _vp],
    "kb_fused_trt_step_3d_zrange": [_vp, _cvp, _vp, _vp, _vp, _vp, _u8p, _i, _i, _i, _i, _i, _d,
                                    _d, _i, _i, _vp],
    "kb_set_kernel_variant": [_i, _i],
    "kb_stream_periodic_xz_movingwall_y_3d": [_vp, _cvp, _d, _d, _d, _i, _i, _i, _i, _vp],
    "kb_batch_create": [C.POINTER(_vp), _i, C.POINTER(_i), _dp, _dp, _i, _vp],
    "kb_batch_destroy": [_vp],
    "kb_batch_reset": [_vp, _vp],
    "kb_batch_run": [_vp, _i, _i, _d, _i, _i, _vp],
    "kb_batch_status": [_vp, C.POINTER(C.c_longlong), C.POINTER(_i), C.POINTER(_i), _vp],
    "kb_batch_case": [_vp, _i, C.POINTER(_i), C.POINTER(_i), _dp, C.POINTER(_i),
                      C.POINTER(C.c_float), C.POINTER(C.c_float), _vp],
    "kb_batch_autotune": [_vp, _i, C.POINTER(_i), C.POINTER(_i), _dp, _dp, _vp],
    "kb_batch_populations": [_vp, _i, C.POINTER(_vp), C.POINTER(_i), _vp],
    "kb_graph_begin": [_vp],
    "kb_graph_end": [_vp, C.POINTER(_vp)],
    "kb_graph_launch": [_vp, _vp],
    "kb_graph_destroy": [_vp],
    "kb_selftest_bounded_wait": [C.c_longlong, C.POINTER(_i), _vp],
    "kb_convert_populations": [_vp, _i, _cvp, _i, _i, _sz, _vp],
    "kb_set_stochastic_seed": [C.c_uint, _vp],
    "kb_get_stochastic_seed": [C.POINTER(C.c_uint), _vp],
    "kb_staged_step_status": [_vp, _vp],
    "kb_mass": [_cvp, _i, _sz, _i, _dp, _vp],
    "kb_mass_static": [_cvp, _i, _sz, _i, _dp, _vp],
    "kb_residual": [_cvp, _cvp, _cvp, _cvp, _cvp, _cvp, _u8p, _sz, _i, _dp, _vp],
    "kb_gemm_bf16": [_cvp, _cvp, _vp, _i, _i, _i, _i, _i, _vp, _vp],
    "kb_surrogate_create": [C.POINTER(_vp), _i, _i, _i, _i, C.c_ulonglong, _vp],
    "kb_surrogate_destroy": [_vp],
    "kb_surrogate_num_params": [_vp, C.POINTER(C.c_longlong)],
    "kb_surrogate_layer": [_vp, _i, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i),
                           C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)],
    "kb_surrogate_set_normalisation": [_vp, C.POINTER(C.c_float), C.POINTER(C.c_float)],
    "kb_surrogate_set_grad_weight": [_vp, C.c_float],
    "kb_surrogate_params": [_vp, _vp, _cvp, _vp],
    "kb_surrogate_grads": [_vp, _vp, _vp],
    "kb_surrogate_cavity_inputs": [_vp, _vp, _cvp, _i, _i, _vp],
    "kb_surrogate_infer": [_vp, _cvp, _i, _vp, _vp],
    "kb_surrogate_loss_backward": [_vp, _cvp, _cvp, _i, _vp, _vp],
    "kb_surrogate_adam": [_vp, C.c_float, C.c_float, C.c_float, C.c_float, _i, _vp],
    "kb_surrogate_train_step": [_vp, _cvp, _cvp, _i, C.c_float, _i, _vp, _vp],
    "kb_surrogate_status": [_vp, C.POINTER(_i), _vp],
    "kb_surrogate_flops": [_vp, _i, _dp, _dp],
}
_RESTYPES = {"kb_version": C.c_char_p, "kb_last_error": C.c_char_p}


class KrakenError(RuntimeError):
    """A library call failed (CUDA error, timeout, non-finite reduction...)."""

    def __init__(self, name: str, code: int, msg: str):
        super().__init__(f"{name} failed ({code}): {msg}")
        self.code = code


class KrakenArgumentError(KrakenError, ValueError):
    """Bad argument or unsupported combination (the reference's ArgumentError)."""


_LIB = None
_LOAD_ERROR: str | None = None


def load() -> C.CDLL:
    """Load the shared library once; raise if it is not there."""
    global _LIB, _LOAD_ERROR
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        _LOAD_ERROR = (f"{LIB_PATH} is missing: build it with `python krakenn.jl_b200/build.py` "
                       "(the B200 path has no CPU fallback)")
        raise RuntimeError(_LOAD_ERROR)
    lib = C.CDLL(str(LIB_PATH))
    for name, argt in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argt
        fn.restype = _RESTYPES.get(name, C.c_int)
    _LIB = lib
    return lib


def exported_symbols() -> list[str]:
    return list(SIGNATURES)


def call(name: str, *args) -> int:
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != KB_OK:
        msg = lib.kb_last_error().decode(errors="replace")
        if rc in (KB_ERR_ARG, KB_ERR_UNSUPPORTED):
            raise KrakenArgumentError(name, rc, msg)
        raise KrakenError(name, rc, msg)
    return rc


def version() -> str:
    return load().kb_version().decode()
