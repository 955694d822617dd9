"""numpy front end of the parity oracle (libkboracle.so, built from kb_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product never calls it.

Arrays use the memory order of the reference's column-major arrays:
D2Q9 populations (9, Ny, Nx), D3Q19 (19, Nz, Ny, Nx), fields (Ny, Nx) or
(Nz, Ny, Nx), all float64 C-contiguous; masks uint8/bool.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libkboracle.so"

_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_U8 = C.c_void_p
_i, _d = C.c_int, C.c_double

_SIG = {
    "or_equilibrium_d2q9": ([_d, _d, _d, _i], _d),
    "or_equilibrium_d3q19": ([_d, _d, _d, _d, _i], _d),
    "or_stream_2d": ([_D, _D, _i, _i], None),
    "or_collide_2d": ([_D, _U8, _i, _i, _d], None),
    "or_zou_he_north_2d": ([_D, _d, _i, _i], None),
    "or_zou_he_south_2d": ([_D, _d, _i, _i], None),
    "or_zou_he_west_2d": ([_D, _d, _i, _i], None),
    "or_zou_he_pressure_east_2d": ([_D, _i, _i, _d], None),
    "or_zou_he_pressure_west_2d": ([_D, _i, _i, _d], None),
    "or_extrapolate_east_2d": ([_D, _i, _i], None),
    "or_bounce_back_wall_2d": ([_D, _i, _i, _i], None),
    "or_macroscopic_2d": ([_D, _D, _D, _D, _i, _i], None),
    "or_fused_bgk_2d": ([_D, _D, _D, _D, _D, _U8, _i, _i, _d], None),
    "or_trt_rates": ([_d, _d, _D, _D], None),
    "or_cavity_movingwall_bgk_2d": ([_D, _D, _D, _D, _D, _U8, _i, _i, _d, _d], None),
    "or_fused_trt_2d": ([_D, _D, _D, _D, _D, _U8, _i, _i, _d, _d], None),
    "or_collide_mrt_2d": ([_D, _U8, _i, _i, _d, _d, _d, _d], None),
    "or_stream_fully_periodic_2d": ([_D, _D, _i, _i], None),
    "or_stream_periodic_x_wall_y_2d": ([_D, _D, _i, _i], None),
    "or_run_cavity_2d": ([_D, _D, _D, _D, _D, _U8, _i, _i, _d, _d, _i], None),
    "or_stream_3d": ([_D, _D, _i, _i, _i], None),
    "or_collide_3d": ([_D, _U8, _i, _i, _i, _d], None),
    "or_macroscopic_3d": ([_D, _D, _D, _D, _D, _i, _i, _i], None),
    "or_zou_he_velocity_3d": ([_D, _i, _i, _i, _i, _i, _d, _d, _d], None),
    "or_zou_he_pressure_3d": ([_D, _i, _i, _i, _i, _i, _d], None),
    "or_zou_he_top_3d": ([_D, _d, _i, _i, _i], None),
    "or_run_cavity_3d": ([_D, _D, _D, _D, _D, _D, _U8, _i, _i, _i, _d, _d, _i], None),
    "or_fused_trt_3d": ([_D, _D, _D, _D, _D, _D, _U8, _i, _i, _i, _d, _d, _i, _i, _i], None),
    "or_fused_trt_3d_f32": ([_F, _F, _F, _F, _F, _F, _U8, _i, _i, _i, C.c_float, C.c_float, _i,
                             _i, _i], None),
    "or_stream_periodic_xz_movingwall_y_3d": ([_D, _D, _d, _d, _d, _i, _i, _i], None),
    "or_fused_natconv_2d": ([_D, _D, _D, _D, _D, _i, _i, _d, _d, _d, _d, _d, _d], None),
    "or_fused_natconv_vt_2d": ([_D, _D, _D, _D, _D, _i, _i, _d, _d, _d, _d, _d, _d, _d, _d], None),
    "or_temperature_2d": ([_D, _D, _i, _i], None),
    "or_collide_thermal_2d": ([_D, _D, _D, _i, _i, _d], None),
    "or_collide_thermal_masked_2d": ([_D, _D, _D, _U8, _i, _i, _d], None),
    "or_fixed_temp_face_2d": ([_D, _i, _i, _i, _d, _d, _d, _i, _i], None),
    "or_fixed_temp_2d": ([_D, _i, _i, C.c_uint, _D], None),
    "or_collide_boussinesq_2d": ([_D, _D, _U8, _i, _i, _i, _d, _d, _d, _d, _d, _d], None),
    "or_collide_thermal_3d": ([_D, _D, _D, _D, _i, _i, _i, _d], None),
    "or_temperature_3d": ([_D, _D, _i, _i, _i], None),
    "or_fixed_temp_face_3d": ([_D, _i, _i, _i, _i, _d, _D, C.c_uint], None),
    "or_fixed_temp_3d": ([_D, _i, _i, _i, C.c_uint, _D], None),
    "or_collide_boussinesq_3d": ([_D, _D, _U8, _i, _i, _i, _d, _d, _d], None),
    "or_macroscopic_forced_2d": ([_D, _D, _D, _D, _i, _i, _d, _d], None),
    "or_macroscopic_forced_3d": ([_D, _D, _D, _D, _D, _i, _i, _i, _d, _d, _d, _D, _D, _D], None),
    "or_stream_periodic_3d": ([_D, _D, _i, _i, _i, _i, _i, _i], None),
    "or_collide_guo_2d": ([_D, _U8, _D, _D, _i, _i, _d, _d, _d], None),
    "or_collide_guo_3d": ([_D, _U8, _i, _i, _i, _d, _d, _d, _d], None),
    "or_collide_guo_field_3d": ([_D, _U8, _D, _D, _D, _i, _i, _i, _d], None),
    "or_fused_trt_libb_2d": ([_D, _D, _D, _D, _D, _U8, _D, _D, _D, _i, _i, _d, _d], None),
    "or_fused_trt_libb_3d": ([_D, _D, _D, _D, _D, _D, _U8, _D, _D, _D, _D, _i, _i, _i, _d, _d,
                              _i, _i, _i], None),
    "or_residual": ([_D, _D, _D, _D, _D, _D, _U8, C.c_size_t, _i], _d),
    "or_max_threads": ([], _i),
    "or_set_threads": ([_i], None),
}

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            from . import build as _build  # type: ignore
            _build.build()
        _lib = C.CDLL(str(LIB_PATH))
        for name, (argt, res) in _SIG.items():
            fn = getattr(_lib, name)
            fn.argtypes = argt
            fn.restype = res
    return _lib


def _p(a):
    if a is None:
        return None
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError("oracle arrays must be C-contiguous float64")
    return a.ctypes.data_as(_D)


def _m(mask):
    if mask is None:
        return None
    if mask.dtype not in (np.uint8, np.bool_) or not mask.flags.c_contiguous:
        raise ValueError("oracle masks must be C-contiguous uint8/bool")
    return C.c_void_p(mask.ctypes.data)


def set_threads(n: int):
    lib().or_set_threads(int(n))


def max_threads() -> int:
    return lib().or_max_threads()


# ---- D2Q9 ------------------------------------------------------------------
def _nxny(f):
    return int(f.shape[2]), int(f.shape[1])


def stream_2d(f_out, f_in):
    lib().or_stream_2d(_p(f_out), _p(f_in), *_nxny(f_in))


def collide_2d(f, solid, omega):
    lib().or_collide_2d(_p(f), _m(solid), *_nxny(f), omega)


def zou_he_north_2d(f, u):
    lib().or_zou_he_north_2d(_p(f), u, *_nxny(f))


def zou_he_south_2d(f, u):
    lib().or_zou_he_south_2d(_p(f), u, *_nxny(f))


def zou_he_west_2d(f, u):
    lib().or_zou_he_west_2d(_p(f), u, *_nxny(f))


def zou_he_pressure_east_2d(f, rho_out=1.0):
    lib().or_zou_he_pressure_east_2d(_p(f), *_nxny(f), rho_out)


def zou_he_pressure_west_2d(f, rho_in=1.0):
    lib().or_zou_he_pressure_west_2d(_p(f), *_nxny(f), rho_in)


def extrapolate_east_2d(f):
    lib().or_extrapolate_east_2d(_p(f), *_nxny(f))


def bounce_back_wall_2d(f, wall_id):
    lib().or_bounce_back_wall_2d(_p(f), *_nxny(f), wall_id)


def macroscopic_2d(f):
    Nx, Ny = _nxny(f)
    rho, ux, uy = (np.empty((Ny, Nx)) for _ in range(3))
    lib().or_macroscopic_2d(_p(rho), _p(ux), _p(uy), _p(f), Nx, Ny)
    return rho, ux, uy


def fused_bgk_2d(f_out, f_in, rho, ux, uy, solid, omega):
    lib().or_fused_bgk_2d(_p(f_out), _p(f_in), _p(rho), _p(ux), _p(uy), _m(solid), *_nxny(f_in), omega)


def cavity_movingwall_bgk_2d(f_out, f_in, rho, ux, uy, solid, omega, u_lid):
    lib().or_cavity_movingwall_bgk_2d(_p(f_out), _p(f_in), _p(rho), _p(ux), _p(uy), _m(solid),
                                      *_nxny(f_in), omega, u_lid)


def trt_rates(nu, lam=3 / 16):
    a, b = C.c_double(), C.c_double()
    lib().or_trt_rates(nu, lam, C.byref(a), C.byref(b))
    return a.value, b.value


def fused_trt_2d(f_out, f_in, rho, ux, uy, solid, sp, sm):
    lib().or_fused_trt_2d(_p(f_out), _p(f_in), _p(rho), _p(ux), _p(uy), _m(solid), *_nxny(f_in), sp, sm)


def collide_mrt_2d(f, solid, nu, s_e=1.4, s_eps=1.4, s_q=1.2):
    s_nu = 1.0 / (3.0 * nu + 0.5)
    lib().or_collide_mrt_2d(_p(f), _m(solid), *_nxny(f), s_e, s_eps, s_q, s_nu)


def stream_fully_periodic_2d(f_out, f_in):
    lib().or_stream_fully_periodic_2d(_p(f_out), _p(f_in), *_nxny(f_in))


def stream_periodic_x_wall_y_2d(f_out, f_in):
    lib().or_stream_periodic_x_wall_y_2d(_p(f_out), _p(f_in), *_nxny(f_in))


def run_cavity_2d(f, Nx, Ny, omega, u_lid, steps, solid=None):
    """Path-B cavity loop; f (9, Ny, Nx) is updated in place.  Returns rho, ux, uy."""
    fb = np.empty_like(f)
    rho, ux, uy = (np.empty((Ny, Nx)) for _ in range(3))
    lib().or_run_cavity_2d(_p(f), _p(fb), _p(rho), _p(ux), _p(uy), _m(solid), Nx, Ny, omega, u_lid, steps)
    return rho, ux, uy


def fused_natconv_2d(f_out, f_in, g_out, g_in, Temp, w_f, w_T, beta_g, T_ref, T_hot, T_cold):
    lib().or_fused_natconv_2d(_p(f_out), _p(f_in), _p(g_out), _p(g_in), _p(Temp), *_nxny(f_in),
                              w_f, w_T, beta_g, T_ref, T_hot, T_cold)


def fused_natconv_vt_2d(f_out, f_in, g_out, g_in, Temp, nu_ref, T0, a_visc, w_T, beta_g, T_ref,
                        T_hot, T_cold):
    lib().or_fused_natconv_vt_2d(_p(f_out), _p(f_in), _p(g_out), _p(g_in), _p(Temp), *_nxny(f_in),
                                 nu_ref, T0, a_visc, w_T, beta_g, T_ref, T_hot, T_cold)


def temperature_2d(g):
    Nx, Ny = _nxny(g)
    T = np.empty((Ny, Nx))
    lib().or_temperature_2d(_p(T), _p(g), Nx, Ny)
    return T


FACES_2D = {"west": 0, "east": 1, "south": 2, "north": 3}
FACES_3D = {"west": 0, "east": 1, "south": 2, "north": 3, "bottom": 4, "top": 5}


def collide_thermal_2d(g, ux, uy, w_T):
    lib().or_collide_thermal_2d(_p(g), _p(ux), _p(uy), *_nxny(g), float(w_T))


def collide_thermal_masked_2d(g, ux, uy, w_T, is_skip):
    lib().or_collide_thermal_masked_2d(_p(g), _p(ux), _p(uy), _m(is_skip), *_nxny(g), float(w_T))


def fixed_temp_face_2d(g, face, T_wall, T_corner=None, skip=(False, False)):
    """_fixed_temp_<face>_2d!; T_corner defaults to (T_wall, T_wall)."""
    tc = (T_wall, T_wall) if T_corner is None else T_corner
    lib().or_fixed_temp_face_2d(_p(g), *_nxny(g), FACES_2D[face], float(T_wall), float(tc[0]),
                                float(tc[1]), int(bool(skip[0])), int(bool(skip[1])))


def _face_set(temps, names):
    mask, T = 0, np.zeros(len(names))
    for n, name in enumerate(names):
        if temps.get(name) is not None:
            mask |= 1 << n
            T[n] = float(temps[name])
    return mask, T


def fixed_temp_2d(g, **temps):
    """apply_fixed_temp_2d!(g, Nx, Ny; west, east, south, north)"""
    mask, T = _face_set(temps, list(FACES_2D))
    lib().or_fixed_temp_2d(_p(g), *_nxny(g), mask, _p(T))


def collide_boussinesq_2d(f, Temp, solid, omega, beta_g, T_ref):
    lib().or_collide_boussinesq_2d(_p(f), _p(Temp), _m(solid), *_nxny(f), 0, float(omega), 0.0,
                                   0.0, 0.0, float(beta_g), float(T_ref))


def collide_boussinesq_vt_2d(f, Temp, solid, nu_ref, T_ref, A_arr, beta_g):
    lib().or_collide_boussinesq_2d(_p(f), _p(Temp), _m(solid), *_nxny(f), 1, 0.0, float(nu_ref),
                                   float(T_ref), float(A_arr), float(beta_g), float(T_ref))


def collide_boussinesq_vt_modified_2d(f, Temp, solid, nu_ref, T0_visc, alpha_visc, beta_g,
                                      T_ref_buoy):
    lib().or_collide_boussinesq_2d(_p(f), _p(Temp), _m(solid), *_nxny(f), 2, 0.0, float(nu_ref),
                                   float(T0_visc), float(alpha_visc), float(beta_g),
                                   float(T_ref_buoy))


# ---- D3Q19 -----------------------------------------------------------------
def _n3(f):
    return int(f.shape[3]), int(f.shape[2]), int(f.shape[1])


def stream_3d(f_out, f_in):
    lib().or_stream_3d(_p(f_out), _p(f_in), *_n3(f_in))


def collide_3d(f, solid, omega):
    lib().or_collide_3d(_p(f), _m(solid), *_n3(f), omega)


def macroscopic_3d(f):
    Nx, Ny, Nz = _n3(f)
    out = [np.empty((Nz, Ny, Nx)) for _ in range(4)]
    lib().or_macroscopic_3d(*map(_p, out), _p(f), Nx, Ny, Nz)
    return tuple(out)


FACES = {"west": 0, "east": 1, "south": 2, "north": 3, "bottom": 4, "top": 5}


def _fixed(face, Nx, Ny, Nz):
    n = {0: Nx, 1: Nx, 2: Ny, 3: Ny, 4: Nz, 5: Nz}[face]
    return n - 1 if face % 2 == 1 else 0


def zou_he_velocity_3d(f, face, u_n, u_t1, u_t2):
    Nx, Ny, Nz = _n3(f)
    fc = FACES[face] if isinstance(face, str) else face
    lib().or_zou_he_velocity_3d(_p(f), Nx, Ny, Nz, fc, _fixed(fc, Nx, Ny, Nz), u_n, u_t1, u_t2)


def zou_he_pressure_3d(f, face, rho_out=1.0):
    Nx, Ny, Nz = _n3(f)
    fc = FACES[face] if isinstance(face, str) else face
    lib().or_zou_he_pressure_3d(_p(f), Nx, Ny, Nz, fc, _fixed(fc, Nx, Ny, Nz), rho_out)


def zou_he_top_3d(f, u):
    lib().or_zou_he_top_3d(_p(f), u, *_n3(f))


def run_cavity_3d(f, omega, u_lid, steps, solid=None):
    Nx, Ny, Nz = _n3(f)
    fb = np.empty_like(f)
    out = [np.empty((Nz, Ny, Nx)) for _ in range(4)]
    lib().or_run_cavity_3d(_p(f), _p(fb), *map(_p, out), _m(solid), Nx, Ny, Nz, omega, u_lid, steps)
    return tuple(out)


def fused_trt_3d(f_out, f_in, moments, solid, sp, sm, periodic=(0, 0, 0)):
    """moments: tuple of four (Nz, Ny, Nx) arrays, or None."""
    Nx, Ny, Nz = _n3(f_in)
    m = moments if moments is not None else (None,) * 4
    lib().or_fused_trt_3d(_p(f_out), _p(f_in), *map(_p, m), _m(solid), Nx, Ny, Nz, sp, sm,
                          int(bool(periodic[0])), int(bool(periodic[1])), int(bool(periodic[2])))


def _pf(a):
    if a is None:
        return None
    if a.dtype != np.float32 or not a.flags.c_contiguous:
        raise ValueError("single-precision oracle arrays must be C-contiguous float32")
    return a.ctypes.data_as(_F)


def fused_trt_3d_f32(f_out, f_in, moments, solid, sp, sm, periodic=(0, 0, 0)):
    """fused_trt_3d in single precision (the reference's T = Float32 path):
    float32 arrays, rates rounded to float32.  The timed CPU baseline of the
    FP32 storages."""
    Nx, Ny, Nz = _n3(f_in)
    m = moments if moments is not None else (None,) * 4
    lib().or_fused_trt_3d_f32(_pf(f_out), _pf(f_in), *map(_pf, m), _m(solid), Nx, Ny, Nz,
                              float(np.float32(sp)), float(np.float32(sm)),
                              int(bool(periodic[0])), int(bool(periodic[1])),
                              int(bool(periodic[2])))


def stream_periodic_xz_movingwall_y_3d(f_out, f_in, Ub, Ut, rho_w=1.0):
    lib().or_stream_periodic_xz_movingwall_y_3d(_p(f_out), _p(f_in), Ub, Ut, rho_w, *_n3(f_in))


def residual(ux, uy, uxp, uyp, uz=None, uzp=None, solid=None):
    n = ux.size
    return lib().or_residual(_p(ux), _p(uy), _p(uz), _p(uxp), _p(uyp), _p(uzp), _m(solid), n,
                             3 if uz is not None else 2)


def equilibrium_d2q9(rho, ux, uy, q):
    return lib().or_equilibrium_d2q9(rho, ux, uy, q)


def equilibrium_d3q19(rho, ux, uy, uz, q):
    return lib().or_equilibrium_d3q19(rho, ux, uy, uz, q)


def collide_thermal_3d(g, ux, uy, uz, w_T):
    lib().or_collide_thermal_3d(_p(g), _p(ux), _p(uy), _p(uz), *_n3(g), float(w_T))


def temperature_3d(g):
    Nx, Ny, Nz = _n3(g)
    T = np.empty((Nz, Ny, Nx))
    lib().or_temperature_3d(_p(T), _p(g), Nx, Ny, Nz)
    return T


def fixed_temp_face_3d(g, face, T_wall, T_edge=None, skip=0):
    """_fixed_temp_<face>_3d!; T_edge defaults to T_wall on all four edges."""
    te = np.full(4, float(T_wall)) if T_edge is None else np.asarray(T_edge, dtype=np.float64)
    lib().or_fixed_temp_face_3d(_p(g), *_n3(g), FACES_3D[face], float(T_wall), _p(te), int(skip))


def fixed_temp_3d(g, **temps):
    """apply_fixed_temp_3d!(g, Nx, Ny, Nz; west, east, south, north, bottom, top)"""
    mask, T = _face_set(temps, list(FACES_3D))
    lib().or_fixed_temp_3d(_p(g), *_n3(g), mask, _p(T))


def collide_boussinesq_3d(f, Temp, solid, omega, beta_g, T_ref):
    lib().or_collide_boussinesq_3d(_p(f), _p(Temp), _m(solid), *_n3(f), float(omega),
                                   float(beta_g), float(T_ref))


def fused_trt_libb_2d(f_out, f_in, rho, ux, uy, solid, q_wall, uw_x, uw_y, sp, sm):
    """fused_trt_libb_v2_step! with the rates already rounded to the storage type"""
    lib().or_fused_trt_libb_2d(_p(f_out), _p(f_in), _p(rho), _p(ux), _p(uy), _m(solid),
                               _p(q_wall), _p(uw_x), _p(uw_y), *_nxny(f_in), float(sp), float(sm))


def fused_trt_libb_3d(f_out, f_in, moments, solid, q_wall, uw_x, uw_y, uw_z, sp, sm,
                      periodic=(0, 0, 0)):
    """fused_trt_libb_v2_step_3d!; moments = (rho, ux, uy, uz) arrays or None"""
    m = moments if moments is not None else (None,) * 4
    lib().or_fused_trt_libb_3d(_p(f_out), _p(f_in), *map(_p, m), _m(solid), _p(q_wall),
                               _p(uw_x), _p(uw_y), _p(uw_z), *_n3(f_in), float(sp), float(sm),
                               *[int(bool(x)) for x in periodic])


def collide_guo_2d(f, solid, omega, Fx, Fy):
    """collide_guo_2d!(f, is_solid, omega, Fx, Fy)"""
    lib().or_collide_guo_2d(_p(f), _m(solid), None, None, *_nxny(f), float(omega), float(Fx),
                            float(Fy))


def collide_guo_field_2d(f, solid, Fx_field, Fy_field, omega):
    lib().or_collide_guo_2d(_p(f), _m(solid), _p(Fx_field), _p(Fy_field), *_nxny(f),
                            float(omega), 0.0, 0.0)


def collide_guo_3d(f, solid, omega, Fx, Fy, Fz):
    lib().or_collide_guo_3d(_p(f), _m(solid), *_n3(f), float(omega), float(Fx), float(Fy),
                            float(Fz))


def collide_guo_field_3d(f, solid, Fx_field, Fy_field, Fz_field, omega):
    lib().or_collide_guo_field_3d(_p(f), _m(solid), _p(Fx_field), _p(Fy_field), _p(Fz_field),
                                  *_n3(f), float(omega))


def macroscopic_forced_2d(f, Fx, Fy):
    Nx, Ny = _nxny(f)
    rho, ux, uy = (np.empty((Ny, Nx)) for _ in range(3))
    lib().or_macroscopic_forced_2d(_p(rho), _p(ux), _p(uy), _p(f), Nx, Ny, float(Fx), float(Fy))
    return rho, ux, uy


def macroscopic_forced_3d(f, Fx, Fy, Fz):
    """Fx, Fy, Fz scalars or per-node arrays (compute_macroscopic_forced_field_3d!)"""
    Nx, Ny, Nz = _n3(f)
    out = [np.empty((Nz, Ny, Nx)) for _ in range(4)]
    if isinstance(Fx, np.ndarray):
        lib().or_macroscopic_forced_3d(*map(_p, out), _p(f), Nx, Ny, Nz, 0.0, 0.0, 0.0, _p(Fx),
                                       _p(Fy), _p(Fz))
    else:
        lib().or_macroscopic_forced_3d(*map(_p, out), _p(f), Nx, Ny, Nz, float(Fx), float(Fy),
                                       float(Fz), None, None, None)
    return tuple(out)


def stream_periodic_xz_wall_y_3d(f_out, f_in):
    lib().or_stream_periodic_3d(_p(f_out), _p(f_in), *_n3(f_in), 1, 0, 1)
