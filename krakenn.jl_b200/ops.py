"""Kernel-level API: the reference's stream-collide functions on B200 tensors.

Every function here calls one C-ABI entry point of libkrakenb200.so on the
current torch CUDA stream.  Names follow Kraken.jl with the trailing `!`
written as `_` (in-place), and the positional arguments keep the reference's
order and meaning.  Arrays are torch CUDA tensors laid out like the
reference's column-major arrays: a Julia `f[i, j, q]` of size (Nx, Ny, 9) is
a contiguous torch tensor of shape (9, Ny, Nx); D3Q19 `f[i, j, k, q]` is
(19, Nz, Ny, Nx); fields `rho[i, j]` are (Ny, Nx).

Storage: float64 and float32 tensors hold f with the reference arithmetic.
float16 / bfloat16 tensors hold the deviation f - w_q (FP32 collision); a
float32 deviation buffer is selected with `deviation=True`.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib


def _arg_error(msg: str) -> _lib.KrakenArgumentError:
    """A refused argument, raised before any call into the library: the same
    exception (a ValueError) and status code (KB_ERR_ARG) as an argument the
    library itself refuses."""
    return _lib.KrakenArgumentError("argument check", _lib.KB_ERR_ARG, msg)
from ._lib import (KB_BF16_DEV, KB_BF16_DEV_SR, KB_F16_DEV, KB_F16_DEV_SR, KB_F32, KB_F32_DEV,
                   KB_F64, call)

_TORCH_DTYPE = {KB_F64: torch.float64, KB_F32: torch.float32, KB_F32_DEV: torch.float32,
                KB_F16_DEV: torch.float16, KB_BF16_DEV: torch.bfloat16}


def storage_dtype(t: torch.Tensor, deviation: bool = False) -> int:
    """kb_dtype code of a population tensor."""
    if t.dtype == torch.float64:
        if deviation:
            raise _arg_error("float64 storage holds f, not a deviation")
        return KB_F64
    if t.dtype == torch.float32:
        return KB_F32_DEV if deviation else KB_F32
    if t.dtype == torch.float16:
        return KB_F16_DEV
    if t.dtype == torch.bfloat16:
        return KB_BF16_DEV
    raise _arg_error(f"unsupported population dtype {t.dtype}")


def torch_dtype(code: int) -> torch.dtype:
    return _TORCH_DTYPE[code]


def field_dtype(code: int) -> torch.dtype:
    """dtype of the macroscopic fields that go with a population storage."""
    return torch.float64 if code == KB_F64 else torch.float32


def _t(t: torch.Tensor | None, name: str):
    if t is None:
        return None
    if not isinstance(t, torch.Tensor):
        raise _arg_error(f"{name} must be a torch tensor")
    if not t.is_cuda:
        raise _arg_error(f"{name} must live on a CUDA device (the B200 path has no CPU fallback)")
    if not t.is_contiguous():
        raise _arg_error(f"{name} must be contiguous")
    return C.c_void_p(t.data_ptr())


def _mask(m: torch.Tensor | None):
    if m is None:
        return None
    if m.dtype not in (torch.bool, torch.uint8):
        raise _arg_error("is_solid must be a bool or uint8 tensor")
    return _t(m, "is_solid")


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _plain(f: torch.Tensor) -> int:
    code = storage_dtype(f)
    if code not in (KB_F64, KB_F32):
        raise _arg_error("this reference kernel takes float64 or float32 populations")
    return code


def _same(code: int, *fields):
    want = field_dtype(code)
    for name, t in fields:
        if t is not None and t.dtype != want:
            raise _arg_error(f"{name} must be {want} for this population storage")


def _dims2(f: torch.Tensor):
    if f.dim() != 3 or f.shape[0] != 9:
        raise _arg_error("D2Q9 populations must have shape (9, Ny, Nx)")
    return int(f.shape[2]), int(f.shape[1])


def _dims3(f: torch.Tensor):
    if f.dim() != 4 or f.shape[0] != 19:
        raise _arg_error("D3Q19 populations must have shape (19, Nz, Ny, Nx)")
    return int(f.shape[3]), int(f.shape[2]), int(f.shape[1])


def _match2(f, Nx, Ny):
    if _dims2(f) != (Nx, Ny):
        raise _arg_error(f"population shape {tuple(f.shape)} does not match Nx={Nx}, Ny={Ny}")


def _match3(f, Nx, Ny, Nz):
    if _dims3(f) != (Nx, Ny, Nz):
        raise _arg_error(f"population shape {tuple(f.shape)} does not match "
                         f"Nx={Nx}, Ny={Ny}, Nz={Nz}")


def _ptrs_2d_fields(code, Nx, Ny, **fields):
    for name, t in fields.items():
        if t is not None and tuple(t.shape) != (Ny, Nx):
            raise _arg_error(f"{name} must have shape (Ny, Nx) = ({Ny}, {Nx})")
    _same(code, *fields.items())


def _ptrs_3d_fields(code, Nx, Ny, Nz, **fields):
    for name, t in fields.items():
        if t is not None and tuple(t.shape) != (Nz, Ny, Nx):
            raise _arg_error(f"{name} must have shape (Nz, Ny, Nx) = ({Nz}, {Ny}, {Nx})")
    _same(code, *fields.items())


# --------------------------------------------------------------------- D2Q9

def stream_2d_(f_out, f_in, Nx, Ny):
    """stream_2d! -- src/kernels/collide_stream_2d.jl:77"""
    code = _plain(f_in)
    _match2(f_in, Nx, Ny); _match2(f_out, Nx, Ny)
    call("kb_stream_2d", _t(f_out, "f_out"), _t(f_in, "f_in"), Nx, Ny, code, _stream())


def collide_2d_(f, is_solid, omega):
    """collide_2d! -- src/kernels/collide_stream_2d.jl:96"""
    code = _plain(f)
    Nx, Ny = _dims2(f)
    call("kb_collide_2d", _t(f, "f"), _mask(is_solid), Nx, Ny, float(omega), code, _stream())


def apply_zou_he_north_2d_(f, u_wall_x, Nx, Ny):
    """apply_zou_he_north_2d! -- src/kernels/boundary_2d.jl:56"""
    code = _plain(f); _match2(f, Nx, Ny)
    call("kb_apply_zou_he_north_2d", _t(f, "f"), float(u_wall_x), Nx, Ny, code, _stream())


def apply_zou_he_south_2d_(f, u_wall_x, Nx):
    """apply_zou_he_south_2d! -- src/kernels/boundary_2d.jl:163"""
    code = _plain(f)
    nx, ny = _dims2(f)
    if nx != Nx:
        raise _arg_error("Nx does not match the population shape")
    call("kb_apply_zou_he_south_2d", _t(f, "f"), float(u_wall_x), Nx, ny, code, _stream())


def apply_zou_he_west_2d_(f, u_in, Nx, Ny):
    """apply_zou_he_west_2d! -- src/kernels/boundary_2d.jl:198"""
    code = _plain(f); _match2(f, Nx, Ny)
    call("kb_apply_zou_he_west_2d", _t(f, "f"), float(u_in), Nx, Ny, code, _stream())


def apply_zou_he_pressure_east_2d_(f, Nx, Ny, rho_out=1.0):
    """apply_zou_he_pressure_east_2d! -- src/kernels/boundary_2d.jl:237"""
    code = _plain(f); _match2(f, Nx, Ny)
    call("kb_apply_zou_he_pressure_east_2d", _t(f, "f"), Nx, Ny, float(rho_out), code, _stream())


def apply_zou_he_pressure_west_2d_(f, Nx, Ny, rho_in=1.0):
    """apply_zou_he_pressure_west_2d! -- src/kernels/boundary_2d.jl:295"""
    code = _plain(f); _match2(f, Nx, Ny)
    call("kb_apply_zou_he_pressure_west_2d", _t(f, "f"), Nx, Ny, float(rho_in), code, _stream())


def apply_extrapolate_east_2d_(f, Nx, Ny):
    """apply_extrapolate_east_2d! -- src/kernels/boundary_2d.jl:319"""
    code = _plain(f); _match2(f, Nx, Ny)
    call("kb_apply_extrapolate_east_2d", _t(f, "f"), Nx, Ny, code, _stream())


_SIDES = {"south": 1, "west": 2, "east": 3, "north": 4}


def apply_bounce_back_wall_2d_(f, Nx, Ny, side):
    """apply_bounce_back_wall_2d! -- src/kernels/boundary_2d.jl:117"""
    code = _plain(f); _match2(f, Nx, Ny)
    if side not in _SIDES:
        raise _arg_error(f"apply_bounce_back_wall_2d!: unknown side {side}")
    call("kb_apply_bounce_back_wall_2d", _t(f, "f"), Nx, Ny, _SIDES[side], code, _stream())


def apply_bounce_back_walls_2d_(f, Nx, Ny):
    """apply_bounce_back_walls_2d! (south, west, east) -- src/kernels/boundary_2d.jl:98"""
    for side in ("south", "west", "east"):
        apply_bounce_back_wall_2d_(f, Nx, Ny, side)


def compute_macroscopic_2d_(rho, ux, uy, f):
    """compute_macroscopic_2d! -- src/kernels/macroscopic.jl:32"""
    code = _plain(f)
    Nx, Ny = _dims2(f)
    _ptrs_2d_fields(code, Nx, Ny, rho=rho, ux=ux, uy=uy)
    call("kb_compute_macroscopic_2d", _t(rho, "rho"), _t(ux, "ux"), _t(uy, "uy"), _t(f, "f"),
         Nx, Ny, code, _stream())


def fused_bgk_step_(f_out, f_in, rho, ux, uy, is_solid, Nx, Ny, omega):
    """fused_bgk_step! -- src/kernels/fused_bgk_2d.jl:67"""
    code = _plain(f_in)
    _match2(f_in, Nx, Ny); _match2(f_out, Nx, Ny)
    _ptrs_2d_fields(code, Nx, Ny, rho=rho, ux=ux, uy=uy)
    call("kb_fused_bgk_step", _t(f_out, "f_out"), _t(f_in, "f_in"), _t(rho, "rho"),
         _t(ux, "ux"), _t(uy, "uy"), _mask(is_solid), Nx, Ny, float(omega), code, _stream())


def trt_rates(nu, Lambda=3 / 16):
    """trt_rates(nu; Lambda) -> (s_plus, s_minus) -- src/kernels/fused_trt_2d.jl:129"""
    sp, sm = C.c_double(), C.c_double()
    call("kb_trt_rates", float(nu), float(Lambda), C.byref(sp), C.byref(sm))
    return sp.value, sm.value


def fused_trt_step_(f_out, f_in, rho, ux, uy, is_solid, Nx, Ny, nu, Lambda=3 / 16):
    """fused_trt_step! -- src/kernels/fused_trt_2d.jl:145"""
    code = _plain(f_in)
    _match2(f_in, Nx, Ny); _match2(f_out, Nx, Ny)
    _ptrs_2d_fields(code, Nx, Ny, rho=rho, ux=ux, uy=uy)
    call("kb_fused_trt_step", _t(f_out, "f_out"), _t(f_in, "f_in"), _t(rho, "rho"),
         _t(ux, "ux"), _t(uy, "uy"), _mask(is_solid), Nx, Ny, float(nu), float(Lambda), code,
         _stream())


def compute_macroscopic_forced_2d_(rho, ux, uy, f, Fx, Fy):
    """compute_macroscopic_forced_2d! -- src/kernels/macroscopic.jl:112"""
    code = _plain(f)
    Nx, Ny = _dims2(f)
    _ptrs_2d_fields(code, Nx, Ny, rho=rho, ux=ux, uy=uy)
    call("kb_compute_macroscopic_forced_2d", _t(rho, "rho"), _t(ux, "ux"), _t(uy, "uy"),
         _t(f, "f"), Nx, Ny, float(Fx), float(Fy), code, _stream())


def collide_guo_2d_(f, is_solid, omega, Fx, Fy):
    """collide_guo_2d! -- src/kernels/collide_guo_2d.jl:84"""
    code = _plain(f)
    Nx, Ny = _dims2(f)
    call("kb_collide_guo_2d", _t(f, "f"), _mask(is_solid), Nx, Ny, float(omega), float(Fx),
         float(Fy), code, _stream())


def collide_guo_field_2d_(f, is_solid, Fx_field, Fy_field, omega):
    """collide_guo_field_2d! -- src/kernels/collide_guo_2d.jl:157"""
    code = _plain(f)
    Nx, Ny = _dims2(f)
    for name, t in (("Fx_field", Fx_field), ("Fy_field", Fy_field)):
        if t is None or t.dtype != f.dtype or tuple(t.shape) != (Ny, Nx):
            raise _arg_error(f"{name} must be a {f.dtype} tensor of shape (Ny, Nx)")
    call("kb_collide_guo_field_2d", _t(f, "f"), _mask(is_solid), _t(Fx_field, "Fx_field"),
         _t(Fy_field, "Fy_field"), Nx, Ny, float(omega), code, _stream())


def fused_trt_libb_v2_step_(f_out, f_in, rho, ux, uy, is_solid, q_wall, uw_link_x, uw_link_y,
                            Nx, Ny, nu, Lambda=3 / 16):
    """fused_trt_libb_v2_step! -- src/kernels/li_bb_2d_v2.jl:104 (TRT with
    Bouzidi interpolated bounce-back on the links flagged in q_wall)"""
    code = _plain(f_in)
    _match2(f_in, Nx, Ny); _match2(f_out, Nx, Ny)
    for name, t in (("q_wall", q_wall), ("uw_link_x", uw_link_x), ("uw_link_y", uw_link_y)):
        if t is None or t.dtype != f_in.dtype or tuple(t.shape) != tuple(f_in.shape):
            raise _arg_error(f"{name} must be a {f_in.dtype} tensor shaped like f")
    _ptrs_2d_fields(code, Nx, Ny, rho=rho, ux=ux, uy=uy)
    call("kb_fused_trt_libb_step", _t(f_out, "f_out"), _t(f_in, "f_in"), _t(rho, "rho"),
         _t(ux, "ux"), _t(uy, "uy"), _mask(is_solid), _t(q_wall, "q_wall"),
         _t(uw_link_x, "uw_link_x"), _t(uw_link_y, "uw_link_y"), Nx, Ny, float(nu),
         float(Lambda), code, _stream())


def aa_stream_step_2d_(f, rho, ux, uy, is_solid, Nx, Ny, omega):
    """In-place A-A step, state S -> P (gather from neighbours, collide,
    scatter); the race-free form of aa_even_step!/aa_odd_step!
    (src/kernels/aa_bgk_2d.jl:125,138).  Moments may be None."""
    code = _plain(f); _match2(f, Nx, Ny)
    _ptrs_2d_fields(code, Nx, Ny, rho=rho, ux=ux, uy=uy)
    call("kb_aa_stream_step_2d", _t(f, "f"), _t(rho, "rho"), _t(ux, "ux"), _t(uy, "uy"),
         _mask(is_solid), Nx, Ny, float(omega), code, _stream())


def aa_local_step_2d_(f, rho, ux, uy, is_solid, Nx, Ny, omega):
    """In-place A-A step, state P -> S (read local, collide, write swapped)."""
    code = _plain(f); _match2(f, Nx, Ny)
    _ptrs_2d_fields(code, Nx, Ny, rho=rho, ux=ux, uy=uy)
    call("kb_aa_local_step_2d", _t(f, "f"), _t(rho, "rho"), _t(ux, "ux"), _t(uy, "uy"),
         _mask(is_solid), Nx, Ny, float(omega), code, _stream())


AA_SWAP_2D = (0, 3, 4, 1, 2, 7, 8, 5, 6)


def persistent_aa_bgk_(f, is_solid, Nx, Ny, omega, Nt):
    """persistent_aa_bgk! (src/kernels/persistent_bgk_2d.jl:182): Nt A-A steps
    queued without synchronisation on one pull-format buffer f (slot q holds
    the post-collision f_q), returned in the same format.  Nt must be even."""
    if Nt % 2:
        raise _arg_error("persistent_aa_bgk_: Nt must be even (pairs of A-A steps)")
    idx = torch.tensor(AA_SWAP_2D, device=f.device)
    f.copy_(f.index_select(0, idx))
    for _ in range(Nt // 2):
        aa_stream_step_2d_(f, None, None, None, is_solid, Nx, Ny, omega)
        aa_local_step_2d_(f, None, None, None, is_solid, Nx, Ny, omega)
    f.copy_(f.index_select(0, idx))
    return f


def persistent_fused_bgk_(f_in, f_out, rho, ux, uy, is_solid, Nx, Ny, omega, Nt):
    """persistent_fused_bgk! (src/kernels/persistent_bgk_2d.jl:160): Nt fused
    BGK steps queued with no host synchronisation; returns (a, b) with a the
    buffer holding the latest populations."""
    a, b = f_in, f_out
    for _ in range(Nt):
        fused_bgk_step_(b, a, rho, ux, uy, is_solid, Nx, Ny, omega)
        a, b = b, a
    return a, b


def collide_mrt_2d_(f, is_solid, nu, s_e=1.4, s_eps=1.4, s_q=1.2):
    """collide_mrt_2d! -- src/kernels/collide_mrt_2d.jl:118"""
    code = _plain(f)
    Nx, Ny = _dims2(f)
    call("kb_collide_mrt_2d", _t(f, "f"), _mask(is_solid), Nx, Ny, float(nu), float(s_e),
         float(s_eps), float(s_q), code, _stream())


def stream_fully_periodic_2d_(f_out, f_in, Nx, Ny):
    """stream_fully_periodic_2d! -- src/kernels/stream_periodic_2d.jl:112"""
    code = _plain(f_in); _match2(f_in, Nx, Ny); _match2(f_out, Nx, Ny)
    call("kb_stream_fully_periodic_2d", _t(f_out, "f_out"), _t(f_in, "f_in"), Nx, Ny, code,
         _stream())


def stream_periodic_x_wall_y_2d_(f_out, f_in, Nx, Ny):
    """stream_periodic_x_wall_y_2d! -- src/kernels/stream_periodic_2d.jl:71"""
    code = _plain(f_in); _match2(f_in, Nx, Ny); _match2(f_out, Nx, Ny)
    call("kb_stream_periodic_x_wall_y_2d", _t(f_out, "f_out"), _t(f_in, "f_in"), Nx, Ny, code,
         _stream())


def cavity_step_2d_(f_out, f_in, rho, ux, uy, is_solid, Nx, Ny, omega, u_lid):
    """One run_cavity_2d step (src/drivers/basic.jl:121-136) in one launch."""
    code = _plain(f_in)
    _match2(f_in, Nx, Ny); _match2(f_out, Nx, Ny)
    _ptrs_2d_fields(code, Nx, Ny, rho=rho, ux=ux, uy=uy)
    call("kb_cavity_step_2d", _t(f_out, "f_out"), _t(f_in, "f_in"), _t(rho, "rho"),
         _t(ux, "ux"), _t(uy, "uy"), _mask(is_solid), Nx, Ny, float(omega), float(u_lid), code,
         _stream())


def cavity_movingwall_step_2d_(f_out, f_in, rho, ux, uy, is_solid, Nx, Ny, omega, u_lid):
    """Cavity step with a moving-wall half-way bounce-back lid (fused_bgk_step!
    + the lid link rule of src/kernels/dsl/bricks.jl:447-487); moments may be None."""
    code = _plain(f_in)
    _match2(f_in, Nx, Ny); _match2(f_out, Nx, Ny)
    _ptrs_2d_fields(code, Nx, Ny, rho=rho, ux=ux, uy=uy)
    call("kb_cavity_movingwall_step_2d", _t(f_out, "f_out"), _t(f_in, "f_in"), _t(rho, "rho"),
         _t(ux, "ux"), _t(uy, "uy"), _mask(is_solid), Nx, Ny, float(omega), float(u_lid), code,
         _stream())


def cavity_mrt_step_2d_(f_out, f_in, rho, ux, uy, is_solid, Nx, Ny, nu, u_lid, s_e=1.4,
                        s_eps=1.4, s_q=1.2):
    """One MRT cavity step (test/test_mrt.jl:19-25) in one launch; moments may be None."""
    code = _plain(f_in)
    _match2(f_in, Nx, Ny); _match2(f_out, Nx, Ny)
    _ptrs_2d_fields(code, Nx, Ny, rho=rho, ux=ux, uy=uy)
    call("kb_cavity_mrt_step_2d", _t(f_out, "f_out"), _t(f_in, "f_in"), _t(rho, "rho"),
         _t(ux, "ux"), _t(uy, "uy"), _mask(is_solid), Nx, Ny, float(nu), float(s_e),
         float(s_eps), float(s_q), float(u_lid), code, _stream())


def _natconv_code(f_in, g_in, deviation, stochastic_rounding):
    """kb_dtype of a natural-convection step: the reference's FP64 / FP32, or
    (deviation) f - w_q and g - w_q T_ref in float32 / float16 / bfloat16."""
    if g_in.dtype != f_in.dtype:
        raise _arg_error("f and g populations must have the same dtype")
    if not deviation:
        if stochastic_rounding:
            raise _arg_error("stochastic rounding applies to float16/bfloat16 deviation storage")
        return _plain(f_in)
    code = storage_dtype(f_in, True)
    if stochastic_rounding:
        if code not in (KB_F16_DEV, KB_BF16_DEV):
            raise _arg_error("stochastic rounding applies to float16/bfloat16 deviation storage")
        code = KB_F16_DEV_SR if code == KB_F16_DEV else KB_BF16_DEV_SR
    return code


def thermal_deviation(g, T_ref, to_deviation=True):
    """g - w_q T_ref (to_deviation) or its inverse, for the thermal DDF
    populations of a D2Q9 natural-convection step on deviation storage; g of
    shape (9, Ny, Nx).  Returns a float64 tensor on g's device."""
    w = torch.tensor([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4, dtype=torch.float64, device=g.device)
    shift = (w * float(T_ref))[:, None, None]
    return g.double() - shift if to_deviation else g.double() + shift


def fused_natconv_step_(f_out, f_in, g_out, g_in, Temp, Nx, Ny, omega_f, omega_T, beta_g,
                        T_ref_buoy, T_hot, T_cold, deviation=False, stochastic_rounding=False):
    """fused_natconv_step! -- src/kernels/fused_thermal_2d.jl:251.  With
    deviation, f holds f - w_q and g holds g - w_q T_ref_buoy (float32,
    float16 or bfloat16) and the step runs in FP32; Temp is float32."""
    code = _natconv_code(f_in, g_in, deviation, stochastic_rounding)
    for t in (f_in, f_out, g_in, g_out):
        _match2(t, Nx, Ny)
    _ptrs_2d_fields(code, Nx, Ny, Temp=Temp)
    call("kb_fused_natconv_step", _t(f_out, "f_out"), _t(f_in, "f_in"), _t(g_out, "g_out"),
         _t(g_in, "g_in"), _t(Temp, "Temp"), Nx, Ny, float(omega_f), float(omega_T),
         float(beta_g), float(T_ref_buoy), float(T_hot), float(T_cold), code, _stream())


def fused_natconv_vt_step_(f_out, f_in, g_out, g_in, Temp, Nx, Ny, nu_ref, T0_visc, alpha_visc,
                           omega_T, beta_g, T_ref_buoy, T_hot, T_cold, deviation=False,
                           stochastic_rounding=False):
    """fused_natconv_vt_step! -- src/kernels/fused_thermal_2d.jl:268 (storages
    as fused_natconv_step_)"""
    code = _natconv_code(f_in, g_in, deviation, stochastic_rounding)
    for t in (f_in, f_out, g_in, g_out):
        _match2(t, Nx, Ny)
    _ptrs_2d_fields(code, Nx, Ny, Temp=Temp)
    call("kb_fused_natconv_vt_step", _t(f_out, "f_out"), _t(f_in, "f_in"), _t(g_out, "g_out"),
         _t(g_in, "g_in"), _t(Temp, "Temp"), Nx, Ny, float(nu_ref), float(T0_visc),
         float(alpha_visc), float(omega_T), float(beta_g), float(T_ref_buoy), float(T_hot),
         float(T_cold), code, _stream())


def compute_temperature_2d_(Temp, g):
    """compute_temperature_2d! -- src/kernels/thermal_2d.jl:113"""
    code = _plain(g)
    Nx, Ny = _dims2(g)
    _ptrs_2d_fields(code, Nx, Ny, Temp=Temp)
    call("kb_compute_temperature_2d", _t(Temp, "Temp"), _t(g, "g"), Nx, Ny, code, _stream())


FACES_2D = {"west": 0, "east": 1, "south": 2, "north": 3}


def collide_thermal_2d_(g, ux, uy, omega_T):
    """collide_thermal_2d! -- src/kernels/thermal_2d.jl:76"""
    code = _plain(g)
    Nx, Ny = _dims2(g)
    _ptrs_2d_fields(code, Nx, Ny, ux=ux, uy=uy)
    call("kb_collide_thermal_2d", _t(g, "g"), _t(ux, "ux"), _t(uy, "uy"), Nx, Ny,
         float(omega_T), code, _stream())


def collide_thermal_masked_2d_(g, ux, uy, omega_T, is_skip):
    """collide_thermal_masked_2d! -- src/kernels/thermal_2d.jl:104"""
    code = _plain(g)
    Nx, Ny = _dims2(g)
    _ptrs_2d_fields(code, Nx, Ny, ux=ux, uy=uy)
    call("kb_collide_thermal_masked_2d", _t(g, "g"), _t(ux, "ux"), _t(uy, "uy"), _mask(is_skip),
         Nx, Ny, float(omega_T), code, _stream())


def _fixed_temp_face_2d_(g, face, T_wall, T_corner, skip):
    code = _plain(g)
    Nx, Ny = _dims2(g)
    call("kb_apply_fixed_temp_face_2d", _t(g, "g"), Nx, Ny, FACES_2D[face], float(T_wall),
         float(T_corner[0]), float(T_corner[1]), int(bool(skip[0])), int(bool(skip[1])), code,
         _stream())


def apply_fixed_temp_south_2d_(g, T_wall, Nx):
    """apply_fixed_temp_south_2d! -- src/kernels/thermal_2d.jl:219"""
    _match2(g, Nx, _dims2(g)[1])
    _fixed_temp_face_2d_(g, "south", T_wall, (T_wall, T_wall), (False, False))


def apply_fixed_temp_north_2d_(g, T_wall, Nx, Ny):
    """apply_fixed_temp_north_2d! -- src/kernels/thermal_2d.jl:248"""
    _match2(g, Nx, Ny)
    _fixed_temp_face_2d_(g, "north", T_wall, (T_wall, T_wall), (False, False))


def apply_fixed_temp_west_2d_(g, T_wall, Ny):
    """apply_fixed_temp_west_2d! -- src/kernels/thermal_2d.jl:311"""
    _match2(g, _dims2(g)[0], Ny)
    _fixed_temp_face_2d_(g, "west", T_wall, (T_wall, T_wall), (False, False))


def apply_fixed_temp_east_2d_(g, T_wall, Nx, Ny):
    """apply_fixed_temp_east_2d! -- src/kernels/thermal_2d.jl:340"""
    _match2(g, Nx, Ny)
    _fixed_temp_face_2d_(g, "east", T_wall, (T_wall, T_wall), (False, False))


def _face_temps(temps, names):
    mask, T = 0, (C.c_double * len(names))()
    for n, name in enumerate(names):
        if temps.get(name) is not None:
            mask |= 1 << n
            T[n] = float(temps[name])
    return mask, T


def apply_fixed_temp_2d_(g, Nx, Ny, west=None, east=None, south=None, north=None):
    """apply_fixed_temp_2d! -- src/kernels/thermal_2d.jl:413 (corner slots of two
    Dirichlet faces flipped once, with the mean temperature)"""
    code = _plain(g)
    _match2(g, Nx, Ny)
    mask, T = _face_temps(dict(west=west, east=east, south=south, north=north), list(FACES_2D))
    call("kb_apply_fixed_temp_2d", _t(g, "g"), Nx, Ny, mask, T, code, _stream())


def collide_boussinesq_2d_(f, Temp, is_solid, omega, beta_g, T_ref):
    """collide_boussinesq_2d! -- src/kernels/thermal_2d.jl:573"""
    code = _plain(f)
    Nx, Ny = _dims2(f)
    _ptrs_2d_fields(code, Nx, Ny, Temp=Temp)
    call("kb_collide_boussinesq_2d", _t(f, "f"), _t(Temp, "Temp"), _mask(is_solid), Nx, Ny,
         float(omega), float(beta_g), float(T_ref), code, _stream())


def collide_boussinesq_vt_2d_(f, Temp, is_solid, nu_ref, T_ref, A_arr, beta_g):
    """collide_boussinesq_vt_2d! -- src/kernels/thermal_2d.jl:553"""
    code = _plain(f)
    Nx, Ny = _dims2(f)
    _ptrs_2d_fields(code, Nx, Ny, Temp=Temp)
    call("kb_collide_boussinesq_vt_2d", _t(f, "f"), _t(Temp, "Temp"), _mask(is_solid), Nx, Ny,
         float(nu_ref), float(T_ref), float(A_arr), float(beta_g), code, _stream())


def collide_boussinesq_vt_modified_2d_(f, Temp, is_solid, nu_ref, T0_visc, alpha_visc, beta_g,
                                       T_ref_buoy):
    """collide_boussinesq_vt_modified_2d! -- src/kernels/thermal_2d.jl:664"""
    code = _plain(f)
    Nx, Ny = _dims2(f)
    _ptrs_2d_fields(code, Nx, Ny, Temp=Temp)
    call("kb_collide_boussinesq_vt_modified_2d", _t(f, "f"), _t(Temp, "Temp"), _mask(is_solid),
         Nx, Ny, float(nu_ref), float(T0_visc), float(alpha_visc), float(beta_g),
         float(T_ref_buoy), code, _stream())


# -------------------------------------------------------------------- D3Q19

def stream_3d_(f_out, f_in, Nx, Ny, Nz):
    """stream_3d! -- src/kernels/collide_stream_3d.jl:119"""
    code = _plain(f_in); _match3(f_in, Nx, Ny, Nz); _match3(f_out, Nx, Ny, Nz)
    call("kb_stream_3d", _t(f_out, "f_out"), _t(f_in, "f_in"), Nx, Ny, Nz, code, _stream())


def collide_3d_(f, is_solid, omega):
    """collide_3d! -- src/kernels/collide_stream_3d.jl:137"""
    code = _plain(f)
    Nx, Ny, Nz = _dims3(f)
    call("kb_collide_3d", _t(f, "f"), _mask(is_solid), Nx, Ny, Nz, float(omega), code, _stream())


FACES_3D = {"west": 0, "east": 1, "south": 2, "north": 3, "bottom": 4, "top": 5}


def apply_zou_he_velocity_3d_(f, face, u_normal, u_tang1, u_tang2):
    """_apply_zou_he_velocity_3d! -- src/kernels/boundary_3d.jl:300"""
    code = _plain(f)
    Nx, Ny, Nz = _dims3(f)
    call("kb_apply_zou_he_velocity_3d", _t(f, "f"), Nx, Ny, Nz, FACES_3D[face],
         float(u_normal), float(u_tang1), float(u_tang2), code, _stream())


def apply_zou_he_top_3d_(f, u_wall_x, Nx, Ny, Nz):
    """apply_zou_he_top_3d! -- src/kernels/boundary_3d.jl:326"""
    code = _plain(f); _match3(f, Nx, Ny, Nz)
    call("kb_apply_zou_he_top_3d", _t(f, "f"), float(u_wall_x), Nx, Ny, Nz, code, _stream())


def apply_zou_he_pressure_3d_(f, face, rho_out=1.0):
    """_apply_zou_he_pressure_3d! -- src/kernels/boundary_3d.jl:307"""
    code = _plain(f)
    Nx, Ny, Nz = _dims3(f)
    call("kb_apply_zou_he_pressure_3d", _t(f, "f"), Nx, Ny, Nz, FACES_3D[face], float(rho_out),
         code, _stream())


def compute_macroscopic_3d_(rho, ux, uy, uz, f):
    """compute_macroscopic_3d! -- src/kernels/macroscopic.jl:75"""
    code = _plain(f)
    Nx, Ny, Nz = _dims3(f)
    _ptrs_3d_fields(code, Nx, Ny, Nz, rho=rho, ux=ux, uy=uy, uz=uz)
    call("kb_compute_macroscopic_3d", _t(rho, "rho"), _t(ux, "ux"), _t(uy, "uy"), _t(uz, "uz"),
         _t(f, "f"), Nx, Ny, Nz, code, _stream())


def collide_thermal_3d_(g, ux, uy, uz, omega_T):
    """collide_thermal_3d! -- src/kernels/thermal_3d.jl:119"""
    code = _plain(g)
    Nx, Ny, Nz = _dims3(g)
    _ptrs_3d_fields(code, Nx, Ny, Nz, ux=ux, uy=uy, uz=uz)
    call("kb_collide_thermal_3d", _t(g, "g"), _t(ux, "ux"), _t(uy, "uy"), _t(uz, "uz"), Nx, Ny,
         Nz, float(omega_T), code, _stream())


def compute_temperature_3d_(Temp, g):
    """compute_temperature_3d! -- src/kernels/thermal_3d.jl:150"""
    code = _plain(g)
    Nx, Ny, Nz = _dims3(g)
    _ptrs_3d_fields(code, Nx, Ny, Nz, Temp=Temp)
    call("kb_compute_temperature_3d", _t(Temp, "Temp"), _t(g, "g"), Nx, Ny, Nz, code, _stream())


def _fixed_temp_face_3d_(g, face, T_wall, T_edge=None, skip=0):
    code = _plain(g)
    Nx, Ny, Nz = _dims3(g)
    te = None if T_edge is None else (C.c_double * 4)(*[float(t) for t in T_edge])
    call("kb_apply_fixed_temp_face_3d", _t(g, "g"), Nx, Ny, Nz, FACES_3D[face], float(T_wall), te,
         int(skip), code, _stream())


def apply_fixed_temp_west_3d_(g, T_wall, Ny, Nz):
    """apply_fixed_temp_west_3d! -- src/kernels/thermal_3d.jl:225"""
    _match3(g, _dims3(g)[0], Ny, Nz)
    _fixed_temp_face_3d_(g, "west", T_wall)


def apply_fixed_temp_east_3d_(g, T_wall, Nx, Ny, Nz):
    """apply_fixed_temp_east_3d! -- src/kernels/thermal_3d.jl:273"""
    _match3(g, Nx, Ny, Nz)
    _fixed_temp_face_3d_(g, "east", T_wall)


def apply_fixed_temp_south_3d_(g, T_wall, Nx, Nz):
    """apply_fixed_temp_south_3d! -- src/kernels/thermal_3d.jl:321"""
    _match3(g, Nx, _dims3(g)[1], Nz)
    _fixed_temp_face_3d_(g, "south", T_wall)


def apply_fixed_temp_north_3d_(g, T_wall, Nx, Ny, Nz):
    """apply_fixed_temp_north_3d! -- src/kernels/thermal_3d.jl:369"""
    _match3(g, Nx, Ny, Nz)
    _fixed_temp_face_3d_(g, "north", T_wall)


def apply_fixed_temp_bottom_3d_(g, T_wall, Nx, Ny):
    """apply_fixed_temp_bottom_3d! -- src/kernels/thermal_3d.jl:417"""
    _match3(g, Nx, Ny, _dims3(g)[2])
    _fixed_temp_face_3d_(g, "bottom", T_wall)


def apply_fixed_temp_top_3d_(g, T_wall, Nx, Ny, Nz):
    """apply_fixed_temp_top_3d! -- src/kernels/thermal_3d.jl:465"""
    _match3(g, Nx, Ny, Nz)
    _fixed_temp_face_3d_(g, "top", T_wall)


def apply_fixed_temp_3d_(g, Nx, Ny, Nz, west=None, east=None, south=None, north=None,
                         bottom=None, top=None):
    """apply_fixed_temp_3d! -- src/kernels/thermal_3d.jl:547 (edge slots of two
    Dirichlet faces flipped once, with the mean temperature)"""
    code = _plain(g)
    _match3(g, Nx, Ny, Nz)
    mask, T = _face_temps(dict(west=west, east=east, south=south, north=north, bottom=bottom,
                               top=top), list(FACES_3D))
    call("kb_apply_fixed_temp_3d", _t(g, "g"), Nx, Ny, Nz, mask, T, code, _stream())


def compute_macroscopic_forced_3d_(rho, ux, uy, uz, f, Fx, Fy, Fz):
    """compute_macroscopic_forced_3d! (src/kernels/macroscopic.jl:155); tensors
    Fx, Fy, Fz select compute_macroscopic_forced_field_3d! (:195)"""
    import torch as _torch
    code = _plain(f)
    Nx, Ny, Nz = _dims3(f)
    _ptrs_3d_fields(code, Nx, Ny, Nz, rho=rho, ux=ux, uy=uy, uz=uz)
    if isinstance(Fx, _torch.Tensor):
        _ptrs_3d_fields(code, Nx, Ny, Nz, Fx=Fx, Fy=Fy, Fz=Fz)
        call("kb_compute_macroscopic_forced_field_3d", _t(rho, "rho"), _t(ux, "ux"), _t(uy, "uy"),
             _t(uz, "uz"), _t(f, "f"), _t(Fx, "Fx"), _t(Fy, "Fy"), _t(Fz, "Fz"), Nx, Ny, Nz,
             code, _stream())
    else:
        call("kb_compute_macroscopic_forced_3d", _t(rho, "rho"), _t(ux, "ux"), _t(uy, "uy"),
             _t(uz, "uz"), _t(f, "f"), Nx, Ny, Nz, float(Fx), float(Fy), float(Fz), code,
             _stream())


def stream_periodic_xz_wall_y_3d_(f_out, f_in, Nx, Ny, Nz):
    """stream_periodic_xz_wall_y_3d! -- src/kernels/stream_periodic_3d.jl:88"""
    code = _plain(f_in); _match3(f_in, Nx, Ny, Nz); _match3(f_out, Nx, Ny, Nz)
    call("kb_stream_periodic_xz_wall_y_3d", _t(f_out, "f_out"), _t(f_in, "f_in"), Nx, Ny, Nz,
         code, _stream())


def slab_fill_ghosts_3d_(f, lo, hi, deviation=False):
    """Ghost planes of a one-rank z-slab on a periodic z axis from the slab's
    own end planes (kb_slab_fill_ghosts_3d); f is (19, nz_alloc, Ny, Nx)."""
    if f.dim() != 4 or f.shape[0] != 19 or not f.is_contiguous():
        raise _arg_error("f must be a contiguous (19, nz_alloc, Ny, Nx) tensor")
    call("kb_slab_fill_ghosts_3d", _t(f, "f"), f.shape[3], f.shape[2], f.shape[1], int(bool(lo)),
         int(bool(hi)), storage_dtype(f, deviation), _stream())


def collide_guo_3d_(f, is_solid, omega, Fx, Fy, Fz):
    """collide_guo_3d! -- src/kernels/collide_guo_3d.jl:190"""
    code = _plain(f)
    Nx, Ny, Nz = _dims3(f)
    call("kb_collide_guo_3d", _t(f, "f"), _mask(is_solid), Nx, Ny, Nz, float(omega), float(Fx),
         float(Fy), float(Fz), code, _stream())


def collide_guo_field_3d_(f, is_solid, Fx_field, Fy_field, Fz_field, omega):
    """collide_guo_field_3d! -- src/kernels/collide_guo_3d.jl:327"""
    code = _plain(f)
    Nx, Ny, Nz = _dims3(f)
    for name, t in (("Fx_field", Fx_field), ("Fy_field", Fy_field), ("Fz_field", Fz_field)):
        if t is None or t.dtype != f.dtype or tuple(t.shape) != (Nz, Ny, Nx):
            raise _arg_error(f"{name} must be a {f.dtype} tensor of shape (Nz, Ny, Nx)")
    call("kb_collide_guo_field_3d", _t(f, "f"), _mask(is_solid), _t(Fx_field, "Fx_field"),
         _t(Fy_field, "Fy_field"), _t(Fz_field, "Fz_field"), Nx, Ny, Nz, float(omega), code,
         _stream())


def collide_boussinesq_3d_(f, Temp, is_solid, omega, beta_g, T_ref):
    """collide_boussinesq_3d! -- src/kernels/thermal_3d.jl:727"""
    code = _plain(f)
    Nx, Ny, Nz = _dims3(f)
    _ptrs_3d_fields(code, Nx, Ny, Nz, Temp=Temp)
    call("kb_collide_boussinesq_3d", _t(f, "f"), _t(Temp, "Temp"), _mask(is_solid), Nx, Ny, Nz,
         float(omega), float(beta_g), float(T_ref), code, _stream())


def set_trt3d_variant(variant: int):
    """0 automatic, 1 one node per thread, 2 nodes x and x+32 per thread,
    3 adjacent node pairs with vector accesses (even Nx), 4 adjacent node
    quads with 8-byte accesses (16-bit storages, Nx % 4 == 0), 5 persistent
    256-node row tiles staged in shared memory by tensor-memory-accelerator
    copies (16-bit storages, Nx % 8 == 0, 16-byte aligned buffers), two rows
    per tile where Ny is even, 6 the staged kernel with one row per tile."""
    call("kb_set_kernel_variant", 1, int(variant))


def set_umma_engine(engine: int):
    """Tensor-core engine of the warm-start network and kb_gemm_bf16: 0 the
    warp-specialised persistent kernel with cp.async staging, 1 one CTA per
    output tile with cp.async staging, 2 (default) the persistent kernel with
    TMA staging into swizzled layouts (shapes it cannot tile run on 1)."""
    call("kb_set_kernel_variant", 2, int(engine))


def periodic_mask(periodic) -> int:
    if isinstance(periodic, int):
        return periodic
    px, py, pz = periodic
    return int(bool(px)) | (int(bool(py)) << 1) | (int(bool(pz)) << 2)


def fused_trt_step_3d_(f_out, f_in, rho, ux, uy, uz, is_solid, Nx, Ny, Nz, nu, Lambda=3 / 16,
                       periodic=(False, False, False), deviation=False, stochastic_rounding=False):
    """Fused D3Q19 TRT step -- the reference's fused_trt_libb_v2_step_3d!
    (src/kernels/li_bb_3d_v2.jl:31) without interpolated-wall links, with
    per-axis periodic wrap.  Moments may be None (then not written).  With
    stochastic_rounding, 16-bit deviation storages are written with
    unbiased stochastic rounding (KB_F16_DEV_SR / KB_BF16_DEV_SR)."""
    code = storage_dtype(f_in, deviation)
    if storage_dtype(f_out, deviation) != code:
        raise _arg_error("f_in and f_out must have the same storage")
    if stochastic_rounding:
        if code not in (KB_F16_DEV, KB_BF16_DEV):
            raise _arg_error("stochastic rounding applies to float16/bfloat16 deviation storage")
        code = KB_F16_DEV_SR if code == KB_F16_DEV else KB_BF16_DEV_SR
    _match3(f_in, Nx, Ny, Nz); _match3(f_out, Nx, Ny, Nz)
    _ptrs_3d_fields(code, Nx, Ny, Nz, rho=rho, ux=ux, uy=uy, uz=uz)
    call("kb_fused_trt_step_3d", _t(f_out, "f_out"), _t(f_in, "f_in"), _t(rho, "rho"),
         _t(ux, "ux"), _t(uy, "uy"), _t(uz, "uz"), _mask(is_solid), Nx, Ny, Nz, float(nu),
         float(Lambda), periodic_mask(periodic), code, _stream())


def fused_trt_step_3d_zrange_(f_out, f_in, rho, ux, uy, uz, is_solid, Nx, Ny, Nz_alloc, k_begin,
                              k_end, nu, Lambda=3 / 16, periodic_xy=(False, False),
                              deviation=False, stochastic_rounding=False):
    """fused_trt_step_3d_ over the z-planes [k_begin, k_end) of a slab
    allocation of Nz_alloc planes; planes k_begin - 1 and k_end are read as
    halo planes.  Every array spans the whole allocation; only the range is
    written.  No reference counterpart (the reference steps whole arrays,
    src/kernels/li_bb_3d_v2.jl:31)."""
    code = storage_dtype(f_in, deviation)
    if storage_dtype(f_out, deviation) != code:
        raise _arg_error("f_in and f_out must have the same storage")
    if stochastic_rounding:
        if code not in (KB_F16_DEV, KB_BF16_DEV):
            raise _arg_error("stochastic rounding applies to float16/bfloat16 deviation storage")
        code = KB_F16_DEV_SR if code == KB_F16_DEV else KB_BF16_DEV_SR
    _match3(f_in, Nx, Ny, Nz_alloc); _match3(f_out, Nx, Ny, Nz_alloc)
    _ptrs_3d_fields(code, Nx, Ny, Nz_alloc, rho=rho, ux=ux, uy=uy, uz=uz)
    if is_solid is not None and tuple(is_solid.shape) != (Nz_alloc, Ny, Nx):
        raise _arg_error(f"is_solid must have shape (Nz_alloc, Ny, Nx) = ({Nz_alloc}, {Ny}, {Nx})")
    px, py = periodic_xy
    call("kb_fused_trt_step_3d_zrange", _t(f_out, "f_out"), _t(f_in, "f_in"), _t(rho, "rho"),
         _t(ux, "ux"), _t(uy, "uy"), _t(uz, "uz"), _mask(is_solid), Nx, Ny, Nz_alloc,
         int(k_begin), int(k_end), float(nu), float(Lambda), int(bool(px)) | 2 * int(bool(py)),
         code, _stream())


def fused_trt_libb_v2_step_3d_(f_out, f_in, rho, ux, uy, uz, is_solid, q_wall, uw_link_x,
                               uw_link_y, uw_link_z, Nx, Ny, Nz, nu, Lambda=3 / 16,
                               periodic=(False, False, False)):
    """fused_trt_libb_v2_step_3d! -- src/kernels/li_bb_3d_v2.jl:31"""
    code = _plain(f_in)
    _match3(f_in, Nx, Ny, Nz); _match3(f_out, Nx, Ny, Nz)
    for name, t in (("q_wall", q_wall), ("uw_link_x", uw_link_x), ("uw_link_y", uw_link_y),
                    ("uw_link_z", uw_link_z)):
        if t is None or t.dtype != f_in.dtype or tuple(t.shape) != tuple(f_in.shape):
            raise _arg_error(f"{name} must be a {f_in.dtype} tensor shaped like f")
    _ptrs_3d_fields(code, Nx, Ny, Nz, rho=rho, ux=ux, uy=uy, uz=uz)
    call("kb_fused_trt_libb_step_3d", _t(f_out, "f_out"), _t(f_in, "f_in"), _t(rho, "rho"),
         _t(ux, "ux"), _t(uy, "uy"), _t(uz, "uz"), _mask(is_solid), _t(q_wall, "q_wall"),
         _t(uw_link_x, "uw_link_x"), _t(uw_link_y, "uw_link_y"), _t(uw_link_z, "uw_link_z"),
         Nx, Ny, Nz, float(nu), float(Lambda), periodic_mask(periodic), code, _stream())


def fused_trt_libb_links_step_3d_(f_out, f_in, rho, ux, uy, uz, links, nu, Lambda=3 / 16,
                                  periodic=(False, False, False), deviation=False,
                                  stochastic_rounding=False):
    """fused_trt_libb_v2_step_3d! with a compact cut-link table
    (`libb.CutLinks`); any storage (float16/bfloat16 and deviation=True hold
    f - w; stochastic_rounding as in fused_trt_step_3d_)."""
    code = storage_dtype(f_in, deviation)
    if stochastic_rounding:
        if code not in (KB_F16_DEV, KB_BF16_DEV):
            raise _arg_error("stochastic rounding applies to float16/bfloat16 deviation storage")
        code = KB_F16_DEV_SR if code == KB_F16_DEV else KB_BF16_DEV_SR
    Nx, Ny, Nz = links.Nx, links.Ny, links.Nz
    _match3(f_in, Nx, Ny, Nz); _match3(f_out, Nx, Ny, Nz)
    _ptrs_3d_fields(code, Nx, Ny, Nz, rho=rho, ux=ux, uy=uy, uz=uz)
    call("kb_fused_trt_libb_links_step_3d", _t(f_out, "f_out"), _t(f_in, "f_in"), _t(rho, "rho"),
         _t(ux, "ux"), _t(uy, "uy"), _t(uz, "uz"), links.handle, float(nu), float(Lambda),
         periodic_mask(periodic), code, _stream())


def stream_periodic_xz_movingwall_y_3d_(f_out, f_in, Ub, Ut, Nx, Ny, Nz, rho_w=1.0):
    """stream_periodic_xz_movingwall_y_3d! -- src/kernels/stream_periodic_3d.jl:178"""
    code = _plain(f_in); _match3(f_in, Nx, Ny, Nz); _match3(f_out, Nx, Ny, Nz)
    call("kb_stream_periodic_xz_movingwall_y_3d", _t(f_out, "f_out"), _t(f_in, "f_in"),
         float(Ub), float(Ut), float(rho_w), Nx, Ny, Nz, code, _stream())


# ------------------------------------------------------- precision + FP64 sums

def convert_populations(dst, src, dst_deviation=False, src_deviation=False):
    """Convert populations between storages (f <-> f - w_q, any precision)."""
    if dst.shape != src.shape:
        raise _arg_error("src and dst shapes differ")
    Q = int(src.shape[0])
    n = src.numel() // Q
    call("kb_convert_populations", _t(dst, "dst"), storage_dtype(dst, dst_deviation),
         _t(src, "src"), storage_dtype(src, src_deviation), Q, n, _stream())


def set_stochastic_seed(seed: int):
    """Seed the random bits of the stochastic-rounding storages (synchronises)."""
    call("kb_set_stochastic_seed", C.c_uint(seed & 0xFFFFFFFF), _stream())


def get_stochastic_seed() -> int:
    """The launch counter that seeds the stochastic-rounding bits (synchronises)."""
    out = C.c_uint(0)
    call("kb_get_stochastic_seed", C.byref(out), _stream())
    return int(out.value)


def staged_step_timed_out() -> bool:
    """True if a staged step (variant 5) gave up a bounded wait on its copies
    since the last call; clears the flag (synchronises the stream)."""
    out = C.c_int(0)
    call("kb_staged_step_status", C.byref(out), _stream())
    return bool(out.value)


def mass(f, deviation=False) -> float:
    """FP64 compensated total mass sum(f) (synchronises the stream)."""
    out = C.c_double()
    Q = int(f.shape[0])
    call("kb_mass", _t(f, "f"), Q, f.numel() // Q, storage_dtype(f, deviation), C.byref(out),
         _stream())
    return out.value


def residual(ux, uy, ux_prev, uy_prev, uz=None, uz_prev=None, is_solid=None) -> float:
    """r_u = ||u - u_prev|| / ||u|| over fluid nodes (FP64 sums; synchronises)."""
    code = KB_F64 if ux.dtype == torch.float64 else KB_F32
    out = C.c_double()
    call("kb_residual", _t(ux, "ux"), _t(uy, "uy"), _t(uz, "uz"), _t(ux_prev, "ux_prev"),
         _t(uy_prev, "uy_prev"), _t(uz_prev, "uz_prev"), _mask(is_solid), ux.numel(), code,
         C.byref(out), _stream())
    return out.value


def synchronize():
    """KernelAbstractions.synchronize(backend)."""
    call("kb_sync", _stream())


__all__ = [n for n in dir() if n.endswith("_") and not n.startswith("_")] + [
    "trt_rates", "convert_populations", "mass", "residual", "synchronize", "storage_dtype",
    "set_trt3d_variant", "set_stochastic_seed", "get_stochastic_seed", "thermal_deviation", "staged_step_timed_out", "set_umma_engine", "AA_SWAP_2D",
    "torch_dtype", "field_dtype", "periodic_mask", "FACES_3D"]

_ = _lib  # keep the module import explicit for readers
