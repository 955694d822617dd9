"""
    KrakenB200

Julia binding of libkrakenb200.so: the `b200` backend of Kraken.jl's
stream-collide path.  Each method below `ccall`s one entry point of
include/krakenb200.h with the raw device pointers of CuArrays (Kraken.jl's
column-major (Nx, Ny, Q) arrays pass unchanged) and CUDA.jl's current
stream.  A non-zero status raises `ArgumentError` (bad argument or
unsupported combination) or `ErrorException` (CUDA failure) carrying
`kb_last_error()`; nothing ever falls back to the CPU.

Not exercised in this repository (no Julia toolchain on the build machine);
the same entry points are exercised through ctypes by tests/.
"""
module KrakenB200

using CUDA

const LIB = get(ENV, "KRAKENB200_LIB", joinpath(@__DIR__, "..", "libkrakenb200.so"))

const KB_F64, KB_F32, KB_F32_DEV, KB_F16_DEV, KB_BF16_DEV = 0, 1, 2, 3, 4

struct B200Backend end

kb_dtype(::Type{Float64}) = KB_F64
kb_dtype(::Type{Float32}) = KB_F32
kb_dtype(::Type{Float16}) = KB_F16_DEV

_stream() = CUDA.stream().handle
_ptr(a::CuArray) = reinterpret(Ptr{Cvoid}, pointer(a))
_ptr(::Nothing) = C_NULL
_mask(a::CuArray{Bool}) = reinterpret(Ptr{UInt8}, pointer(a))
_mask(::Nothing) = Ptr{UInt8}(C_NULL)

function _check(name::AbstractString, rc::Cint)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:kb_last_error, LIB), Cstring, ()))
    rc in (-1, -2) && throw(ArgumentError("$name: $msg"))
    error("$name failed ($rc): $msg")
end

"stream_2d!(f_out, f_in, Nx, Ny) -- src/kernels/collide_stream_2d.jl:77"
function stream_2d!(f_out::CuArray{T,3}, f_in::CuArray{T,3}, Nx, Ny) where {T}
    _check("kb_stream_2d", ccall((:kb_stream_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cvoid}),
        _ptr(f_out), _ptr(f_in), Nx, Ny, kb_dtype(T), _stream()))
end

"collide_2d!(f, is_solid, ω) -- src/kernels/collide_stream_2d.jl:96"
function collide_2d!(f::CuArray{T,3}, is_solid, ω) where {T}
    Nx, Ny = size(f, 1), size(f, 2)
    _check("kb_collide_2d", ccall((:kb_collide_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint, Cdouble, Cint, Ptr{Cvoid}),
        _ptr(f), _mask(is_solid), Nx, Ny, ω, kb_dtype(T), _stream()))
end

"apply_zou_he_north_2d!(f, u, Nx, Ny) -- src/kernels/boundary_2d.jl:56"
function apply_zou_he_north_2d!(f::CuArray{T,3}, u, Nx, Ny) where {T}
    _check("kb_apply_zou_he_north_2d", ccall((:kb_apply_zou_he_north_2d, LIB), Cint,
        (Ptr{Cvoid}, Cdouble, Cint, Cint, Cint, Ptr{Cvoid}),
        _ptr(f), u, Nx, Ny, kb_dtype(T), _stream()))
end

"compute_macroscopic_2d!(ρ, ux, uy, f) -- src/kernels/macroscopic.jl:32"
function compute_macroscopic_2d!(ρ, ux, uy, f::CuArray{T,3}) where {T}
    Nx, Ny = size(ρ)
    _check("kb_compute_macroscopic_2d", ccall((:kb_compute_macroscopic_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cvoid}),
        _ptr(ρ), _ptr(ux), _ptr(uy), _ptr(f), Nx, Ny, kb_dtype(T), _stream()))
end

"fused_bgk_step!(f_out, f_in, ρ, ux, uy, is_solid, Nx, Ny, ω) -- src/kernels/fused_bgk_2d.jl:67"
function fused_bgk_step!(f_out::CuArray{T,3}, f_in::CuArray{T,3}, ρ, ux, uy, is_solid,
                         Nx, Ny, ω) where {T}
    _check("kb_fused_bgk_step", ccall((:kb_fused_bgk_step, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint,
         Cdouble, Cint, Ptr{Cvoid}),
        _ptr(f_out), _ptr(f_in), _ptr(ρ), _ptr(ux), _ptr(uy), _mask(is_solid), Nx, Ny, ω,
        kb_dtype(T), _stream()))
end

"fused_trt_step!(f_out, f_in, ρ, ux, uy, is_solid, Nx, Ny, ν; Λ) -- src/kernels/fused_trt_2d.jl:145"
function fused_trt_step!(f_out::CuArray{T,3}, f_in::CuArray{T,3}, ρ, ux, uy, is_solid,
                         Nx, Ny, ν; Λ::Real=3/16) where {T}
    _check("kb_fused_trt_step", ccall((:kb_fused_trt_step, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint,
         Cdouble, Cdouble, Cint, Ptr{Cvoid}),
        _ptr(f_out), _ptr(f_in), _ptr(ρ), _ptr(ux), _ptr(uy), _mask(is_solid), Nx, Ny, ν, Λ,
        kb_dtype(T), _stream()))
end

"collide_mrt_2d!(f, is_solid, ν; s_e, s_eps, s_q) -- src/kernels/collide_mrt_2d.jl:118"
function collide_mrt_2d!(f::CuArray{T,3}, is_solid, ν; s_e=1.4, s_eps=1.4, s_q=1.2) where {T}
    Nx, Ny = size(f, 1), size(f, 2)
    _check("kb_collide_mrt_2d", ccall((:kb_collide_mrt_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint, Cdouble, Cdouble, Cdouble, Cdouble, Cint,
         Ptr{Cvoid}),
        _ptr(f), _mask(is_solid), Nx, Ny, ν, s_e, s_eps, s_q, kb_dtype(T), _stream()))
end

"fused_natconv_step!(...) -- src/kernels/fused_thermal_2d.jl:251"
function fused_natconv_step!(f_out::CuArray{T,3}, f_in, g_out, g_in, Temp, Nx, Ny,
                             ω_f, ω_T, β_g, T_ref_buoy, T_hot, T_cold) where {T}
    _check("kb_fused_natconv_step", ccall((:kb_fused_natconv_step, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cdouble,
         Cdouble, Cdouble, Cdouble, Cdouble, Cdouble, Cint, Ptr{Cvoid}),
        _ptr(f_out), _ptr(f_in), _ptr(g_out), _ptr(g_in), _ptr(Temp), Nx, Ny, ω_f, ω_T, β_g,
        T_ref_buoy, T_hot, T_cold, kb_dtype(T), _stream()))
end

"Fused D3Q19 TRT step (li_bb_3d_v2.jl:31 without LI-BB links), periodic = (px, py, pz)."
function fused_trt_step_3d!(f_out::CuArray{T,4}, f_in::CuArray{T,4}, ρ, ux, uy, uz, is_solid,
                            Nx, Ny, Nz, ν; Λ::Real=3/16, periodic=(false, false, false),
                            dtype::Integer=kb_dtype(T)) where {T}
    per = Int(periodic[1]) | (Int(periodic[2]) << 1) | (Int(periodic[3]) << 2)
    _check("kb_fused_trt_step_3d", ccall((:kb_fused_trt_step_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8},
         Cint, Cint, Cint, Cdouble, Cdouble, Cint, Cint, Ptr{Cvoid}),
        _ptr(f_out), _ptr(f_in), _ptr(ρ), _ptr(ux), _ptr(uy), _ptr(uz), _mask(is_solid),
        Nx, Ny, Nz, ν, Λ, per, dtype, _stream()))
end

"stream_3d!(f_out, f_in, Nx, Ny, Nz) -- src/kernels/collide_stream_3d.jl:119"
function stream_3d!(f_out::CuArray{T,4}, f_in::CuArray{T,4}, Nx, Ny, Nz) where {T}
    _check("kb_stream_3d", ccall((:kb_stream_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Cint, Ptr{Cvoid}),
        _ptr(f_out), _ptr(f_in), Nx, Ny, Nz, kb_dtype(T), _stream()))
end

"collide_3d!(f, is_solid, ω) -- src/kernels/collide_stream_3d.jl:137"
function collide_3d!(f::CuArray{T,4}, is_solid, ω) where {T}
    Nx, Ny, Nz = size(f, 1), size(f, 2), size(f, 3)
    _check("kb_collide_3d", ccall((:kb_collide_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint, Cint, Cdouble, Cint, Ptr{Cvoid}),
        _ptr(f), _mask(is_solid), Nx, Ny, Nz, ω, kb_dtype(T), _stream()))
end

"apply_zou_he_top_3d!(f, u, Nx, Ny, Nz) -- src/kernels/boundary_3d.jl:326"
function apply_zou_he_top_3d!(f::CuArray{T,4}, u, Nx, Ny, Nz) where {T}
    _check("kb_apply_zou_he_top_3d", ccall((:kb_apply_zou_he_top_3d, LIB), Cint,
        (Ptr{Cvoid}, Cdouble, Cint, Cint, Cint, Cint, Ptr{Cvoid}),
        _ptr(f), u, Nx, Ny, Nz, kb_dtype(T), _stream()))
end

"compute_macroscopic_3d!(ρ, ux, uy, uz, f) -- src/kernels/macroscopic.jl:75"
function compute_macroscopic_3d!(ρ, ux, uy, uz, f::CuArray{T,4}) where {T}
    Nx, Ny, Nz = size(ρ)
    _check("kb_compute_macroscopic_3d", ccall((:kb_compute_macroscopic_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Cint,
         Ptr{Cvoid}),
        _ptr(ρ), _ptr(ux), _ptr(uy), _ptr(uz), _ptr(f), Nx, Ny, Nz, kb_dtype(T), _stream()))
end

end # module
