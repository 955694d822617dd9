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

"""
Fused D3Q19 TRT step over the z-planes `k_begin .. k_end-1` (0-based, as in the C
header) of a z-slab allocation of `Nz_alloc` planes whose planes 0 and `Nz_alloc-1`
are halo planes, read as they are.  Every array spans the whole allocation; only the
range is written.  No reference counterpart (the reference steps whole arrays).
"""
function fused_trt_step_3d_zrange!(f_out::CuArray{T,4}, f_in::CuArray{T,4}, ρ, ux, uy, uz,
                                   is_solid, Nx, Ny, Nz_alloc, k_begin, k_end, ν;
                                   Λ::Real=3/16, periodic_xy=(false, false),
                                   dtype::Integer=kb_dtype(T)) where {T}
    per = Int(periodic_xy[1]) | (Int(periodic_xy[2]) << 1)
    _check("kb_fused_trt_step_3d_zrange", ccall((:kb_fused_trt_step_3d_zrange, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8},
         Cint, Cint, Cint, Cint, Cint, Cdouble, Cdouble, Cint, Cint, Ptr{Cvoid}),
        _ptr(f_out), _ptr(f_in), _ptr(ρ), _ptr(ux), _ptr(uy), _ptr(uz), _mask(is_solid),
        Nx, Ny, Nz_alloc, k_begin, k_end, ν, Λ, per, dtype, _stream()))
end

"Ghost planes of one z-slab on a periodic z axis from its own end planes (one launch)."
function slab_fill_ghosts_3d!(f::CuArray{T,4}, lo::Bool, hi::Bool;
                              dtype::Integer=kb_dtype(T)) where {T}
    Nx, Ny, Nz_alloc = size(f, 1), size(f, 2), size(f, 3)
    _check("kb_slab_fill_ghosts_3d", ccall((:kb_slab_fill_ghosts_3d, LIB), Cint,
        (Ptr{Cvoid}, Cint, Cint, Cint, Cint, Cint, Cint, Ptr{Cvoid}),
        _ptr(f), Nx, Ny, Nz_alloc, Int(lo), Int(hi), dtype, _stream()))
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

"collide_thermal_2d!(g, ux, uy, ω_T) -- src/kernels/thermal_2d.jl:76"
function collide_thermal_2d!(g::CuArray{T,3}, ux, uy, ω_T) where {T}
    Nx, Ny = size(g, 1), size(g, 2)
    _check("kb_collide_thermal_2d", ccall((:kb_collide_thermal_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cdouble, Cint, Ptr{Cvoid}),
        _ptr(g), _ptr(ux), _ptr(uy), Nx, Ny, ω_T, kb_dtype(T), _stream()))
end

# One face of half-way anti-bounce-back; face 0 west, 1 east, 2 south, 3 north.
function _fixed_temp_face_2d!(g::CuArray{T,3}, face, T_wall, T_c, skip_c) where {T}
    Nx, Ny = size(g, 1), size(g, 2)
    _check("kb_apply_fixed_temp_face_2d", ccall((:kb_apply_fixed_temp_face_2d, LIB), Cint,
        (Ptr{Cvoid}, Cint, Cint, Cint, Cdouble, Cdouble, Cdouble, Cint, Cint, Cint, Ptr{Cvoid}),
        _ptr(g), Nx, Ny, face, T_wall, T_c[1], T_c[2], skip_c[1], skip_c[2], kb_dtype(T),
        _stream()))
end

"apply_fixed_temp_west_2d!(g, T_wall, Ny) -- src/kernels/thermal_2d.jl:311"
apply_fixed_temp_west_2d!(g::CuArray, T_wall, Ny) =
    _fixed_temp_face_2d!(g, 0, T_wall, (T_wall, T_wall), (false, false))
"apply_fixed_temp_east_2d!(g, T_wall, Nx, Ny) -- src/kernels/thermal_2d.jl:340"
apply_fixed_temp_east_2d!(g::CuArray, T_wall, Nx, Ny) =
    _fixed_temp_face_2d!(g, 1, T_wall, (T_wall, T_wall), (false, false))
"apply_fixed_temp_south_2d!(g, T_wall, Nx) -- src/kernels/thermal_2d.jl:219"
apply_fixed_temp_south_2d!(g::CuArray, T_wall, Nx) =
    _fixed_temp_face_2d!(g, 2, T_wall, (T_wall, T_wall), (false, false))
"apply_fixed_temp_north_2d!(g, T_wall, Nx, Ny) -- src/kernels/thermal_2d.jl:248"
apply_fixed_temp_north_2d!(g::CuArray, T_wall, Nx, Ny) =
    _fixed_temp_face_2d!(g, 3, T_wall, (T_wall, T_wall), (false, false))

"apply_fixed_temp_2d!(g, Nx, Ny; west, east, south, north) -- src/kernels/thermal_2d.jl:413"
function apply_fixed_temp_2d!(g::CuArray{T,3}, Nx, Ny; west=nothing, east=nothing,
                              south=nothing, north=nothing) where {T}
    temps = (west, east, south, north)
    mask = UInt32(0); Tf = zeros(Float64, 4)
    for (n, t) in enumerate(temps)
        t === nothing && continue
        mask |= UInt32(1) << (n - 1); Tf[n] = Float64(t)
    end
    _check("kb_apply_fixed_temp_2d", ccall((:kb_apply_fixed_temp_2d, LIB), Cint,
        (Ptr{Cvoid}, Cint, Cint, Cuint, Ptr{Cdouble}, Cint, Ptr{Cvoid}),
        _ptr(g), Nx, Ny, mask, Tf, kb_dtype(T), _stream()))
end

"collide_boussinesq_2d!(f, Temp, is_solid, ω, β_g, T_ref) -- src/kernels/thermal_2d.jl:573"
function collide_boussinesq_2d!(f::CuArray{T,3}, Temp, is_solid, ω, β_g, T_ref) where {T}
    Nx, Ny = size(f, 1), size(f, 2)
    _check("kb_collide_boussinesq_2d", ccall((:kb_collide_boussinesq_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint, Cdouble, Cdouble, Cdouble, Cint,
         Ptr{Cvoid}),
        _ptr(f), _ptr(Temp), _mask(is_solid), Nx, Ny, ω, β_g, T_ref, kb_dtype(T), _stream()))
end

"fused_trt_libb_v2_step!(f_out, f_in, ρ, ux, uy, is_solid, q_wall, uw_x, uw_y, Nx, Ny, ν; Λ) -- src/kernels/li_bb_2d_v2.jl:104"
function fused_trt_libb_v2_step!(f_out::CuArray{T,3}, f_in::CuArray{T,3}, ρ, ux, uy, is_solid,
                                 q_wall, uw_link_x, uw_link_y, Nx, Ny, ν;
                                 Λ::Real=3/16) where {T}
    _check("kb_fused_trt_libb_step", ccall((:kb_fused_trt_libb_step, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8}, Ptr{Cvoid},
         Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cdouble, Cdouble, Cint, Ptr{Cvoid}),
        _ptr(f_out), _ptr(f_in), _ptr(ρ), _ptr(ux), _ptr(uy), _mask(is_solid), _ptr(q_wall),
        _ptr(uw_link_x), _ptr(uw_link_y), Nx, Ny, ν, Λ, kb_dtype(T), _stream()))
end

"fused_trt_libb_v2_step_3d!(...) -- src/kernels/li_bb_3d_v2.jl:31"
function fused_trt_libb_v2_step_3d!(f_out::CuArray{T,4}, f_in::CuArray{T,4}, ρ, ux, uy, uz,
                                    is_solid, q_wall, uw_link_x, uw_link_y, uw_link_z,
                                    Nx, Ny, Nz, ν; Λ::Real=3/16) where {T}
    _check("kb_fused_trt_libb_step_3d", ccall((:kb_fused_trt_libb_step_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8},
         Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Cdouble, Cdouble,
         Cint, Cint, Ptr{Cvoid}),
        _ptr(f_out), _ptr(f_in), _ptr(ρ), _ptr(ux), _ptr(uy), _ptr(uz), _mask(is_solid),
        _ptr(q_wall), _ptr(uw_link_x), _ptr(uw_link_y), _ptr(uw_link_z), Nx, Ny, Nz, ν, Λ, 0,
        kb_dtype(T), _stream()))
end

"collide_thermal_3d!(g, ux, uy, uz, ω_T) -- src/kernels/thermal_3d.jl:119"
function collide_thermal_3d!(g::CuArray{T,4}, ux, uy, uz, ω_T) where {T}
    Nx, Ny, Nz = size(g, 1), size(g, 2), size(g, 3)
    _check("kb_collide_thermal_3d", ccall((:kb_collide_thermal_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Cdouble, Cint,
         Ptr{Cvoid}),
        _ptr(g), _ptr(ux), _ptr(uy), _ptr(uz), Nx, Ny, Nz, ω_T, kb_dtype(T), _stream()))
end

"compute_temperature_3d!(Temp, g) -- src/kernels/thermal_3d.jl:150"
function compute_temperature_3d!(Temp, g::CuArray{T,4}) where {T}
    Nx, Ny, Nz = size(Temp)
    _check("kb_compute_temperature_3d", ccall((:kb_compute_temperature_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Cint, Ptr{Cvoid}),
        _ptr(Temp), _ptr(g), Nx, Ny, Nz, kb_dtype(T), _stream()))
end

"apply_fixed_temp_3d!(g, Nx, Ny, Nz; west, east, south, north, bottom, top) -- src/kernels/thermal_3d.jl:547"
function apply_fixed_temp_3d!(g::CuArray{T,4}, Nx, Ny, Nz; west=nothing, east=nothing,
                              south=nothing, north=nothing, bottom=nothing,
                              top=nothing) where {T}
    temps = (west, east, south, north, bottom, top)
    mask = UInt32(0); Tf = zeros(Float64, 6)
    for (n, t) in enumerate(temps)
        t === nothing && continue
        mask |= UInt32(1) << (n - 1); Tf[n] = Float64(t)
    end
    _check("kb_apply_fixed_temp_3d", ccall((:kb_apply_fixed_temp_3d, LIB), Cint,
        (Ptr{Cvoid}, Cint, Cint, Cint, Cuint, Ptr{Cdouble}, Cint, Ptr{Cvoid}),
        _ptr(g), Nx, Ny, Nz, mask, Tf, kb_dtype(T), _stream()))
end

"collide_boussinesq_3d!(f, Temp, is_solid, ω, β_g, T_ref) -- src/kernels/thermal_3d.jl:727"
function collide_boussinesq_3d!(f::CuArray{T,4}, Temp, is_solid, ω, β_g, T_ref) where {T}
    Nx, Ny, Nz = size(f, 1), size(f, 2), size(f, 3)
    _check("kb_collide_boussinesq_3d", ccall((:kb_collide_boussinesq_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint, Cint, Cdouble, Cdouble, Cdouble, Cint,
         Ptr{Cvoid}),
        _ptr(f), _ptr(Temp), _mask(is_solid), Nx, Ny, Nz, ω, β_g, T_ref, kb_dtype(T), _stream()))
end

end # module
