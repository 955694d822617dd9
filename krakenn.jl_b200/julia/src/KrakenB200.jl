"""
    KrakenB200

The `b200` backend of Kraken.jl's stream-collide path, as a KernelAbstractions
backend whose kernels are the hand-written sm_100a CUDA kernels of
libkrakenb200.so (C ABI: include/krakenb200.h).

- `B200Backend <: KernelAbstractions.GPU` is what Kraken's drivers receive as
  `backend` (from `run_cavity_2d(config; backend=B200Backend())`, or from the
  `.krk` directive `Backend b200` through Kraken's
  `_require_functional_gpu_backend(:b200, <this package>, :B200Backend)`).
- `KernelAbstractions.zeros/ones/allocate(B200Backend(), T, dims...)` return
  `B200Array`s: CUDA device memory in Kraken's column-major layout, wrapped
  in a type of their own so that a plain `CuArray` keeps the `:cuda`
  backend.  `KernelAbstractions.get_backend(::B200Array)` is `B200Backend()`.
- Methods of Kraken's kernel wrappers (`Kraken.fused_bgk_step!`,
  `Kraken.stream_2d!`, ... the list at the end of this file) are defined
  for `B200Array` populations.  Each checks the element type and size of
  every array argument, then `ccall`s the library with the raw device
  pointers and CUDA.jl's current stream.  A non-zero status raises
  `ArgumentError` (bad argument, unsupported combination) or
  `ErrorException` (CUDA failure) carrying `kb_last_error()`.
- Nothing falls back: this backend has no KernelAbstractions compiler, so a
  Kraken kernel that is not listed here raises a `MethodError` instead of
  running elsewhere.

Kraken's kernels take Float64 or Float32 populations with fields of the same
type.  The deviation storages of the B200 path (f - w_q held in Float32,
Float16 or BFloat16, collided in Float32) are reached only through this
package's own `fused_trt_step_3d!` with an explicit `storage` keyword; a
Float16 array is never taken for a deviation array by accident.

The Python package beside this one exercises the same entry points through
ctypes in its test suite; this file has not been run here (no Julia
toolchain on the build machine).
"""
module KrakenB200

using CUDA
import KernelAbstractions
const KA = KernelAbstractions
import Kraken

export B200Backend, B200Array, functional

const LIB = get(ENV, "KRAKENB200_LIB",
                normpath(joinpath(@__DIR__, "..", "..", "libkrakenb200.so")))

# kb_status and kb_dtype of include/krakenb200.h
const KB_ERR_ARG, KB_ERR_UNSUPPORTED = -1, -2
const KB_F64, KB_F32, KB_F32_DEV, KB_F16_DEV, KB_BF16_DEV = 0, 1, 2, 3, 4
const KB_F16_DEV_SR, KB_BF16_DEV_SR = 5, 6

# ------------------------------------------------------------ availability

"""
    functional() -> Bool

`true` when CUDA.jl has a usable current device of compute capability 10.0
(B200: the library holds sm_100a code only) and libkrakenb200.so loads.
Kraken's `_require_functional_gpu_backend` calls this before it hands out
`B200Backend()`.
"""
function functional()
    try
        CUDA.functional() || return false
        CUDA.capability(CUDA.device()) == v"10.0" || return false
        isfile(LIB) || return false
        v = unsafe_string(ccall((:kb_version, LIB), Cstring, ()))
        return startswith(v, "krakenb200")
    catch
        return false
    end
end

# --------------------------------------------------------- backend, arrays

"""
    B200Backend()

KernelAbstractions backend of the B200 stream-collide library.
"""
struct B200Backend <: KA.GPU end

"""
    B200Array{T,N}

Device array of the b200 backend: a `CuArray{T,N}` (Kraken's column-major
layout, so the library reads it zero-copy) in a type of its own.  Bulk
operations (`fill!`, `copyto!` to and from host arrays, `Array`) work;
element access follows CUDA.jl's scalar-indexing rules.
"""
struct B200Array{T,N} <: AbstractArray{T,N}
    data::CuArray{T,N}
end

Base.parent(a::B200Array) = a.data
Base.size(a::B200Array) = size(a.data)
Base.IndexStyle(::Type{<:B200Array}) = IndexLinear()
Base.getindex(a::B200Array, i::Int) = a.data[i]
Base.setindex!(a::B200Array, v, i::Int) = (a.data[i] = v; a)
Base.similar(a::B200Array, ::Type{S}, dims::Dims) where {S} = B200Array(similar(a.data, S, dims))
Base.fill!(a::B200Array, x) = (fill!(a.data, x); a)
Base.copyto!(d::B200Array, s::B200Array) = (copyto!(d.data, s.data); d)
Base.copyto!(d::B200Array, s::Array) = (copyto!(d.data, s); d)
Base.copyto!(d::Array, s::B200Array) = (copyto!(d, s.data); d)
Base.Array(a::B200Array) = Array(a.data)
Base.collect(a::B200Array) = Array(a.data)
Base.show(io::IO, a::B200Array{T,N}) where {T,N} = print(io, "B200Array{$T,$N}", size(a))
Base.show(io::IO, ::MIME"text/plain", a::B200Array) = show(io, a)

KA.get_backend(::B200Array) = B200Backend()

function KA.allocate(::B200Backend, ::Type{T}, dims::Tuple; unified::Bool=false) where {T}
    unified && throw(ArgumentError("b200 backend: unified memory is not supported"))
    return B200Array(CuArray{T}(undef, dims))
end

KA.synchronize(::B200Backend) = _check("kb_sync", ccall((:kb_sync, LIB), Cint, (Ptr{Cvoid},),
                                                       _stream()))

# --------------------------------------------------------------- plumbing

_stream() = CUDA.stream().handle

function _check(name::AbstractString, rc::Integer)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:kb_last_error, LIB), Cstring, ()))
    rc in (KB_ERR_ARG, KB_ERR_UNSUPPORTED) && throw(ArgumentError("$name: $msg"))
    error("$name failed ($rc): $msg")
end

# kb_dtype of Kraken's population storages (reference arithmetic)
function _plain(name, f::B200Array)
    T = eltype(f)
    T === Float64 && return KB_F64
    T === Float32 && return KB_F32
    throw(ArgumentError("$name: the b200 backend runs Kraken's kernels on Float64 or Float32 " *
                        "populations, got $T; deviation storage (f - w_q) is " *
                        "KrakenB200.fused_trt_step_3d! with an explicit `storage` keyword"))
end

# The device pointer of a B200Array{T} of size `dims`, after checking both.
function _arr(name, a, ::Type{T}, dims::Tuple) where {T}
    a isa B200Array || throw(ArgumentError(
        "$name: expected a B200Array (allocated on B200Backend()), got $(typeof(a))"))
    eltype(a) === T || throw(ArgumentError(
        "$name: element type $(eltype(a)), expected $T (fields take the population's type; " *
        "Float32 for deviation storages)"))
    size(a) == dims || throw(ArgumentError("$name: size $(size(a)), expected $dims"))
    return reinterpret(Ptr{Cvoid}, pointer(a.data))
end

# Optional field: `nothing` passes NULL (the kernel skips that write).
_opt(name, a, ::Type{T}, dims) where {T} = a === nothing ? C_NULL : _arr(name, a, T, dims)

# Solid mask: a B200Array{Bool} of the grid's size, or nothing (no solid node).
function _mask(a, dims::Tuple)
    a === nothing && return Ptr{UInt8}(C_NULL)
    return reinterpret(Ptr{UInt8}, _arr("is_solid", a, Bool, dims))
end

_ftype(code) = code == KB_F64 ? Float64 : Float32

function _sync(sync::Bool)
    sync && KA.synchronize(B200Backend())
    return nothing
end

# --------------------------------------------------------------- D2Q9

"stream_2d!(f_out, f_in, Nx, Ny; sync) -- src/kernels/collide_stream_2d.jl:77"
function Kraken.stream_2d!(f_out::B200Array, f_in::B200Array, Nx, Ny; sync=false)
    c = _plain("stream_2d!", f_in); T = eltype(f_in); d = (Nx, Ny, 9)
    _check("kb_stream_2d", ccall((:kb_stream_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cvoid}),
        _arr("f_out", f_out, T, d), _arr("f_in", f_in, T, d), Nx, Ny, c, _stream()))
    _sync(sync)
end

"collide_2d!(f, is_solid, ω; sync) -- src/kernels/collide_stream_2d.jl:96"
function Kraken.collide_2d!(f::B200Array, is_solid, ω; sync=false)
    c = _plain("collide_2d!", f); Nx, Ny = size(f, 1), size(f, 2)
    _check("kb_collide_2d", ccall((:kb_collide_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint, Cdouble, Cint, Ptr{Cvoid}),
        _arr("f", f, eltype(f), (Nx, Ny, 9)), _mask(is_solid, (Nx, Ny)), Nx, Ny, ω, c,
        _stream()))
    _sync(sync)
end

"apply_zou_he_north_2d!(f, u_wall_x, Nx, Ny) -- src/kernels/boundary_2d.jl:56"
function Kraken.apply_zou_he_north_2d!(f::B200Array, u_wall_x, Nx, Ny)
    c = _plain("apply_zou_he_north_2d!", f)
    _check("kb_apply_zou_he_north_2d", ccall((:kb_apply_zou_he_north_2d, LIB), Cint,
        (Ptr{Cvoid}, Cdouble, Cint, Cint, Cint, Ptr{Cvoid}),
        _arr("f", f, eltype(f), (Nx, Ny, 9)), u_wall_x, Nx, Ny, c, _stream()))
end

"compute_macroscopic_2d!(ρ, ux, uy, f; sync) -- src/kernels/macroscopic.jl:32"
function Kraken.compute_macroscopic_2d!(ρ, ux, uy, f::B200Array; sync=false)
    c = _plain("compute_macroscopic_2d!", f); T = _ftype(c)
    Nx, Ny = size(f, 1), size(f, 2); g = (Nx, Ny)
    _check("kb_compute_macroscopic_2d", ccall((:kb_compute_macroscopic_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cvoid}),
        _arr("ρ", ρ, T, g), _arr("ux", ux, T, g), _arr("uy", uy, T, g),
        _arr("f", f, eltype(f), (Nx, Ny, 9)), Nx, Ny, c, _stream()))
    _sync(sync)
end

"fused_bgk_step!(f_out, f_in, ρ, ux, uy, is_solid, Nx, Ny, ω) -- src/kernels/fused_bgk_2d.jl:67"
function Kraken.fused_bgk_step!(f_out::B200Array, f_in::B200Array, ρ, ux, uy, is_solid,
                                Nx, Ny, ω)
    c = _plain("fused_bgk_step!", f_in); T = eltype(f_in); g = (Nx, Ny); d = (Nx, Ny, 9)
    _check("kb_fused_bgk_step", ccall((:kb_fused_bgk_step, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint,
         Cdouble, Cint, Ptr{Cvoid}),
        _arr("f_out", f_out, T, d), _arr("f_in", f_in, T, d), _arr("ρ", ρ, T, g),
        _arr("ux", ux, T, g), _arr("uy", uy, T, g), _mask(is_solid, g), Nx, Ny, ω, c,
        _stream()))
end

"fused_trt_step!(f_out, f_in, ρ, ux, uy, is_solid, Nx, Ny, ν; Λ) -- src/kernels/fused_trt_2d.jl:145"
function Kraken.fused_trt_step!(f_out::B200Array, f_in::B200Array, ρ, ux, uy, is_solid,
                                Nx, Ny, ν; Λ::Real=3/16)
    c = _plain("fused_trt_step!", f_in); T = eltype(f_in); g = (Nx, Ny); d = (Nx, Ny, 9)
    _check("kb_fused_trt_step", ccall((:kb_fused_trt_step, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint,
         Cdouble, Cdouble, Cint, Ptr{Cvoid}),
        _arr("f_out", f_out, T, d), _arr("f_in", f_in, T, d), _arr("ρ", ρ, T, g),
        _arr("ux", ux, T, g), _arr("uy", uy, T, g), _mask(is_solid, g), Nx, Ny, ν, Λ, c,
        _stream()))
end

"collide_mrt_2d!(f, is_solid, ν; s_e, s_eps, s_q) -- src/kernels/collide_mrt_2d.jl:118"
function Kraken.collide_mrt_2d!(f::B200Array, is_solid, ν; s_e=1.4, s_eps=1.4, s_q=1.2)
    c = _plain("collide_mrt_2d!", f); Nx, Ny = size(f, 1), size(f, 2)
    _check("kb_collide_mrt_2d", ccall((:kb_collide_mrt_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint, Cdouble, Cdouble, Cdouble, Cdouble, Cint,
         Ptr{Cvoid}),
        _arr("f", f, eltype(f), (Nx, Ny, 9)), _mask(is_solid, (Nx, Ny)), Nx, Ny, ν, s_e, s_eps,
        s_q, c, _stream()))
end

"stream_fully_periodic_2d!(f_out, f_in, Nx, Ny) -- src/kernels/stream_periodic_2d.jl:112"
function Kraken.stream_fully_periodic_2d!(f_out::B200Array, f_in::B200Array, Nx, Ny)
    c = _plain("stream_fully_periodic_2d!", f_in); T = eltype(f_in); d = (Nx, Ny, 9)
    _check("kb_stream_fully_periodic_2d", ccall((:kb_stream_fully_periodic_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cvoid}),
        _arr("f_out", f_out, T, d), _arr("f_in", f_in, T, d), Nx, Ny, c, _stream()))
end

"stream_periodic_x_wall_y_2d!(f_out, f_in, Nx, Ny) -- src/kernels/stream_periodic_2d.jl:71"
function Kraken.stream_periodic_x_wall_y_2d!(f_out::B200Array, f_in::B200Array, Nx, Ny)
    c = _plain("stream_periodic_x_wall_y_2d!", f_in); T = eltype(f_in); d = (Nx, Ny, 9)
    _check("kb_stream_periodic_x_wall_y_2d", ccall((:kb_stream_periodic_x_wall_y_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cvoid}),
        _arr("f_out", f_out, T, d), _arr("f_in", f_in, T, d), Nx, Ny, c, _stream()))
end

"collide_guo_2d!(f, is_solid, ω, Fx, Fy) -- src/kernels/collide_guo_2d.jl:84"
function Kraken.collide_guo_2d!(f::B200Array, is_solid, ω, Fx, Fy)
    c = _plain("collide_guo_2d!", f); Nx, Ny = size(f, 1), size(f, 2)
    _check("kb_collide_guo_2d", ccall((:kb_collide_guo_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint, Cdouble, Cdouble, Cdouble, Cint, Ptr{Cvoid}),
        _arr("f", f, eltype(f), (Nx, Ny, 9)), _mask(is_solid, (Nx, Ny)), Nx, Ny, ω, Fx, Fy, c,
        _stream()))
end

"fused_natconv_step!(f_out, f_in, g_out, g_in, Temp, Nx, Ny, ω_f, ω_T, β_g, T_ref_buoy, T_hot, T_cold) -- src/kernels/fused_thermal_2d.jl:251"
function Kraken.fused_natconv_step!(f_out::B200Array, f_in::B200Array, g_out, g_in, Temp,
                                    Nx, Ny, ω_f, ω_T, β_g, T_ref_buoy, T_hot, T_cold)
    c = _plain("fused_natconv_step!", f_in); T = eltype(f_in); d = (Nx, Ny, 9)
    _check("kb_fused_natconv_step", ccall((:kb_fused_natconv_step, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cdouble,
         Cdouble, Cdouble, Cdouble, Cdouble, Cdouble, Cint, Ptr{Cvoid}),
        _arr("f_out", f_out, T, d), _arr("f_in", f_in, T, d), _arr("g_out", g_out, T, d),
        _arr("g_in", g_in, T, d), _arr("Temp", Temp, T, (Nx, Ny)), Nx, Ny, ω_f, ω_T, β_g,
        T_ref_buoy, T_hot, T_cold, c, _stream()))
end

"compute_temperature_2d!(Temp, g) -- src/kernels/thermal_2d.jl:133"
function Kraken.compute_temperature_2d!(Temp, g::B200Array)
    c = _plain("compute_temperature_2d!", g); T = eltype(g); Nx, Ny = size(g, 1), size(g, 2)
    _check("kb_compute_temperature_2d", ccall((:kb_compute_temperature_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cvoid}),
        _arr("Temp", Temp, T, (Nx, Ny)), _arr("g", g, T, (Nx, Ny, 9)), Nx, Ny, c, _stream()))
end

"collide_thermal_2d!(g, ux, uy, ω_T) -- src/kernels/thermal_2d.jl:76"
function Kraken.collide_thermal_2d!(g::B200Array, ux, uy, ω_T)
    c = _plain("collide_thermal_2d!", g); T = eltype(g); Nx, Ny = size(g, 1), size(g, 2)
    _check("kb_collide_thermal_2d", ccall((:kb_collide_thermal_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cdouble, Cint, Ptr{Cvoid}),
        _arr("g", g, T, (Nx, Ny, 9)), _arr("ux", ux, T, (Nx, Ny)), _arr("uy", uy, T, (Nx, Ny)),
        Nx, Ny, ω_T, c, _stream()))
end

# One face of half-way anti-bounce-back: 0 west, 1 east, 2 south, 3 north.
function _fixed_temp_face_2d!(g::B200Array, face, T_wall)
    c = _plain("apply_fixed_temp_*_2d!", g); Nx, Ny = size(g, 1), size(g, 2)
    _check("kb_apply_fixed_temp_face_2d", ccall((:kb_apply_fixed_temp_face_2d, LIB), Cint,
        (Ptr{Cvoid}, Cint, Cint, Cint, Cdouble, Cdouble, Cdouble, Cint, Cint, Cint, Ptr{Cvoid}),
        _arr("g", g, eltype(g), (Nx, Ny, 9)), Nx, Ny, face, T_wall, T_wall, T_wall, 0, 0, c,
        _stream()))
end

"apply_fixed_temp_west_2d!(g, T_wall, Ny) -- src/kernels/thermal_2d.jl:311"
Kraken.apply_fixed_temp_west_2d!(g::B200Array, T_wall, Ny) = _fixed_temp_face_2d!(g, 0, T_wall)
"apply_fixed_temp_east_2d!(g, T_wall, Nx, Ny) -- src/kernels/thermal_2d.jl:340"
Kraken.apply_fixed_temp_east_2d!(g::B200Array, T_wall, Nx, Ny) = _fixed_temp_face_2d!(g, 1, T_wall)
"apply_fixed_temp_south_2d!(g, T_wall, Nx) -- src/kernels/thermal_2d.jl:219"
Kraken.apply_fixed_temp_south_2d!(g::B200Array, T_wall, Nx) = _fixed_temp_face_2d!(g, 2, T_wall)
"apply_fixed_temp_north_2d!(g, T_wall, Nx, Ny) -- src/kernels/thermal_2d.jl:248"
Kraken.apply_fixed_temp_north_2d!(g::B200Array, T_wall, Nx, Ny) = _fixed_temp_face_2d!(g, 3, T_wall)

function _face_temps(temps)
    mask = UInt32(0)
    Tf = zeros(Float64, length(temps))
    for (n, t) in enumerate(temps)
        t === nothing && continue
        mask |= UInt32(1) << (n - 1)
        Tf[n] = Float64(t)
    end
    return mask, Tf
end

"apply_fixed_temp_2d!(g, Nx, Ny; west, east, south, north) -- src/kernels/thermal_2d.jl:413"
function Kraken.apply_fixed_temp_2d!(g::B200Array, Nx, Ny; west=nothing, east=nothing,
                                     south=nothing, north=nothing)
    c = _plain("apply_fixed_temp_2d!", g)
    mask, Tf = _face_temps((west, east, south, north))
    _check("kb_apply_fixed_temp_2d", ccall((:kb_apply_fixed_temp_2d, LIB), Cint,
        (Ptr{Cvoid}, Cint, Cint, Cuint, Ptr{Cdouble}, Cint, Ptr{Cvoid}),
        _arr("g", g, eltype(g), (Nx, Ny, 9)), Nx, Ny, mask, Tf, c, _stream()))
end

"collide_boussinesq_2d!(f, Temp, is_solid, ω, β_g, T_ref) -- src/kernels/thermal_2d.jl:573"
function Kraken.collide_boussinesq_2d!(f::B200Array, Temp, is_solid, ω, β_g, T_ref)
    c = _plain("collide_boussinesq_2d!", f); T = eltype(f); Nx, Ny = size(f, 1), size(f, 2)
    _check("kb_collide_boussinesq_2d", ccall((:kb_collide_boussinesq_2d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint, Cdouble, Cdouble, Cdouble, Cint,
         Ptr{Cvoid}),
        _arr("f", f, T, (Nx, Ny, 9)), _arr("Temp", Temp, T, (Nx, Ny)), _mask(is_solid, (Nx, Ny)),
        Nx, Ny, ω, β_g, T_ref, c, _stream()))
end

"fused_trt_libb_v2_step!(f_out, f_in, ρ, ux, uy, is_solid, q_wall, uw_link_x, uw_link_y, Nx, Ny, ν; Λ) -- src/kernels/li_bb_2d_v2.jl:104"
function Kraken.fused_trt_libb_v2_step!(f_out::B200Array, f_in::B200Array, ρ, ux, uy, is_solid,
                                        q_wall, uw_link_x, uw_link_y, Nx, Ny, ν; Λ::Real=3/16)
    c = _plain("fused_trt_libb_v2_step!", f_in); T = eltype(f_in); g = (Nx, Ny); d = (Nx, Ny, 9)
    _check("kb_fused_trt_libb_step", ccall((:kb_fused_trt_libb_step, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8}, Ptr{Cvoid},
         Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cdouble, Cdouble, Cint, Ptr{Cvoid}),
        _arr("f_out", f_out, T, d), _arr("f_in", f_in, T, d), _arr("ρ", ρ, T, g),
        _arr("ux", ux, T, g), _arr("uy", uy, T, g), _mask(is_solid, g),
        _arr("q_wall", q_wall, T, d), _arr("uw_link_x", uw_link_x, T, d),
        _arr("uw_link_y", uw_link_y, T, d), Nx, Ny, ν, Λ, c, _stream()))
end

# --------------------------------------------------------------- D3Q19

"stream_3d!(f_out, f_in, Nx, Ny, Nz) -- src/kernels/collide_stream_3d.jl:119"
function Kraken.stream_3d!(f_out::B200Array, f_in::B200Array, Nx, Ny, Nz)
    c = _plain("stream_3d!", f_in); T = eltype(f_in); d = (Nx, Ny, Nz, 19)
    _check("kb_stream_3d", ccall((:kb_stream_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Cint, Ptr{Cvoid}),
        _arr("f_out", f_out, T, d), _arr("f_in", f_in, T, d), Nx, Ny, Nz, c, _stream()))
end

"collide_3d!(f, is_solid, ω) -- src/kernels/collide_stream_3d.jl:137"
function Kraken.collide_3d!(f::B200Array, is_solid, ω)
    c = _plain("collide_3d!", f); Nx, Ny, Nz = size(f, 1), size(f, 2), size(f, 3)
    _check("kb_collide_3d", ccall((:kb_collide_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint, Cint, Cdouble, Cint, Ptr{Cvoid}),
        _arr("f", f, eltype(f), (Nx, Ny, Nz, 19)), _mask(is_solid, (Nx, Ny, Nz)), Nx, Ny, Nz, ω,
        c, _stream()))
end

"apply_zou_he_top_3d!(f, u_wall_x, Nx, Ny, Nz) -- src/kernels/boundary_3d.jl:326"
function Kraken.apply_zou_he_top_3d!(f::B200Array, u_wall_x, Nx, Ny, Nz)
    c = _plain("apply_zou_he_top_3d!", f)
    _check("kb_apply_zou_he_top_3d", ccall((:kb_apply_zou_he_top_3d, LIB), Cint,
        (Ptr{Cvoid}, Cdouble, Cint, Cint, Cint, Cint, Ptr{Cvoid}),
        _arr("f", f, eltype(f), (Nx, Ny, Nz, 19)), u_wall_x, Nx, Ny, Nz, c, _stream()))
end

"compute_macroscopic_3d!(ρ, ux, uy, uz, f) -- src/kernels/macroscopic.jl:75"
function Kraken.compute_macroscopic_3d!(ρ, ux, uy, uz, f::B200Array)
    c = _plain("compute_macroscopic_3d!", f); T = _ftype(c)
    Nx, Ny, Nz = size(f, 1), size(f, 2), size(f, 3); g = (Nx, Ny, Nz)
    _check("kb_compute_macroscopic_3d", ccall((:kb_compute_macroscopic_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Cint,
         Ptr{Cvoid}),
        _arr("ρ", ρ, T, g), _arr("ux", ux, T, g), _arr("uy", uy, T, g), _arr("uz", uz, T, g),
        _arr("f", f, eltype(f), (Nx, Ny, Nz, 19)), Nx, Ny, Nz, c, _stream()))
end

"collide_thermal_3d!(g, ux, uy, uz, ω_T) -- src/kernels/thermal_3d.jl:119"
function Kraken.collide_thermal_3d!(g::B200Array, ux, uy, uz, ω_T)
    c = _plain("collide_thermal_3d!", g); T = eltype(g)
    Nx, Ny, Nz = size(g, 1), size(g, 2), size(g, 3); s = (Nx, Ny, Nz)
    _check("kb_collide_thermal_3d", ccall((:kb_collide_thermal_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Cdouble, Cint,
         Ptr{Cvoid}),
        _arr("g", g, T, (Nx, Ny, Nz, 19)), _arr("ux", ux, T, s), _arr("uy", uy, T, s),
        _arr("uz", uz, T, s), Nx, Ny, Nz, ω_T, c, _stream()))
end

"compute_temperature_3d!(Temp, g) -- src/kernels/thermal_3d.jl:150"
function Kraken.compute_temperature_3d!(Temp, g::B200Array)
    c = _plain("compute_temperature_3d!", g); T = eltype(g)
    Nx, Ny, Nz = size(g, 1), size(g, 2), size(g, 3)
    _check("kb_compute_temperature_3d", ccall((:kb_compute_temperature_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Cint, Ptr{Cvoid}),
        _arr("Temp", Temp, T, (Nx, Ny, Nz)), _arr("g", g, T, (Nx, Ny, Nz, 19)), Nx, Ny, Nz, c,
        _stream()))
end

"apply_fixed_temp_3d!(g, Nx, Ny, Nz; west, east, south, north, bottom, top) -- src/kernels/thermal_3d.jl:547"
function Kraken.apply_fixed_temp_3d!(g::B200Array, Nx, Ny, Nz; west=nothing, east=nothing,
                                     south=nothing, north=nothing, bottom=nothing, top=nothing)
    c = _plain("apply_fixed_temp_3d!", g)
    mask, Tf = _face_temps((west, east, south, north, bottom, top))
    _check("kb_apply_fixed_temp_3d", ccall((:kb_apply_fixed_temp_3d, LIB), Cint,
        (Ptr{Cvoid}, Cint, Cint, Cint, Cuint, Ptr{Cdouble}, Cint, Ptr{Cvoid}),
        _arr("g", g, eltype(g), (Nx, Ny, Nz, 19)), Nx, Ny, Nz, mask, Tf, c, _stream()))
end

"collide_boussinesq_3d!(f, Temp, is_solid, ω, β_g, T_ref) -- src/kernels/thermal_3d.jl:727"
function Kraken.collide_boussinesq_3d!(f::B200Array, Temp, is_solid, ω, β_g, T_ref)
    c = _plain("collide_boussinesq_3d!", f); T = eltype(f)
    Nx, Ny, Nz = size(f, 1), size(f, 2), size(f, 3)
    _check("kb_collide_boussinesq_3d", ccall((:kb_collide_boussinesq_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint, Cint, Cdouble, Cdouble, Cdouble, Cint,
         Ptr{Cvoid}),
        _arr("f", f, T, (Nx, Ny, Nz, 19)), _arr("Temp", Temp, T, (Nx, Ny, Nz)),
        _mask(is_solid, (Nx, Ny, Nz)), Nx, Ny, Nz, ω, β_g, T_ref, c, _stream()))
end

"fused_trt_libb_v2_step_3d!(f_out, f_in, ρ, ux, uy, uz, is_solid, q_wall, uw_link_x, uw_link_y, uw_link_z, Nx, Ny, Nz, ν; Λ) -- src/kernels/li_bb_3d_v2.jl:31"
function Kraken.fused_trt_libb_v2_step_3d!(f_out::B200Array, f_in::B200Array, ρ, ux, uy, uz,
                                           is_solid, q_wall, uw_link_x, uw_link_y, uw_link_z,
                                           Nx, Ny, Nz, ν; Λ::Real=3/16)
    c = _plain("fused_trt_libb_v2_step_3d!", f_in); T = eltype(f_in)
    g = (Nx, Ny, Nz); d = (Nx, Ny, Nz, 19)
    _check("kb_fused_trt_libb_step_3d", ccall((:kb_fused_trt_libb_step_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8},
         Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Cint, Cint, Cdouble, Cdouble,
         Cint, Cint, Ptr{Cvoid}),
        _arr("f_out", f_out, T, d), _arr("f_in", f_in, T, d), _arr("ρ", ρ, T, g),
        _arr("ux", ux, T, g), _arr("uy", uy, T, g), _arr("uz", uz, T, g), _mask(is_solid, g),
        _arr("q_wall", q_wall, T, d), _arr("uw_link_x", uw_link_x, T, d),
        _arr("uw_link_y", uw_link_y, T, d), _arr("uw_link_z", uw_link_z, T, d), Nx, Ny, Nz, ν, Λ,
        0, c, _stream()))
end

# ------------------------------------------------ B200-only entry points

_is_bf16(::Type{T}) where {T} = sizeof(T) == 2 && nameof(T) === :BFloat16

# storage keyword -> (kb_dtype, check of the population eltype, field eltype)
function _storage(name, storage::Symbol, ::Type{E}) where {E}
    ok, code = if storage === :plain
        (E === Float64 || E === Float32), (E === Float64 ? KB_F64 : KB_F32)
    elseif storage === :f32dev
        E === Float32, KB_F32_DEV
    elseif storage === :f16dev || storage === :f16dev_sr
        E === Float16, (storage === :f16dev ? KB_F16_DEV : KB_F16_DEV_SR)
    elseif storage === :bf16dev || storage === :bf16dev_sr
        _is_bf16(E), (storage === :bf16dev ? KB_BF16_DEV : KB_BF16_DEV_SR)
    else
        throw(ArgumentError("$name: unknown storage :$storage (:plain, :f32dev, :f16dev, " *
                            ":f16dev_sr, :bf16dev, :bf16dev_sr)"))
    end
    ok || throw(ArgumentError("$name: storage :$storage does not hold $E populations"))
    return code, (code == KB_F64 ? Float64 : Float32)
end

function _moments_all_or_none(name, ρ, ux, uy, uz)
    n = count(x -> x === nothing, (ρ, ux, uy, uz))
    n == 0 || n == 4 || throw(ArgumentError("$name: ρ, ux, uy, uz must be all set or all nothing"))
    return nothing
end

"""
    fused_trt_step_3d!(f_out, f_in, ρ, ux, uy, uz, is_solid, Nx, Ny, Nz, ν;
                       Λ=3/16, periodic=(false, false, false), storage=:plain)

Fused D3Q19 TRT step (pull with half-way bounce-back, solid nodes at rest,
TRT collision, moments): the step of `fused_trt_libb_v2_step_3d!`
(src/kernels/li_bb_3d_v2.jl:31) without cut links, with a periodic wrap per
axis.  `storage` picks the population format: `:plain` (Float64/Float32
populations, fields of the same type), `:f32dev` (Float32 f - w_q),
`:f16dev`, `:bf16dev` (16-bit f - w_q, collision in Float32) and their
stochastic-rounding forms `:f16dev_sr`, `:bf16dev_sr`; deviation storages
take Float32 fields.  `ρ`, `ux`, `uy`, `uz` may all be `nothing` (no moment
writes); `is_solid` may be `nothing`.
"""
function fused_trt_step_3d!(f_out::B200Array, f_in::B200Array, ρ, ux, uy, uz, is_solid,
                            Nx, Ny, Nz, ν; Λ::Real=3/16, periodic=(false, false, false),
                            storage::Symbol=:plain)
    code, F = _storage("fused_trt_step_3d!", storage, eltype(f_in))
    E = eltype(f_in); g = (Nx, Ny, Nz); d = (Nx, Ny, Nz, 19)
    _moments_all_or_none("fused_trt_step_3d!", ρ, ux, uy, uz)
    per = Int(periodic[1]) | (Int(periodic[2]) << 1) | (Int(periodic[3]) << 2)
    _check("kb_fused_trt_step_3d", ccall((:kb_fused_trt_step_3d, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8},
         Cint, Cint, Cint, Cdouble, Cdouble, Cint, Cint, Ptr{Cvoid}),
        _arr("f_out", f_out, E, d), _arr("f_in", f_in, E, d), _opt("ρ", ρ, F, g),
        _opt("ux", ux, F, g), _opt("uy", uy, F, g), _opt("uz", uz, F, g), _mask(is_solid, g),
        Nx, Ny, Nz, ν, Λ, per, code, _stream()))
end

"""
    fused_trt_step_3d_zrange!(f_out, f_in, ρ, ux, uy, uz, is_solid, Nx, Ny, Nz_alloc,
                              k_begin, k_end, ν; Λ=3/16, periodic_xy=(false, false),
                              storage=:plain)

The step of `fused_trt_step_3d!` over the z-planes `k_begin .. k_end-1` (0-based,
as in the C header) of a z-slab allocation of `Nz_alloc` planes whose first and
last planes are halo planes, read as they are.  Every array spans the whole
allocation; only the range is written.  No reference counterpart (the reference
steps whole arrays).
"""
function fused_trt_step_3d_zrange!(f_out::B200Array, f_in::B200Array, ρ, ux, uy, uz, is_solid,
                                   Nx, Ny, Nz_alloc, k_begin, k_end, ν; Λ::Real=3/16,
                                   periodic_xy=(false, false), storage::Symbol=:plain)
    code, F = _storage("fused_trt_step_3d_zrange!", storage, eltype(f_in))
    E = eltype(f_in); g = (Nx, Ny, Nz_alloc); d = (Nx, Ny, Nz_alloc, 19)
    _moments_all_or_none("fused_trt_step_3d_zrange!", ρ, ux, uy, uz)
    per = Int(periodic_xy[1]) | (Int(periodic_xy[2]) << 1)
    _check("kb_fused_trt_step_3d_zrange", ccall((:kb_fused_trt_step_3d_zrange, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8},
         Cint, Cint, Cint, Cint, Cint, Cdouble, Cdouble, Cint, Cint, Ptr{Cvoid}),
        _arr("f_out", f_out, E, d), _arr("f_in", f_in, E, d), _opt("ρ", ρ, F, g),
        _opt("ux", ux, F, g), _opt("uy", uy, F, g), _opt("uz", uz, F, g), _mask(is_solid, g),
        Nx, Ny, Nz_alloc, k_begin, k_end, ν, Λ, per, code, _stream()))
end

"Ghost planes of one z-slab on a periodic z axis from its own end planes (one launch)."
function slab_fill_ghosts_3d!(f::B200Array, lo::Bool, hi::Bool; storage::Symbol=:plain)
    code, _ = _storage("slab_fill_ghosts_3d!", storage, eltype(f))
    Nx, Ny, Nz_alloc = size(f, 1), size(f, 2), size(f, 3)
    _check("kb_slab_fill_ghosts_3d", ccall((:kb_slab_fill_ghosts_3d, LIB), Cint,
        (Ptr{Cvoid}, Cint, Cint, Cint, Cint, Cint, Cint, Ptr{Cvoid}),
        _arr("f", f, eltype(f), (Nx, Ny, Nz_alloc, 19)), Nx, Ny, Nz_alloc, Int(lo), Int(hi),
        code, _stream()))
end

end # module
