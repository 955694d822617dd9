// kb_common.cuh -- shared definitions of the B200 stream-collide library.
//
// Layout (Julia column-major, 0-based):
//   D2Q9   f[i + Nx*(j + Ny*q)]
//   D3Q19  f[i + Nx*(j + Ny*(k + Nz*q))]
// Populations q are 0-based (Kraken.jl's q minus one).
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/krakenb200.h"

namespace kb {

// Error reporting (kb_error.cu).
int set_error(int code, const char *fmt, ...);
int check_launch(const char *what);
void clear_error();

// ---------------------------------------------------------------- lattice --
// D2Q9 (src/lattice/d2q9.jl:19-29) and D3Q19 (src/lattice/d3q19.jl:13-47).
__host__ __device__ constexpr double w9(int q) {
    return q == 0 ? 4.0 / 9.0 : (q < 5 ? 1.0 / 9.0 : 1.0 / 36.0);
}
__host__ __device__ constexpr double w19(int q) {
    return q == 0 ? 1.0 / 3.0 : (q < 7 ? 1.0 / 18.0 : 1.0 / 36.0);
}
__host__ __device__ constexpr int cx19(int q) {
    constexpr int c[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    return c[q];
}
__host__ __device__ constexpr int cy19(int q) {
    constexpr int c[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
    return c[q];
}
__host__ __device__ constexpr int cz19(int q) {
    constexpr int c[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
    return c[q];
}
__host__ __device__ constexpr int opp19(int q) {
    constexpr int o[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
    return o[q];
}

// ---------------------------------------------------------------- storage --
// Storage codecs.  Plain storages (double, float) hold f.  Deviation
// storages hold d = f - w_q and are decoded to float.
template <typename R> struct Dev;
template <> struct Dev<float> {
    static __device__ __forceinline__ float ld(float r) { return r; }
    static __device__ __forceinline__ float st(float d) { return d; }
};
template <> struct Dev<__half> {
    static __device__ __forceinline__ float ld(__half r) { return __half2float(r); }
    static __device__ __forceinline__ __half st(float d) { return __float2half_rn(d); }
};
template <> struct Dev<__nv_bfloat16> {
    static __device__ __forceinline__ float ld(__nv_bfloat16 r) { return __bfloat162float(r); }
    static __device__ __forceinline__ __nv_bfloat16 st(float d) { return __float2bfloat16_rn(d); }
};

// Scalar / packed-pair (float2, sm_100 FADD2/FMUL2/FFMA2) arithmetic for the
// collisions written once for one node (float) or two nodes (float2).
__device__ __forceinline__ float vadd(float a, float b) { return a + b; }
__device__ __forceinline__ float vsub(float a, float b) { return a - b; }
__device__ __forceinline__ float vmul(float a, float b) { return a * b; }
__device__ __forceinline__ float vfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ float vneg(float a) { return -a; }
__device__ __forceinline__ float vsplat(float a, float) { return a; }
__device__ __forceinline__ float vrcp(float a) { return __frcp_rn(a); }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 vsub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 vmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 vneg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 vsplat(float a, float2) { return make_float2(a, a); }
__device__ __forceinline__ float2 vrcp(float2 a) { return make_float2(__frcp_rn(a.x), __frcp_rn(a.y)); }
// Two FP32 lanes (adjacent nodes) with the operators of the reference
// arithmetic: packed round-to-nearest adds and multiplies (never contracted)
// and a per-lane division, so a helper written for T evaluates, with
// T = Lanes2, the same expression tree for each node at half the arithmetic
// instructions.  Measured against the one-node kernels the results agree to
// 3 ulp; about 1 % of the updated populations differ in the last bits.
struct Lanes2 {
    float2 v;
    __device__ __forceinline__ Lanes2() {}
    __device__ __forceinline__ Lanes2(double d) { const float x = (float)d; v = make_float2(x, x); }
    __device__ __forceinline__ static Lanes2 of(float2 a) { Lanes2 r; r.v = a; return r; }
    __device__ __forceinline__ Lanes2 operator-() const { return of(make_float2(-v.x, -v.y)); }
};
__device__ __forceinline__ Lanes2 operator+(Lanes2 a, Lanes2 b) { return Lanes2::of(vadd(a.v, b.v)); }
__device__ __forceinline__ Lanes2 operator-(Lanes2 a, Lanes2 b) { return Lanes2::of(vsub(a.v, b.v)); }
__device__ __forceinline__ Lanes2 operator*(Lanes2 a, Lanes2 b) { return Lanes2::of(vmul(a.v, b.v)); }
__device__ __forceinline__ Lanes2 operator/(Lanes2 a, Lanes2 b) {
    return Lanes2::of(make_float2(a.v.x / b.v.x, a.v.y / b.v.y));
}

// 1/a from the hardware approximation (PTX rcp.approx.ftz.f32, within about
// one unit in the last place).  The deviation-storage collisions divide by
// rho = 1 + drho, which is never near zero or subnormal; the IEEE-rounded
// reciprocal (vrcp) would add a refinement and a range check per node to a
// kernel that is instruction bound at 16-bit storage.
__device__ __forceinline__ float vrcp_fast(float a) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}
__device__ __forceinline__ float2 vrcp_fast(float2 a) { return make_float2(vrcp_fast(a.x), vrcp_fast(a.y)); }

// ------------------------------------------------------ stochastic rounding --
// 32-bit integer hash (lowbias32, C. Wellons) for the random bits of the
// stochastic-rounding stores.
__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// Two floats -> one packed 16-bit pair (lo in the low half, the lower
// address), rounded stochastically by sm_100a's cvt.rs with 32 random bits
// (bits 0-12 / 0-15 drive lo, bits 16-28 / 16-31 hi, for f16 / bf16).
template <typename R> struct SRPack;
template <> struct SRPack<__half> {
    static __device__ __forceinline__ uint32_t pack(float lo, float hi, uint32_t r) {
        uint32_t d;
        asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(r));
        return d;
    }
};
template <> struct SRPack<__nv_bfloat16> {
    static __device__ __forceinline__ uint32_t pack(float lo, float hi, uint32_t r) {
        uint32_t d;
        asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(r));
        return d;
    }
};
template <> struct SRPack<float> {  // never used with SR: FP32 storage rounds to nearest
    static __device__ __forceinline__ uint32_t pack(float, float, uint32_t) { return 0u; }
};

inline size_t dtype_bytes(int dtype) {
    switch (dtype) {
        case KB_F64: return 8;
        case KB_F32: return 4;
        case KB_F32_DEV: return 4;
        case KB_F16_DEV: return 2;
        case KB_BF16_DEV: return 2;
        case KB_F16_DEV_SR: return 2;
        case KB_BF16_DEV_SR: return 2;
        default: return 0;
    }
}

// Memory format of a storage: the stochastic-rounding storages hold the same
// bits as their round-to-nearest counterparts.
__host__ __device__ inline int storage_format(int dtype) {
    return dtype == KB_F16_DEV_SR ? KB_F16_DEV : (dtype == KB_BF16_DEV_SR ? KB_BF16_DEV : dtype);
}

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Number of SMs of the current device (cached per device).
int sm_count();

}  // namespace kb

#define KB_REQUIRE(cond, ...)                                        \
    do {                                                             \
        if (!(cond)) return ::kb::set_error(KB_ERR_ARG, __VA_ARGS__); \
    } while (0)
