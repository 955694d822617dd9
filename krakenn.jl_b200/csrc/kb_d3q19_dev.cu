// kb_d3q19_dev.cu -- fused D3Q19 TRT step on deviation storage.
//
// Populations are stored as d_q = f_q - w_q (FP32, FP16 or BF16) and the
// collision runs in FP32 on the deviations directly, so no FP32 rounding of
// the O(w_q) background enters the update:
//   drho = sum_q d_q,  rho = 1 + drho,  j = sum_q c_q d_q,  u = j / rho
//   deq_q = w_q (drho + rho (3 cu + 4.5 cu^2 - 1.5 u^2))
//   TRT on each opposite pair (q, qb): with n = d - deq,
//   d*_q  = d_q  - s+ (n_q + n_qb)/2 - s- (n_q - n_qb)/2
//   d*_qb = d_qb - s+ (n_q + n_qb)/2 + s- (n_q - n_qb)/2
// which equals the reference's CollideTRTDirect_3D
// (src/kernels/dsl/bricks_3d.jl:179-229): f*_q = f_q - a n_q - b n_qb with
// a = (s+ + s-)/2, b = (s+ - s-)/2.  The pull and the solid rule are the same
// as the reference step (PullHalfwayBB_3D, SolidInert_3D: a solid node is
// reset to rest equilibrium, i.e. d = 0).
//
// Compiled with FMA contraction on: this is the precision tier, checked by
// its max/L2 error against the FP64 run, not bit for bit.
#include "kb_d3q19.cuh"

namespace kb {
namespace d3 {

template <typename R>
struct DevLoad {
    __device__ __forceinline__ float operator()(R r) const { return Dev<R>::ld(r); }
};

// ---------------------------------------------------------------------------
// Stochastic rounding of the 16-bit storages (KB_F16_DEV_SR, KB_BF16_DEV_SR).
// Round-to-nearest storage of slowly varying deviations is biased: an update
// smaller than half a unit in the last place is lost every step.  sm_100a's
// cvt.rs.{f16x2,bf16x2}.f32 rounds up with probability equal to the dropped
// fraction, given 32 random bits per pair, so the rounding error has zero
// mean.  The bits come from an integer hash (lowbias32, C. Wellons) of the
// thread index, the population and a launch counter in device memory that a
// one-thread kernel advances after every such launch (so CUDA-graph replays
// draw fresh bits and a run is reproducible on one stream).
__device__ unsigned int g_sr_epoch = 0;

__global__ void sr_advance_k() { g_sr_epoch += 1u; }

// Per-thread key for this launch; the word for population q is hash32(key + q * golden).
__device__ __forceinline__ uint32_t sr_key() {
    const uint32_t tid = (blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)) * blockDim.x +
                         threadIdx.x;
    const uint32_t e = *(volatile const unsigned int *)&g_sr_epoch;
    return hash32(tid ^ hash32(e + 0x632BE5ABu));
}
__device__ __forceinline__ uint32_t sr_bits(uint32_t key, int q) { return hash32(key + (uint32_t)q * 0x9E3779B9u); }

// Opposite pairs (q, qb) of D3Q19; c_qb = -c_q.  Indexed only with
// compile-time constants (fully unrolled loops), so d[] stays in registers.
__device__ constexpr int kPairQ[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16};
__device__ constexpr int kPairQb[9] = {2, 4, 6, 10, 9, 14, 13, 18, 17};

// TRT collision of D3Q19 deviations d[19] -> o[19] (V = float for one node,
// float2 for two).  With s_m = d_q + d_qb and t_m = d_q - d_qb of the nine
// opposite pairs (q, qb), c_qb = -c_q:
//   drho = d_0 + sum s_m,  j = sum c_q t_m,  rho = 1 + drho,  u = j / rho
//   even mode: n+ = s_m/2 - w (drho + rho (4.5 cu^2 - 1.5 u^2))
//   odd mode:  n- = t_m/2 - 3 w rho cu
//   o_q = d_q - s+ n+ - s- n-,   o_qb = d_qb - s+ n+ + s- n-
// which is CollideTRTDirect_3D (src/kernels/dsl/bricks_3d.jl:179-229)
// written on deviations.  Regrouped on s and t only (d_q = (s + t)/2):
//   X = (1 - s+)/2 s_m + s+ w (base + 4.5 rho cu^2),  base = drho - 1.5 rho u^2
//   Y = (1 - s-)/2 t_m + 3 s- w rho cu
//   o_q = X + Y,  o_qb = X - Y
template <typename V>
__device__ __forceinline__ void trt_dev_collide(const V *d, V *o, V &rho, V &ux, V &uy, V &uz,
                                                float sp, float sm) {
    const V z = vsplat(0.f, d[0]);
    V sv[9], tv[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) {
        sv[m] = vadd(d[kPairQ[m]], d[kPairQb[m]]);
        tv[m] = vsub(d[kPairQ[m]], d[kPairQb[m]]);
    }
    // pair order: (1,2) x, (3,4) y, (5,6) z, (7,10) +x+y, (8,9) -x+y,
    // (11,14) +x+z, (12,13) -x+z, (15,18) +y+z, (16,17) -y+z
    const V drho = vadd(vadd(vadd(d[0], sv[0]), vadd(sv[1], sv[2])),
                        vadd(vadd(vadd(sv[3], sv[4]), vadd(sv[5], sv[6])), vadd(sv[7], sv[8])));
    const V jx = vadd(vsub(vadd(tv[0], tv[3]), tv[4]), vsub(tv[5], tv[6]));
    const V jy = vadd(vadd(vadd(tv[1], tv[3]), tv[4]), vsub(tv[7], tv[8]));
    const V jz = vadd(vadd(vadd(tv[2], tv[5]), tv[6]), vadd(tv[7], tv[8]));
    rho = vadd(vsplat(1.f, z), drho);
    const V inv = vrcp(rho);
    ux = vmul(jx, inv);
    uy = vmul(jy, inv);
    uz = vmul(jz, inv);
    const V usq15 = vmul(vsplat(1.5f, z), vfma(ux, ux, vfma(uy, uy, vmul(uz, uz))));
    const V base = vsub(drho, vmul(rho, usq15));
    // rest population (even mode only): o_0 = (1 - s+) d_0 + s+ w_0 base
    o[0] = vfma(vsplat(1.0f - sp, z), d[0], vmul(vsplat(sp * float(1.0 / 3.0), z), base));
    const V ha = vsplat(0.5f * (1.0f - sp), z), hb = vsplat(0.5f * (1.0f - sm), z);
#pragma unroll
    for (int cls = 0; cls < 2; ++cls) {
        const float w = cls == 0 ? float(1.0 / 18.0) : float(1.0 / 36.0);
        const V A = vmul(vsplat(sp * w, z), base);          // s+ w base
        const V B = vmul(vsplat(4.5f * sp * w, z), rho);    // 4.5 s+ w rho
        const V C = vmul(vsplat(3.0f * sm * w, z), rho);    // 3 s- w rho
#pragma unroll
        for (int m = (cls == 0 ? 0 : 3); m < (cls == 0 ? 3 : 9); ++m) {
            const int q = kPairQ[m], qb = kPairQb[m];
            V cu = z;
            if (cx19(q) == 1) cu = vadd(cu, ux); else if (cx19(q) == -1) cu = vsub(cu, ux);
            if (cy19(q) == 1) cu = vadd(cu, uy); else if (cy19(q) == -1) cu = vsub(cu, uy);
            if (cz19(q) == 1) cu = vadd(cu, uz); else if (cz19(q) == -1) cu = vsub(cu, uz);
            const V X = vfma(ha, sv[m], vfma(vmul(B, cu), cu, A));
            const V Y = vfma(hb, tv[m], vmul(C, cu));
            o[q] = vadd(X, Y);
            o[qb] = vsub(X, Y);
        }
    }
}

template <typename R, bool MOM, bool SOLID, typename I, bool SR>
__global__ void __launch_bounds__(BX) trt_dev_k(R *__restrict__ fo, const R *__restrict__ fi,
                                                 float *__restrict__ rho_o, float *__restrict__ ux_o,
                                                 float *__restrict__ uy_o, float *__restrict__ uz_o,
                                                 const uint8_t *__restrict__ solid, Grid3 g,
                                                 float sp, float sm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= g.Nx) return;
    const size_t c = (size_t)i + (size_t)g.Nx * ((size_t)j + (size_t)g.Ny * k);
    const I P = (I)g.plane;
    R *__restrict__ o0 = fo + c;
    if (SOLID && solid[c]) {
#pragma unroll
        for (int q = 0; q < 19; ++q) o0[q * P] = Dev<R>::st(0.0f);
        if (MOM) { rho_o[c] = 1.0f; ux_o[c] = 0.0f; uy_o[c] = 0.0f; uz_o[c] = 0.0f; }
        return;
    }
    float d[19];
    pull19_at(fi + c, P, pull_geometry<I>(g, i, j, k), d, DevLoad<R>());

    float o[19], rho, ux, uy, uz;
    trt_dev_collide(d, o, rho, ux, uy, uz, sp, sm);
    if (SR) {
        const uint32_t key = sr_key();
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const uint32_t v = SRPack<R>::pack(o[q], 0.f, sr_bits(key, q));
            reinterpret_cast<unsigned short *>(o0)[q * P] = (unsigned short)(v & 0xFFFFu);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 19; ++q) o0[q * P] = Dev<R>::st(o[q]);
    }
    if (MOM) { rho_o[c] = rho; ux_o[c] = ux; uy_o[c] = uy; uz_o[c] = uz; }
}

// One node per thread with the compact cut-link table (kb_libb_links): the
// class byte replaces the solid mask; nodes with cut links apply the
// Bouzidi pre-phase on the deviations.  _libb_branch is affine with weights
// summing to one and maps a population to its opposite, which has the same
// lattice weight, so it applies to d = f - w unchanged.
template <typename R, bool MOM, typename I, bool SR>
__global__ void __launch_bounds__(BX) trt_dev_links_k(R *__restrict__ fo, const R *__restrict__ fi,
                                                       float *__restrict__ rho_o,
                                                       float *__restrict__ ux_o,
                                                       float *__restrict__ uy_o,
                                                       float *__restrict__ uz_o, LinkTable3 L,
                                                       Grid3 g, float sp, float sm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= g.Nx) return;
    const size_t c = (size_t)i + (size_t)g.Nx * ((size_t)j + (size_t)g.Ny * k);
    const I P = (I)g.plane;
    R *__restrict__ o0 = fo + c;
    const uint8_t cl = L.cls[c];
    if (cl == 1) {
#pragma unroll
        for (int q = 0; q < 19; ++q) o0[q * P] = Dev<R>::st(0.0f);
        if (MOM) { rho_o[c] = 1.0f; ux_o[c] = 0.0f; uy_o[c] = 0.0f; uz_o[c] = 0.0f; }
        return;
    }
    float d[19];
    pull19_at(fi + c, P, pull_geometry<I>(g, i, j, k), d, DevLoad<R>());
    if (cl == 2) libb_prephase_3d(fi + c, P, link_record<float>(L, L.rec[c]), d, DevLoad<R>());
    float o[19], rho, ux, uy, uz;
    trt_dev_collide(d, o, rho, ux, uy, uz, sp, sm);
    if (SR) {
        const uint32_t key = sr_key();
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const uint32_t v = SRPack<R>::pack(o[q], 0.f, sr_bits(key, q));
            reinterpret_cast<unsigned short *>(o0)[q * P] = (unsigned short)(v & 0xFFFFu);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 19; ++q) o0[q * P] = Dev<R>::st(o[q]);
    }
    if (MOM) { rho_o[c] = rho; ux_o[c] = ux; uy_o[c] = uy; uz_o[c] = uz; }
}

// ---------------------------------------------------------------------------
// Two nodes per thread: lane l of a warp owns x = x0 + l and x = x0 + l + 32,
// x0 = 64 * (global warp index along the row).  Every load and store stays a
// plain coalesced run of 32 elements; the two nodes share the y/z geometry
// and most address arithmetic (the second node's addresses are the first's
// plus 32 elements, away from x walls).  The collision runs on the pair in
// packed FP32x2 arithmetic (FADD2/FMUL2/FFMA2, sm_100), which halves the
// arithmetic instruction count with FP32 results.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// Resident blocks per SM requested from the compiler for the pair kernels
// (caps their registers); set by the build.
#ifndef KB_PAIR_MIN_BLOCKS
#define KB_PAIR_MIN_BLOCKS 6
#endif

template <typename R, bool MOM, bool SOLID, typename I, bool SR>
__global__ void __launch_bounds__(BX, KB_PAIR_MIN_BLOCKS) trt_dev_x2_k(R *__restrict__ fo, const R *__restrict__ fi,
                                                    float *__restrict__ rho_o, float *__restrict__ ux_o,
                                                    float *__restrict__ uy_o, float *__restrict__ uz_o,
                                                    const uint8_t *__restrict__ solid, Grid3 g,
                                                    float sp, float sm) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int iA = warp * 64 + lane, iB = iA + 32;
    if (iA >= g.Nx) return;
    const bool vB = iB < g.Nx;
    const int j = blockIdx.y, k = blockIdx.z;
    const I P = (I)g.plane;
    const size_t row = (size_t)g.Nx * ((size_t)j + (size_t)g.Ny * k);
    const size_t cA = row + iA, cB = row + (vB ? iB : iA);
    float a[19], b[19];
    pull19_at(fi + cA, P, pull_geometry<I>(g, iA, j, k), a, DevLoad<R>());
    pull19_at(fi + cB, P, pull_geometry<I>(g, vB ? iB : iA, j, k), b, DevLoad<R>());
    float2 d[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) d[q] = make_float2(a[q], b[q]);

    float2 o[19], rho, ux, uy, uz;
    trt_dev_collide(d, o, rho, ux, uy, uz, sp, sm);
    uchar2 sm2 = make_uchar2(0, 0);
    if (SOLID) sm2 = make_uchar2(solid[cA], vB ? solid[cB] : 0);
    if (SR) {
        const uint32_t key = sr_key();
        unsigned short *fs = reinterpret_cast<unsigned short *>(fo);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const uint32_t v = SRPack<R>::pack(SOLID && sm2.x ? 0.f : o[q].x,
                                               SOLID && sm2.y ? 0.f : o[q].y, sr_bits(key, q));
            fs[cA + (size_t)(q * P)] = (unsigned short)(v & 0xFFFFu);
            if (vB) fs[cB + (size_t)(q * P)] = (unsigned short)(v >> 16);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            fo[cA + (size_t)(q * P)] = Dev<R>::st(SOLID && sm2.x ? 0.f : o[q].x);
            if (vB) fo[cB + (size_t)(q * P)] = Dev<R>::st(SOLID && sm2.y ? 0.f : o[q].y);
        }
    }
    if (MOM) {
        const bool sA = SOLID && sm2.x, sB = SOLID && sm2.y;
        rho_o[cA] = sA ? 1.f : rho.x; ux_o[cA] = sA ? 0.f : ux.x;
        uy_o[cA] = sA ? 0.f : uy.x; uz_o[cA] = sA ? 0.f : uz.x;
        if (vB) {
            rho_o[cB] = sB ? 1.f : rho.y; ux_o[cB] = sB ? 0.f : ux.y;
            uy_o[cB] = sB ? 0.f : uy.y; uz_o[cB] = sB ? 0.f : uz.y;
        }
    }
}

// ---------------------------------------------------------------------------
// Vector pairs (even Nx): lane t owns the adjacent nodes x0 = 2t, x0 + 1 of
// its warp's 64-node run, so each population of the pair is ONE aligned
// 2-element access (half2 / bfloat162 / float2) for loads and stores.  The
// x-shifted pulls take the missing element from the neighbouring lane by
// warp shuffle; lane 0 (c_x = +1) and the last lane of the run (c_x = -1)
// load that element directly, which also covers the periodic wrap and the
// half-way bounce-back at x walls.  All loads are issued before any shuffle
// so each thread keeps 19 vector requests in flight.
template <typename R> struct Vec2;
template <> struct Vec2<float> {
    static __device__ __forceinline__ float2 ld(const float *p) { return *reinterpret_cast<const float2 *>(p); }
    static __device__ __forceinline__ void st(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }
};
template <> struct Vec2<__half> {
    static __device__ __forceinline__ float2 ld(const __half *p) {
        return __half22float2(*reinterpret_cast<const __half2 *>(p));
    }
    static __device__ __forceinline__ void st(__half *p, float2 v) {
        *reinterpret_cast<__half2 *>(p) = __floats2half2_rn(v.x, v.y);
    }
};
template <> struct Vec2<__nv_bfloat16> {
    static __device__ __forceinline__ float2 ld(const __nv_bfloat16 *p) {
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(p));
    }
    static __device__ __forceinline__ void st(__nv_bfloat16 *p, float2 v) {
        *reinterpret_cast<__nv_bfloat162 *>(p) = __floats2bfloat162_rn(v.x, v.y);
    }
};

template <typename R, bool MOM, bool SOLID, typename I, bool SR>
__global__ void __launch_bounds__(BX, KB_PAIR_MIN_BLOCKS) trt_dev_v2_k(R *__restrict__ fo, const R *__restrict__ fi,
                                                    float *__restrict__ rho_o, float *__restrict__ ux_o,
                                                    float *__restrict__ uy_o, float *__restrict__ uz_o,
                                                    const uint8_t *__restrict__ solid, Grid3 g,
                                                    float sp, float sm) {
    constexpr int CX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    constexpr int CY[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
    constexpr int CZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
    constexpr int OP[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
    const int lane = threadIdx.x & 31;
    const int x0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int Nx = g.Nx;
    const bool valid = x0 < Nx;
    const bool last = x0 + 2 >= Nx;  // no valid neighbour lane to the right
    const int j = blockIdx.y, k = blockIdx.z;
    const I P = (I)g.plane;
    const bool px = g.per & 1, py = (g.per >> 1) & 1, pz = (g.per >> 2) & 1;
    const I sy = (I)Nx, sz = (I)Nx * (I)g.Ny;
    const bool ym = py || j > 0, yp = py || j < g.Ny - 1;
    const bool zm = pz || k > 0, zp = pz || k < g.Nz - 1;
    const I oym = (j > 0 ? (I)-1 : (I)(g.Ny - 1)) * sy;
    const I oyp = (j < g.Ny - 1 ? (I)1 : -(I)(g.Ny - 1)) * sy;
    const I ozm = (k > 0 ? (I)-1 : (I)(g.Nz - 1)) * sz;
    const I ozp = (k < g.Nz - 1 ? (I)1 : -(I)(g.Nz - 1)) * sz;
    const size_t row = (size_t)Nx * ((size_t)j + (size_t)g.Ny * k);
    const R *__restrict__ f0 = fi + row;  // row x = 0 of population 0, this (j, k)
    const int xv = valid ? x0 : 0;        // invalid lanes read a harmless in-row pair

    // 1. issue every load: the aligned pair and, for x-shifted populations,
    //    the one edge element this lane may need
    float2 a[19];
    float e[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        const bool ok = (CY[q] == 1 ? ym : CY[q] == -1 ? yp : true) &&
                        (CZ[q] == 1 ? zm : CZ[q] == -1 ? zp : true);
        const I srow = (CY[q] == 1 ? oym : CY[q] == -1 ? oyp : (I)0) +
                       (CZ[q] == 1 ? ozm : CZ[q] == -1 ? ozp : (I)0) + (I)q * P;
        const I orow = (I)OP[q] * P;  // own row, opposite population
        a[q] = Vec2<R>::ld(f0 + (ok ? srow : orow) + xv);
        e[q] = 0.f;
        if (CX[q] == 1) {
            // element for node x0: x0-1 in the source row, or wrap, or bounce
            const bool need = ok && (lane == 0);
            const I off = x0 > 0 ? srow + (I)(xv - 1) : (px ? srow + (I)(Nx - 1) : orow + (I)xv);
            if (need && valid) e[q] = Dev<R>::ld(f0[off]);
        } else if (CX[q] == -1) {
            // element for node x0+1: x0+2 in the source row, or wrap, or bounce
            const bool need = ok && (lane == 31 || last);
            const I off = !last ? srow + (I)(xv + 2) : (px ? srow : orow + (I)(xv + 1));
            if (need && valid) e[q] = Dev<R>::ld(f0[off]);
        }
    }
    // 2. assemble the pulled pair of every population
    float2 d[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        const bool ok = (CY[q] == 1 ? ym : CY[q] == -1 ? yp : true) &&
                        (CZ[q] == 1 ? zm : CZ[q] == -1 ? zp : true);
        if (CX[q] == 1) {
            const float up = __shfl_up_sync(0xffffffffu, a[q].y, 1);
            d[q] = ok ? make_float2(lane == 0 ? e[q] : up, a[q].x) : a[q];
        } else if (CX[q] == -1) {
            const float dn = __shfl_down_sync(0xffffffffu, a[q].x, 1);
            d[q] = ok ? make_float2(a[q].y, (lane == 31 || last) ? e[q] : dn) : a[q];
        } else {
            d[q] = a[q];
        }
    }
    if (!valid) return;

    float2 o[19], rho, ux, uy, uz;
    trt_dev_collide(d, o, rho, ux, uy, uz, sp, sm);
    const size_t oc = row + x0;
    uchar2 sm2 = make_uchar2(0, 0);
    if (SOLID) sm2 = *reinterpret_cast<const uchar2 *>(solid + oc);
    R *__restrict__ o0 = fo + oc;
    const uint32_t key = SR ? sr_key() : 0u;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        float2 v = o[q];
        if (SOLID) { if (sm2.x) v.x = 0.f; if (sm2.y) v.y = 0.f; }
        if (SR)
            *reinterpret_cast<uint32_t *>(o0 + (size_t)(q * P)) = SRPack<R>::pack(v.x, v.y, sr_bits(key, q));
        else
            Vec2<R>::st(o0 + (size_t)(q * P), v);
    }
    if (MOM) {
        float2 r = rho, aa = ux, bb = uy, cc = uz;
        if (SOLID) {
            if (sm2.x) { r.x = 1.f; aa.x = bb.x = cc.x = 0.f; }
            if (sm2.y) { r.y = 1.f; aa.y = bb.y = cc.y = 0.f; }
        }
        *reinterpret_cast<float2 *>(rho_o + oc) = r;
        *reinterpret_cast<float2 *>(ux_o + oc) = aa;
        *reinterpret_cast<float2 *>(uy_o + oc) = bb;
        *reinterpret_cast<float2 *>(uz_o + oc) = cc;
    }
}

// ---------------------------------------------------------------------------
// Quads, 16-bit storages (Nx % 4 == 0): lane t of a warp owns the four
// adjacent nodes x0 = 4t .. 4t + 3 of the warp's 128-node run of one row, so
// each population of the quad is ONE aligned 8-byte load and one 8-byte
// store, and the pull geometry (y/z source rows, walls, wraps) is computed
// once for four nodes.  An x-shifted population takes its missing element
// from the neighbouring lane by one 32-bit shuffle; the first / last lane of
// the run load it directly, which also covers the periodic wrap and the
// half-way bounce-back at x walls.  The collision runs as two packed FP32x2
// streams (nodes 0,1 and 2,3).
template <typename R> struct Pack16;
template <> struct Pack16<__half> {
    static __device__ __forceinline__ float2 unpack(uint32_t w) {
        return __half22float2(*reinterpret_cast<const __half2 *>(&w));
    }
    static __device__ __forceinline__ float lo(uint32_t w) {
        return __half2float(__ushort_as_half((unsigned short)(w & 0xFFFFu)));
    }
    static __device__ __forceinline__ float hi(uint32_t w) {
        return __half2float(__ushort_as_half((unsigned short)(w >> 16)));
    }
    static __device__ __forceinline__ uint32_t pack(float a, float b) {
        const __half2 h = __floats2half2_rn(a, b);
        return *reinterpret_cast<const uint32_t *>(&h);
    }
};
template <> struct Pack16<__nv_bfloat16> {
    static __device__ __forceinline__ float2 unpack(uint32_t w) {
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&w));
    }
    static __device__ __forceinline__ float lo(uint32_t w) { return __uint_as_float(w << 16); }
    static __device__ __forceinline__ float hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }
    static __device__ __forceinline__ uint32_t pack(float a, float b) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        return *reinterpret_cast<const uint32_t *>(&h);
    }
};

// Resident blocks per SM requested for the quad kernel (caps its registers).
#ifndef KB_QUAD_MIN_BLOCKS
#define KB_QUAD_MIN_BLOCKS 3
#endif

template <typename R, bool MOM, bool SOLID, typename I, bool SR>
__global__ void __launch_bounds__(128, KB_QUAD_MIN_BLOCKS) trt_dev_v4_k(R *__restrict__ fo, const R *__restrict__ fi,
                                                       float *__restrict__ rho_o, float *__restrict__ ux_o,
                                                       float *__restrict__ uy_o, float *__restrict__ uz_o,
                                                       const uint8_t *__restrict__ solid, Grid3 g,
                                                       float sp, float sm, int warps_per_row) {
    constexpr int CX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    constexpr int CY[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
    constexpr int CZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
    constexpr int OP[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
    using PK = Pack16<R>;
    const int lane = threadIdx.x & 31;
    const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const long long row_id = gw / warps_per_row;          // (j, k) row
    if (row_id >= (long long)g.Ny * g.Nz) return;         // whole warp: no shuffle partner left
    const int seg = (int)(gw - row_id * warps_per_row);
    const int j = (int)(row_id % g.Ny), k = (int)(row_id / g.Ny);
    const int Nx = g.Nx;
    const int x0 = seg * 128 + 4 * lane;
    const bool valid = x0 < Nx;
    const bool last = x0 + 4 >= Nx;  // no valid neighbour lane to the right
    const I P = (I)g.plane;
    const bool px = g.per & 1, py = (g.per >> 1) & 1, pz = (g.per >> 2) & 1;
    const I sy = (I)Nx, sz = (I)Nx * (I)g.Ny;
    const bool ym = py || j > 0, yp = py || j < g.Ny - 1;
    const bool zm = pz || k > 0, zp = pz || k < g.Nz - 1;
    const I oym = (j > 0 ? (I)-1 : (I)(g.Ny - 1)) * sy;
    const I oyp = (j < g.Ny - 1 ? (I)1 : -(I)(g.Ny - 1)) * sy;
    const I ozm = (k > 0 ? (I)-1 : (I)(g.Nz - 1)) * sz;
    const I ozp = (k < g.Nz - 1 ? (I)1 : -(I)(g.Nz - 1)) * sz;
    const size_t row = (size_t)Nx * ((size_t)j + (size_t)g.Ny * k);
    const R *__restrict__ f0 = fi + row;
    const int xv = valid ? x0 : 0;

    // 1. every load: the aligned quad and, for x-shifted populations, the one
    //    edge element this lane may need
    uint2 a[19];
    float e[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        const bool ok = (CY[q] == 1 ? ym : CY[q] == -1 ? yp : true) &&
                        (CZ[q] == 1 ? zm : CZ[q] == -1 ? zp : true);
        const I srow = (CY[q] == 1 ? oym : CY[q] == -1 ? oyp : (I)0) +
                       (CZ[q] == 1 ? ozm : CZ[q] == -1 ? ozp : (I)0) + (I)q * P;
        const I orow = (I)OP[q] * P;
        a[q] = *reinterpret_cast<const uint2 *>(f0 + (ok ? srow : orow) + xv);
        e[q] = 0.f;
        if (CX[q] == 1) {  // node x0 pulls x0 - 1
            const bool need = ok && lane == 0;
            const I off = x0 > 0 ? srow + (I)(xv - 1) : (px ? srow + (I)(Nx - 1) : orow + (I)xv);
            if (need && valid) e[q] = Dev<R>::ld(f0[off]);
        } else if (CX[q] == -1) {  // node x0 + 3 pulls x0 + 4
            const bool need = ok && (lane == 31 || last);
            const I off = !last ? srow + (I)(xv + 4) : (px ? srow : orow + (I)(xv + 3));
            if (need && valid) e[q] = Dev<R>::ld(f0[off]);
        }
    }
    // 2. assemble the pulled quad of every population as two float2
    float2 d0[19], d1[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        const bool ok = (CY[q] == 1 ? ym : CY[q] == -1 ? yp : true) &&
                        (CZ[q] == 1 ? zm : CZ[q] == -1 ? zp : true);
        const float2 l = PK::unpack(a[q].x), h = PK::unpack(a[q].y);  // elements 0,1 | 2,3
        if (CX[q] == 1) {
            const uint32_t up = __shfl_up_sync(0xffffffffu, a[q].y, 1);  // lane-1's elements 2,3
            const float left = lane == 0 ? e[q] : PK::hi(up);
            d0[q] = ok ? make_float2(left, l.x) : l;
            d1[q] = ok ? make_float2(l.y, h.x) : h;
        } else if (CX[q] == -1) {
            const uint32_t dn = __shfl_down_sync(0xffffffffu, a[q].x, 1);  // lane+1's elements 0,1
            const float right = (lane == 31 || last) ? e[q] : PK::lo(dn);
            d0[q] = ok ? make_float2(l.y, h.x) : l;
            d1[q] = ok ? make_float2(h.y, right) : h;
        } else {
            d0[q] = l;
            d1[q] = h;
        }
    }
    if (!valid) return;

    const size_t oc = row + x0;
    uchar4 m4 = make_uchar4(0, 0, 0, 0);
    if (SOLID) m4 = *reinterpret_cast<const uchar4 *>(solid + oc);
    R *__restrict__ o0 = fo + oc;
    const uint32_t key = SR ? sr_key() : 0u;
    uint32_t w0[19];
    float2 r0, ux0, uy0, uz0, r1, ux1, uy1, uz1;
    {
        float2 o[19];
        trt_dev_collide(d0, o, r0, ux0, uy0, uz0, sp, sm);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            float2 v = o[q];
            if (SOLID) { if (m4.x) v.x = 0.f; if (m4.y) v.y = 0.f; }
            w0[q] = SR ? SRPack<R>::pack(v.x, v.y, sr_bits(key, q)) : PK::pack(v.x, v.y);
        }
    }
    {
        float2 o[19];
        trt_dev_collide(d1, o, r1, ux1, uy1, uz1, sp, sm);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            float2 v = o[q];
            if (SOLID) { if (m4.z) v.x = 0.f; if (m4.w) v.y = 0.f; }
            uint32_t w1;
            if (SR) {
                const uint32_t r = sr_bits(key, q) * 0x85EBCA77u;
                w1 = SRPack<R>::pack(v.x, v.y, __funnelshift_l(r, r, 16));
            } else {
                w1 = PK::pack(v.x, v.y);
            }
            *reinterpret_cast<uint2 *>(o0 + (size_t)(q * P)) = make_uint2(w0[q], w1);
        }
    }
    if (MOM) {
        float4 r = make_float4(r0.x, r0.y, r1.x, r1.y), aa = make_float4(ux0.x, ux0.y, ux1.x, ux1.y);
        float4 bb = make_float4(uy0.x, uy0.y, uy1.x, uy1.y), cc = make_float4(uz0.x, uz0.y, uz1.x, uz1.y);
        if (SOLID) {
            if (m4.x) { r.x = 1.f; aa.x = bb.x = cc.x = 0.f; }
            if (m4.y) { r.y = 1.f; aa.y = bb.y = cc.y = 0.f; }
            if (m4.z) { r.z = 1.f; aa.z = bb.z = cc.z = 0.f; }
            if (m4.w) { r.w = 1.f; aa.w = bb.w = cc.w = 0.f; }
        }
        *reinterpret_cast<float4 *>(rho_o + oc) = r;
        *reinterpret_cast<float4 *>(ux_o + oc) = aa;
        *reinterpret_cast<float4 *>(uy_o + oc) = bb;
        *reinterpret_cast<float4 *>(uz_o + oc) = cc;
    }
}

template <typename R, typename I, bool SR>
static void launch_ri(void *f_out, const void *f_in, float *rho, float *ux, float *uy, float *uz,
                      const uint8_t *solid, const Grid3 &g, float sp, float sm, cudaStream_t s,
                      int kind) {
    R *fo = (R *)f_out;
    const R *fi = (const R *)f_in;
    if constexpr (sizeof(R) == 2) {
        if (kind == 4) {
            const int wpr = (g.Nx + 127) / 128;  // warps per row
            const long long warps = (long long)wpr * g.Ny * g.Nz;
            const dim3 grid((unsigned)((warps + 3) / 4));
            if (rho) {
                if (solid) trt_dev_v4_k<R, true, true, I, SR><<<grid, 128, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm, wpr);
                else trt_dev_v4_k<R, true, false, I, SR><<<grid, 128, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm, wpr);
            } else {
                if (solid) trt_dev_v4_k<R, false, true, I, SR><<<grid, 128, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm, wpr);
                else trt_dev_v4_k<R, false, false, I, SR><<<grid, 128, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm, wpr);
            }
            return;
        }
    }
    if (kind == 3) {
        const dim3 grid((g.Nx / 2 + BX - 1) / BX, g.Ny, g.Nz);
        if (rho) {
            if (solid) trt_dev_v2_k<R, true, true, I, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
            else trt_dev_v2_k<R, true, false, I, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
        } else {
            if (solid) trt_dev_v2_k<R, false, true, I, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
            else trt_dev_v2_k<R, false, false, I, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
        }
        return;
    }
    if (kind == 2) {
        const int threads_x = (g.Nx + 63) / 64 * 32;  // one warp per 64 nodes of a row
        const dim3 grid((threads_x + BX - 1) / BX, g.Ny, g.Nz);
        if (rho) {
            if (solid) trt_dev_x2_k<R, true, true, I, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
            else trt_dev_x2_k<R, true, false, I, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
        } else {
            if (solid) trt_dev_x2_k<R, false, true, I, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
            else trt_dev_x2_k<R, false, false, I, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
        }
        return;
    }
    const dim3 grid = nodes_grid(g.Nx, g.Ny, g.Nz);
    if (rho) {
        if (solid) trt_dev_k<R, true, true, I, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
        else trt_dev_k<R, true, false, I, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
    } else {
        if (solid) trt_dev_k<R, false, true, I, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
        else trt_dev_k<R, false, false, I, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
    }
}

template <typename R, bool SR = false>
static void launch_r(void *f_out, const void *f_in, float *rho, float *ux, float *uy, float *uz,
                     const uint8_t *solid, const Grid3 &g, float sp, float sm, cudaStream_t s,
                     int kind) {
    if (offsets_fit_int(g, 19))
        launch_ri<R, int, SR>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, kind);
    else
        launch_ri<R, long long, SR>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, kind);
    if (SR) sr_advance_k<<<1, 1, 0, s>>>();
}

int launch_trt3d_dev(int dtype, void *f_out, const void *f_in, float *rho, float *ux, float *uy,
                     float *uz, const uint8_t *solid, const Grid3 &g, float sp, float sm,
                     cudaStream_t s, int variant) {
    // variant: 0 automatic, 1 one node per thread, 2 nodes x and x+32 per
    // thread, 3 adjacent node pairs with vector accesses (even Nx only),
    // 4 adjacent node quads with 8-byte accesses (16-bit storages, Nx % 4 == 0).
    if (variant == 3 && g.Nx % 2 != 0)
        return set_error(KB_ERR_ARG, "kb_fused_trt_step_3d: the vector-pair kernel needs an even Nx");
    if (variant == 4 && (g.Nx % 4 != 0 || dtype == KB_F32_DEV))
        return set_error(KB_ERR_ARG,
                         "kb_fused_trt_step_3d: the quad kernel needs Nx %% 4 == 0 and 16-bit storage");
    // automatic choice, from measurements at 256^3 on B200: FP32 deviations
    // run fastest as vector pairs, FP16/BF16 as x / x+32 pairs
    int kind = variant;
    if (variant == 0) {
        if (dtype == KB_F32_DEV) kind = g.Nx % 2 == 0 ? 3 : 1;
        else kind = g.Nx >= 64 ? 2 : 1;
    }
    // the x / x+32 stores of the stochastic-rounding variant scatter 16-bit
    // halves; the vector-pair kernel stores each packed pair whole
    const int pairs = kind;
    switch (dtype) {
        case KB_F32_DEV: launch_r<float>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, pairs); break;
        case KB_F16_DEV: launch_r<__half>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, pairs); break;
        case KB_BF16_DEV: launch_r<__nv_bfloat16>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, pairs); break;
        case KB_F16_DEV_SR: launch_r<__half, true>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, pairs); break;
        case KB_BF16_DEV_SR: launch_r<__nv_bfloat16, true>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, pairs); break;
        default: return set_error(KB_ERR_UNSUPPORTED, "kb_fused_trt_step_3d: unknown dtype %d", dtype);
    }
    return check_launch("kb_fused_trt_step_3d");
}

template <typename R, bool SR>
static void launch_links_r(void *f_out, const void *f_in, float *rho, float *ux, float *uy,
                           float *uz, const LinkTable3 &L, const Grid3 &g, float sp, float sm,
                           cudaStream_t s) {
    const dim3 grid((g.Nx + BX - 1) / BX, g.Ny, g.Nz);
    R *fo = (R *)f_out;
    const R *fi = (const R *)f_in;
    if (offsets_fit_int(g, 19)) {
        if (rho) trt_dev_links_k<R, true, int, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
        else trt_dev_links_k<R, false, int, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
    } else {
        if (rho) trt_dev_links_k<R, true, long long, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
        else trt_dev_links_k<R, false, long long, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
    }
    if (SR) sr_advance_k<<<1, 1, 0, s>>>();
}

int launch_trt3d_dev_links(int dtype, void *f_out, const void *f_in, float *rho, float *ux,
                           float *uy, float *uz, const LinkTable3 &L, const Grid3 &g, float sp,
                           float sm, cudaStream_t s) {
    switch (dtype) {
        case KB_F32_DEV: launch_links_r<float, false>(f_out, f_in, rho, ux, uy, uz, L, g, sp, sm, s); break;
        case KB_F16_DEV: launch_links_r<__half, false>(f_out, f_in, rho, ux, uy, uz, L, g, sp, sm, s); break;
        case KB_BF16_DEV: launch_links_r<__nv_bfloat16, false>(f_out, f_in, rho, ux, uy, uz, L, g, sp, sm, s); break;
        case KB_F16_DEV_SR: launch_links_r<__half, true>(f_out, f_in, rho, ux, uy, uz, L, g, sp, sm, s); break;
        case KB_BF16_DEV_SR: launch_links_r<__nv_bfloat16, true>(f_out, f_in, rho, ux, uy, uz, L, g, sp, sm, s); break;
        default: return set_error(KB_ERR_UNSUPPORTED, "kb_fused_trt_libb_links_step_3d: unknown dtype %d", dtype);
    }
    return check_launch("kb_fused_trt_libb_links_step_3d");
}

}  // namespace d3

// ------------------------------------------------------ storage conversion --
namespace conv {

__device__ __forceinline__ double rd(const void *p, int dt, size_t m) {
    switch (dt) {
        case KB_F64: return ((const double *)p)[m];
        case KB_F32: return (double)((const float *)p)[m];
        case KB_F32_DEV: return (double)((const float *)p)[m];
        case KB_F16_DEV: return (double)__half2float(((const __half *)p)[m]);
        default: return (double)__bfloat162float(((const __nv_bfloat16 *)p)[m]);
    }
}

__device__ __forceinline__ void wr(void *p, int dt, size_t m, double v) {
    switch (dt) {
        case KB_F64: ((double *)p)[m] = v; break;
        case KB_F32: ((float *)p)[m] = (float)v; break;
        case KB_F32_DEV: ((float *)p)[m] = (float)v; break;
        case KB_F16_DEV: ((__half *)p)[m] = __double2half(v); break;
        default: ((__nv_bfloat16 *)p)[m] = __double2bfloat16(v); break;
    }
}

__device__ __forceinline__ bool is_dev(int dt) {
    return dt == KB_F32_DEV || dt == KB_F16_DEV || dt == KB_BF16_DEV;
}

__global__ void convert_k(void *dst, int ddt, const void *src, int sdt, int Q, size_t n) {
    ddt = storage_format(ddt);
    sdt = storage_format(sdt);
    const size_t total = (size_t)Q * n;
    for (size_t m = (size_t)blockIdx.x * blockDim.x + threadIdx.x; m < total;
         m += (size_t)gridDim.x * blockDim.x) {
        const int q = (int)(m / n);
        const double w = Q == 9 ? w9(q) : w19(q);
        double v = rd(src, sdt, m);
        if (is_dev(sdt)) v += w;   // to f
        if (is_dev(ddt)) v -= w;   // to f - w
        wr(dst, ddt, m, v);
    }
}

}  // namespace conv
}  // namespace kb

extern "C" int kb_set_stochastic_seed(unsigned int seed, void *stream) {
    if (cudaMemcpyToSymbolAsync(kb::d3::g_sr_epoch, &seed, sizeof(seed), 0, cudaMemcpyHostToDevice,
                                kb::as_stream(stream)) != cudaSuccess)
        return kb::check_launch("kb_set_stochastic_seed");
    // the host value must outlive the asynchronous copy
    if (cudaStreamSynchronize(kb::as_stream(stream)) != cudaSuccess)
        return kb::check_launch("kb_set_stochastic_seed");
    return 0;
}

extern "C" int kb_convert_populations(void *dst, int dst_dtype, const void *src, int src_dtype,
                                      int lattice_q, size_t n_nodes, void *stream) {
    KB_REQUIRE(dst && src, "kb_convert_populations: null pointer");
    KB_REQUIRE(lattice_q == 9 || lattice_q == 19, "kb_convert_populations: lattice_q must be 9 or 19");
    KB_REQUIRE(n_nodes > 0, "kb_convert_populations: n_nodes must be positive");
    KB_REQUIRE(kb::dtype_bytes(dst_dtype) && kb::dtype_bytes(src_dtype),
               "kb_convert_populations: unknown dtype (%d -> %d)", src_dtype, dst_dtype);
    const size_t total = (size_t)lattice_q * n_nodes;
    const size_t db = kb::dtype_bytes(dst_dtype), sb = kb::dtype_bytes(src_dtype);
    const char *d0 = (const char *)dst, *s0 = (const char *)src;
    KB_REQUIRE(d0 + total * db <= s0 || s0 + total * sb <= d0,
               "kb_convert_populations: src and dst overlap");
    const int threads = 256;
    size_t blocks = (total + threads - 1) / threads;
    const size_t cap = (size_t)kb::sm_count() * 8;
    if (blocks > cap) blocks = cap;
    kb::conv::convert_k<<<(unsigned)blocks, threads, 0, kb::as_stream(stream)>>>(
        dst, dst_dtype, src, src_dtype, lattice_q, n_nodes);
    return kb::check_launch("kb_convert_populations");
}
