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
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

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
// mean.  Each thread draws a key from an integer hash (lowbias32, C. Wellons)
// of its index and a launch counter in device memory that a one-thread kernel
// advances after every such launch (so CUDA-graph replays draw fresh bits and
// a run is reproducible on one stream); population q's word is derived from
// the key with one add (sr_bits).
__device__ unsigned int g_sr_epoch = 0;
// Consumer warps of the current staged launch that have finished; the last
// one advances g_sr_epoch (sr_epoch_done), so that kernel needs no
// sr_advance_k launch after it.
__device__ unsigned int g_sr_done = 0;

__global__ void sr_advance_k() { g_sr_epoch += 1u; }

// Called once by lane 0 of each of `warps` warps of a persistent launch, after
// every lane of the warp has read g_sr_epoch: the last warp to arrive
// advances the epoch and resets the count.  All reads of the epoch by this
// launch happen before its advance, as with a separate sr_advance_k.
__device__ __forceinline__ void sr_epoch_done(unsigned int warps) {
    __threadfence();
    if (atomicAdd(&g_sr_done, 1u) == warps - 1u) {
        g_sr_done = 0u;
        g_sr_epoch += 1u;
        __threadfence();
    }
}

// Per-thread key for this launch.
__device__ __forceinline__ uint32_t sr_key() {
    const uint32_t tid = (blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)) * blockDim.x +
                         threadIdx.x;
    const uint32_t e = *(volatile const unsigned int *)&g_sr_epoch;
    return hash32(tid ^ hash32(e + 0x632BE5ABu));
}
// Random word for population q (cvt.rs reads bits 0-12 for the low element
// and 16-28 for the high one): the key, a full hash, times an odd constant,
// plus q times another.  Each word is uniform because the key is, which keeps
// the rounding unbiased; the words of one key are correlated, not independent.
// The compiler forms key * M once, so a word costs one add.
__device__ __forceinline__ uint32_t sr_bits(uint32_t key, int q) {
    return key * 0x7FEB352Du + (uint32_t)q * 0x2C1B3C6Du;
}

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
    const V inv = vrcp_fast(rho);
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
    constexpr int CX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    constexpr int CY[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
    constexpr int CZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int x0 = warp * 64;  // first node of the warp's run (warp-uniform)
    const int iA = x0 + lane, iB = iA + 32;
    if (iA >= g.Nx) return;
    const bool vB = iB < g.Nx;
    const int j = blockIdx.y, k = blockIdx.z;
    const I P = (I)g.plane;
    const size_t cA = (size_t)g.Nx * ((size_t)j + (size_t)g.Ny * k) + iA;
    const bool px = g.per & 1, py = (g.per >> 1) & 1, pz = (g.per >> 2) & 1;
    const bool zh = (g.per & KB_ZHALO) != 0;
    // Fast path: a full 64-node run whose every pull source is a node at a
    // fixed y/z shift (inside the box or wrapped; block-uniform) and an x
    // shift of -1, 0 or +1, wrapped only on the two row-end lanes.  Node B's
    // sources are then node A's plus 32 elements (an immediate offset), and
    // one address per population serves both nodes.  Runs touching an x
    // wall, rows at a y or z wall and ragged run ends take the general pull.
    const bool yz_fast = (py || (j > 0 && j < g.Ny - 1)) && (pz || zh || (k > 0 && k < g.Nz - 1));
    const bool x_fast = x0 + 64 <= g.Nx && (px || (x0 > 0 && x0 + 64 < g.Nx));
    float a[19], b[19];
    if (yz_fast && x_fast) {
        const R *__restrict__ b0 = fi + cA;
        // c_x = +1 sources of node A and c_x = -1 sources of node B, relative
        // to node A: the x neighbour, or the wrapped one at a row end
        const R *__restrict__ bAm = b0 + (iA > 0 ? -1 : g.Nx - 1);
        const R *__restrict__ bBp = b0 + (iB < g.Nx - 1 ? 33 : 33 - g.Nx);
        const I sy = (I)g.Nx, sz = (I)g.Nx * (I)g.Ny;
        const I ym = j > 0 ? -sy : (I)(g.Ny - 1) * sy, yp = j < g.Ny - 1 ? sy : -(I)(g.Ny - 1) * sy;
        const I zm = (k > 0 || zh) ? -sz : (I)(g.Nz - 1) * sz;
        const I zp = (k < g.Nz - 1 || zh) ? sz : -(I)(g.Nz - 1) * sz;
        const DevLoad<R> ld;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const I u = (I)q * P + (CY[q] > 0 ? ym : CY[q] < 0 ? yp : (I)0) +
                        (CZ[q] > 0 ? zm : CZ[q] < 0 ? zp : (I)0);
            const R *__restrict__ p = b0 + u;
            if (CX[q] == 0) {
                a[q] = ld(p[0]);
                b[q] = ld(p[32]);
            } else if (CX[q] > 0) {
                a[q] = ld(bAm[u]);
                b[q] = ld(p[31]);
            } else {
                a[q] = ld(p[1]);
                b[q] = ld(bBp[u]);
            }
        }
    } else {
        pull19_at(fi + cA, P, pull_geometry<I>(g, iA, j, k), a, DevLoad<R>());
        pull19_at(fi + cA + (vB ? 32 : 0), P, pull_geometry<I>(g, vB ? iB : iA, j, k), b, DevLoad<R>());
    }
    float2 d[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) d[q] = make_float2(a[q], b[q]);

    float2 o[19], rho, ux, uy, uz;
    trt_dev_collide(d, o, rho, ux, uy, uz, sp, sm);
    uchar2 sm2 = make_uchar2(0, 0);
    if (SOLID) sm2 = make_uchar2(solid[cA], vB ? solid[cA + 32] : 0);
    R *__restrict__ o0 = fo + cA;  // node B stores at +32 elements
    if (SR) {
        const uint32_t key = sr_key();
        unsigned short *fs = reinterpret_cast<unsigned short *>(o0);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const uint32_t v = SRPack<R>::pack(SOLID && sm2.x ? 0.f : o[q].x,
                                               SOLID && sm2.y ? 0.f : o[q].y, sr_bits(key, q));
            unsigned short *s = fs + (I)q * P;
            s[0] = (unsigned short)(v & 0xFFFFu);
            if (vB) s[32] = (unsigned short)(v >> 16);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            R *s = o0 + (I)q * P;
            s[0] = Dev<R>::st(SOLID && sm2.x ? 0.f : o[q].x);
            if (vB) s[32] = Dev<R>::st(SOLID && sm2.y ? 0.f : o[q].y);
        }
    }
    if (MOM) {
        const bool sA = SOLID && sm2.x, sB = SOLID && sm2.y;
        float *r = rho_o + cA, *x = ux_o + cA, *y = uy_o + cA, *z = uz_o + cA;
        r[0] = sA ? 1.f : rho.x; x[0] = sA ? 0.f : ux.x;
        y[0] = sA ? 0.f : uy.x; z[0] = sA ? 0.f : uz.x;
        if (vB) {
            r[32] = sB ? 1.f : rho.y; x[32] = sB ? 0.f : ux.y;
            y[32] = sB ? 0.f : uy.y; z[32] = sB ? 0.f : uz.y;
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

// LINKS: `solid` is the class-byte row of a compact cut-link table (f1):
// class 1 nodes are solid, class 2 (cut) nodes are left to trt_dev_cut_k,
// which runs beside this kernel and writes only them.
template <typename R, bool MOM, bool SOLID, typename I, bool SR, bool LINKS = false>
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
    const bool zh = (g.per & KB_ZHALO) != 0;
    const bool zm = pz || zh || k > 0, zp = pz || zh || k < g.Nz - 1;
    const I oym = (j > 0 ? (I)-1 : (I)(g.Ny - 1)) * sy;
    const I oyp = (j < g.Ny - 1 ? (I)1 : -(I)(g.Ny - 1)) * sy;
    const I ozm = (k > 0 || zh ? (I)-1 : (I)(g.Nz - 1)) * sz;
    const I ozp = (k < g.Nz - 1 || zh ? (I)1 : -(I)(g.Nz - 1)) * sz;
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
    if (SOLID || LINKS) sm2 = *reinterpret_cast<const uchar2 *>(solid + oc);
    R *__restrict__ o0 = fo + oc;
    const uint32_t key = SR ? sr_key() : 0u;
    if (LINKS) {
        const bool wA = sm2.x != 2, wB = sm2.y != 2;
        if (!(wA && wB)) {
            // a pair with a cut node: only the other node is stored here
            const bool zA = sm2.x == 1, zB = sm2.y == 1;
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                const float vA = zA ? 0.f : o[q].x, vB = zB ? 0.f : o[q].y;
                if (SR) {
                    const uint32_t v = SRPack<R>::pack(vA, vB, sr_bits(key, q));
                    unsigned short *w = reinterpret_cast<unsigned short *>(o0 + (size_t)(q * P));
                    if (wA) w[0] = (unsigned short)(v & 0xFFFFu);
                    if (wB) w[1] = (unsigned short)(v >> 16);
                } else {
                    if (wA) o0[(size_t)(q * P)] = Dev<R>::st(vA);
                    if (wB) o0[(size_t)(q * P) + 1] = Dev<R>::st(vB);
                }
            }
            if (MOM) {
                if (wA) {
                    rho_o[oc] = zA ? 1.f : rho.x; ux_o[oc] = zA ? 0.f : ux.x;
                    uy_o[oc] = zA ? 0.f : uy.x; uz_o[oc] = zA ? 0.f : uz.x;
                }
                if (wB) {
                    rho_o[oc + 1] = zB ? 1.f : rho.y; ux_o[oc + 1] = zB ? 0.f : ux.y;
                    uy_o[oc + 1] = zB ? 0.f : uy.y; uz_o[oc + 1] = zB ? 0.f : uz.y;
                }
            }
            return;
        }
    }
    constexpr bool HS = SOLID || LINKS;  // a mask byte 1 means solid
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        float2 v = o[q];
        if (HS) { if (sm2.x) v.x = 0.f; if (sm2.y) v.y = 0.f; }
        if (SR)
            *reinterpret_cast<uint32_t *>(o0 + (size_t)(q * P)) = SRPack<R>::pack(v.x, v.y, sr_bits(key, q));
        else
            Vec2<R>::st(o0 + (size_t)(q * P), v);
    }
    if (MOM) {
        float2 r = rho, aa = ux, bb = uy, cc = uz;
        if (HS) {
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
    const bool zh = (g.per & KB_ZHALO) != 0;
    const bool zm = pz || zh || k > 0, zp = pz || zh || k < g.Nz - 1;
    const I oym = (j > 0 ? (I)-1 : (I)(g.Ny - 1)) * sy;
    const I oyp = (j < g.Ny - 1 ? (I)1 : -(I)(g.Ny - 1)) * sy;
    const I ozm = (k > 0 || zh ? (I)-1 : (I)(g.Nz - 1)) * sz;
    const I ozp = (k < g.Nz - 1 || zh ? (I)1 : -(I)(g.Nz - 1)) * sz;
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

// ---------------------------------------------------------------------------
// Row tiles staged by the tensor memory accelerator (16-bit storages).
// A persistent block walks tiles of TT = 256 nodes along x (a row segment at
// fixed z, in TY = 1 or 2 consecutive rows).  A producer warp streams each
// tile's pull sources into a ring of shared-memory stages with
// cp.async.bulk.tensor copies,
// each stage completed by a "full" mbarrier transaction count: for every
// population q the 256-element run of plane q at the pull source row
// (y - c_y, z - c_z), wrapped on periodic axes (13 copies: populations that
// share a source row and are adjacent in q travel in one box), and for the
// ten populations with c_x != 0 an 8-element halo run holding the one
// source outside the tile (x0 - 1 for c_x = +1, the element after the
// tile's last node for c_x = -1): the neighbouring segment, the periodic
// wrap, or at an x wall the node's own opposite population (half-way
// bounce-back).  A tile that spans a whole periodic row needs no halo run:
// its x wrap is read from the other end of the staged rows.  Four consumer
// warps wait on "full", read, release the stage
// on its "empty" mbarrier and collide; the loads of the next tiles run
// meanwhile and no register holds a load in flight.  Consumer thread t owns
// the adjacent nodes x0 + 2t, x0 + 2t + 1 and reads population q at the
// fixed shared-memory offset 2t - c_x (no address arithmetic per
// population); it stores each updated pair as one 4-byte word.  Rows whose
// pull meets a y or z wall take the direct pull of every population.
// Needs Nx % 8 == 0 and 16-byte aligned populations (tensor-map rules).
constexpr int TT = 256;                 // nodes per row tile
constexpr int THALO = 64;               // halo slot stride (elements, 128 bytes)
constexpr int TCONS = TT / 2;           // consumer threads: one per adjacent node pair
constexpr int TTHREADS = TCONS + 32;    // + the producer warp
constexpr long long TWAIT = 4000000;    // bounded mbarrier wait (polls)

// Stage layout of a tile of TY rows (y = j0 .. j0 + TY - 1): population q of
// row r at element (q * TY + r) * TT, then the halo slots of THALO elements
// (slot e of row r at (e * TY + r) * THALO: a tensor copy lands on a
// 128-byte boundary, so each halo row has a slot and a copy of its own),
// then the rows' class bytes of a cut-link step.  Two-row tiles halve the
// row copies and the per-tile work of the consumers per node; their stages
// are twice as large, so the ring holds 3 of them (3 blocks per SM fit in
// shared memory either way).
template <int TY> struct TileGeom {
    static constexpr int STAGES = TY == 1 ? 4 : 3;
    static constexpr int CLS = 19 * TT * TY + 10 * TY * THALO;  // element offset of the class bytes
    static constexpr int STAGE = CLS + TT * TY / 2;        // elements per stage
    static constexpr size_t SMEM = 128 + (size_t)STAGES * STAGE * 2;  // + alignment slack
    static constexpr uint32_t ROWBYTES = 19u * TT * 2u * TY;         // the 19 row runs
    static constexpr uint32_t BYTES = ROWBYTES + 10u * 8u * 2u * TY;  // + the 10 halo runs
};

#ifndef KB_TMA_MIN_BLOCKS
#define KB_TMA_MIN_BLOCKS 3
#endif

__device__ int g_tma_timeout = 0;  // set when a staged step gave up a bounded wait

// c_x = +1 populations (left tile end) with their y/z shifts; QM are their
// opposites, the c_x = -1 populations of the right end, with shifts negated.
__device__ constexpr int kQP[5] = {1, 7, 9, 11, 13}, kQM[5] = {2, 10, 8, 14, 12};
__device__ constexpr int kEY[5] = {0, 1, -1, 0, 0}, kEZ[5] = {0, 0, 0, 1, -1};

__device__ __forceinline__ uint32_t s_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ bool tbar_wait(uint32_t bar, uint32_t parity) {
    for (long long it = 0; it < TWAIT; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (it > 32) __nanosleep(128);
    }
    return false;
}
__device__ __forceinline__ void tbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tma_load4(uint32_t dst, const CUtensorMap *tm, int x, int y, int z,
                                          int q, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(q), "r"(bar)
        : "memory");
}

// Tiles are numbered x-segment fastest, then row group (TY rows), then z.
// A block visits tiles b, b + G, b + 2G, ... (G = grid size); a cursor
// (xt, jt, k) advances by G without a division per tile (jt counts row
// groups: rows jt * TY .. jt * TY + TY - 1).  staged() says whether every
// pull source row of a tile exists (interior or wrapped), i.e. it is staged.
template <int TY> struct TileMap {
    int ntx, Nx, Ny, Nz, per, zoff;
    int nyt;         // row groups per plane: Ny / TY
    int dx, dj, dk;  // G decomposed as (x-segments, row groups, planes)
    __device__ __forceinline__ void at(int t, int &xt, int &j, int &k) const {
        xt = t % ntx;
        const int r = t / ntx;
        j = r % nyt;
        k = r / nyt;
    }
    __device__ __forceinline__ void advance(int &xt, int &j, int &k) const {
        xt += dx;
        int c = xt >= ntx;
        xt -= c ? ntx : 0;
        j += dj + c;
        c = j >= nyt;
        j -= c ? nyt : 0;
        k += dk + c;
    }
    __device__ __forceinline__ bool staged(int jt, int k) const {
        const int j0 = jt * TY;
        return ((per & 2) || (j0 > 0 && j0 + TY < Ny)) && ((per & (4 | KB_ZHALO)) || (k > 0 && k < Nz - 1));
    }
};

// The copies of one staged tile (issued by one elected producer lane).
// Maps: t1 / t2 / t3 copy 1 / 2 / 3 consecutive planes of a 256-element
// row run, th an 8-element halo run of one plane.
struct TileMaps {
    const CUtensorMap *t1, *t2, *t3;  // boxes of TY rows
    const CUtensorMap *th;  // one halo row
    const CUtensorMap *tc;  // the rows' class bytes of a cut-link table, or null
    const CUtensorMap *s1;  // one row of one plane (wrapped row groups)
};
__device__ __forceinline__ void tma_load3(uint32_t dst, const CUtensorMap *tm, int x, int y, int z,
                                          uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}
// The copies of one staged tile of TY rows j .. j + TY - 1.  The source rows
// of a population with c_y = +1 / -1 are ym .. / yp .. (wrapped); a group
// whose rows would run past Ny - 1 (only where y wraps: row group 0 for
// c_y = +1, the last one for c_y = -1) travels as one copy per row and plane.
// Halo runs travel one row per copy.
template <int TY>
__device__ __forceinline__ void tma_issue_tile(const TileMaps &mp, uint32_t dst, uint32_t bar,
                                               int x0, int j, int k, const TileMap<TY> &m, bool halos) {
    using G = TileGeom<TY>;
    const uint32_t bytes = (halos ? G::BYTES : G::ROWBYTES) + (mp.tc ? (uint32_t)(TT * TY) : 0u);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
    // tensor-map z coordinates: the map spans the whole allocation, this
    // range starts at plane zoff; with a z halo the neighbours are read as is
    const bool zh = (m.per & KB_ZHALO) != 0;
    const int ym = j > 0 ? j - 1 : m.Ny - 1, yp = j < m.Ny - 1 ? j + 1 : 0;
    const int zm = ((k > 0 || zh) ? k - 1 : m.Nz - 1) + m.zoff;
    const int zp = ((k < m.Nz - 1 || zh) ? k + 1 : 0) + m.zoff;
    k += m.zoff;
    if (mp.tc) tma_load3(dst + G::CLS * 2, mp.tc, x0, j, k, bar);  // own rows' class bytes
    const uint32_t R = TT * 2;  // bytes per staged row
    // populations q0 .. q0 + nq - 1, row 0 sourced from row y of plane z
    const auto rows = [&](const CUtensorMap *tm, int q0, int nq, int y, int z) {
        if (TY == 1 || y + TY <= m.Ny) {
            tma_load4(dst + (uint32_t)(q0 * TY) * R, tm, x0, y, z, q0, bar);
        } else {
            for (int q = q0; q < q0 + nq; ++q)
                for (int r = 0; r < TY; ++r)
                    tma_load4(dst + (uint32_t)(q * TY + r) * R, mp.s1, x0, y + r < m.Ny ? y + r : y + r - m.Ny,
                              z, q, bar);
        }
    };
    rows(mp.t3, 0, 3, j, k);     // q 0, 1, 2: (0, 0)
    rows(mp.t1, 3, 1, ym, k);    // q 3: c_y = +1
    rows(mp.t1, 4, 1, yp, k);    // q 4: c_y = -1
    rows(mp.t1, 5, 1, j, zm);    // q 5: c_z = +1
    rows(mp.t1, 6, 1, j, zp);    // q 6: c_z = -1
    rows(mp.t2, 7, 2, ym, k);    // q 7, 8: c_y = +1
    rows(mp.t2, 9, 2, yp, k);    // q 9, 10: c_y = -1
    rows(mp.t2, 11, 2, j, zm);   // q 11, 12: c_z = +1
    rows(mp.t2, 13, 2, j, zp);   // q 13, 14: c_z = -1
    rows(mp.t1, 15, 1, ym, zm);  // q 15: (+1, +1)
    rows(mp.t1, 16, 1, yp, zm);  // q 16: (-1, +1)
    rows(mp.t1, 17, 1, ym, zp);  // q 17: (+1, -1)
    rows(mp.t1, 18, 1, yp, zp);  // q 18: (-1, -1)
    if (!halos) return;  // a periodic row in one tile: the wrap sources are in the rows
    // halos: slot e (left, c_x = +1) and 5 + e (right, c_x = -1) of row r at
    // (slot * TY + r) * THALO.  At an x wall the slot holds the end node's
    // own opposite population from its own row (node 0 at slot position 0,
    // node Nx - 1 at position 7).
    const bool px = m.per & 1;
    const uint32_t hdst = dst + 19 * TY * R;
    const bool lwall = x0 == 0 && !px, rwall = x0 + TT >= m.Nx && !px;
    const int xl = lwall ? 0 : (x0 > 0 ? x0 - 8 : m.Nx - 8);       // x0 - 1 (or Nx - 1) at 7
    const int xr = rwall ? m.Nx - 8 : (x0 + TT < m.Nx ? x0 + TT : 0); // next column (or 0) at 0
    const auto halo = [&](int slot, int x, int y, int z, int q) {
#pragma unroll
        for (int r = 0; r < TY; ++r)
            tma_load4(hdst + (uint32_t)((slot * TY + r) * THALO * 2), mp.th, x,
                      y + r < m.Ny ? y + r : y + r - m.Ny, z, q, bar);
    };
#pragma unroll
    for (int e = 0; e < 5; ++e) {
        const int yl = lwall ? j : (kEY[e] > 0 ? ym : kEY[e] < 0 ? yp : j);
        const int zl = lwall ? k : (kEZ[e] > 0 ? zm : kEZ[e] < 0 ? zp : k);
        const int yr = rwall ? j : (kEY[e] > 0 ? yp : kEY[e] < 0 ? ym : j);
        const int zr = rwall ? k : (kEZ[e] > 0 ? zp : kEZ[e] < 0 ? zm : k);
        halo(e, xl, yl, zl, lwall ? kQM[e] : kQP[e]);
        halo(5 + e, xr, yr, zr, rwall ? kQP[e] : kQM[e]);
    }
}

// The cut nodes of a compact link table (class 2), one thread per record:
// the same pull, interpolated bounce-back and collision as the one-node
// kernel trt_dev_links_k.  The staged step stores every other node, so the
// two kernels write disjoint nodes, read only f_in, and run side by side.
// The link data are loaded up front (libb_prephase_3d_record).
template <typename R, bool MOM, typename I, bool SR>
__global__ void __launch_bounds__(BX) trt_dev_cut_k(R *__restrict__ fo, const R *__restrict__ fi,
                                                     float *__restrict__ rho_o, float *__restrict__ ux_o,
                                                     float *__restrict__ uy_o, float *__restrict__ uz_o,
                                                     LinkTable3 L, Grid3 g, float sp, float sm) {
    const long long r = (long long)blockIdx.x * BX + threadIdx.x;
    if (r >= L.n_rec) return;
    const size_t c = (size_t)L.node[r];
    const size_t row = c / (size_t)g.Nx;
    const int i = (int)(c - row * (size_t)g.Nx), j = (int)(row % (size_t)g.Ny),
              k = (int)(row / (size_t)g.Ny);
    const I P = (I)g.plane;
    float d[19];
    pull19_at(fi + c, P, pull_geometry<I>(g, i, j, k), d, DevLoad<R>());
    libb_prephase_3d_record(fi + c, P, L, (int)r, d, DevLoad<R>());
    float o[19], rho, ux, uy, uz;
    trt_dev_collide(d, o, rho, ux, uy, uz, sp, sm);
    R *__restrict__ o0 = fo + c;
    if (SR) {
        const uint32_t key =
            hash32((uint32_t)c ^ hash32(*(volatile const unsigned int *)&g_sr_epoch + 0x632BE5ABu));
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

// LINKS: the compact cut-link table (row f1) in place of a solid mask: class
// 1 nodes are solid; class 2 nodes are left to trt_dev_cut_k.  TY: rows per
// tile (1, or 2 for an even Ny); a consumer thread updates its pair of
// nodes in each of the tile's rows in turn.
template <typename R, bool MOM, bool SOLID, typename I, bool SR, bool LINKS = false, int TY = 1>
__global__ void __launch_bounds__(TTHREADS, KB_TMA_MIN_BLOCKS)
    trt_dev_tma_k(const __grid_constant__ CUtensorMap tmap1, const __grid_constant__ CUtensorMap tmap2,
                  const __grid_constant__ CUtensorMap tmap3, const __grid_constant__ CUtensorMap thalo,
                  const __grid_constant__ CUtensorMap tcls, const __grid_constant__ CUtensorMap ts1,
                  R *__restrict__ fo, const R *__restrict__ fi, float *__restrict__ rho_o,
                  float *__restrict__ ux_o, float *__restrict__ uy_o, float *__restrict__ uz_o,
                  const uint8_t *__restrict__ solid, Grid3 g, float sp, float sm, LinkTable3 L) {
    constexpr bool HS = SOLID || LINKS;  // some nodes are solid
    constexpr int CX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    using G = TileGeom<TY>;
    constexpr int NS = G::STAGES;
    extern __shared__ unsigned char tsm_raw[];
    __shared__ __align__(8) uint64_t full[NS], empty[NS];
    R *stage0 = reinterpret_cast<R *>(tsm_raw + ((128u - (s_addr(tsm_raw) & 127u)) & 127u));
    const int t = threadIdx.x;
    TileMap<TY> m;
    m.ntx = (g.Nx + TT - 1) / TT;
    m.Nx = g.Nx;
    m.Ny = g.Ny;
    m.nyt = g.Ny / TY;
    m.Nz = g.Nz;
    m.per = g.per;
    m.zoff = g.zoff;
    m.at((int)gridDim.x, m.dx, m.dj, m.dk);
    if (t == 0) {
        for (int s = 0; s < NS; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(s_addr(&full[s])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_addr(&empty[s])),
                         "r"(TCONS / 32));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int cx, cj, ck;  // this role's current tile
    m.at((int)blockIdx.x, cx, cj, ck);

    if (t >= TCONS) {
        // ------------------------------------------------ producer warp --
        const TileMaps mp{&tmap1, &tmap2, &tmap3, &thalo, LINKS ? &tcls : nullptr, &ts1};
        if (t == TCONS) {
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmap1)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmap2)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmap3)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&thalo)) : "memory");
            if (LINKS)
                asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tcls)) : "memory");
            if (TY > 1)
                asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&ts1)) : "memory");
        }
        // one tile spans a periodic row: its x wrap reads the staged rows, so
        // no halo runs are copied
        const bool halos = !((g.per & 1) && m.ntx == 1);
#pragma unroll 1
        for (int n = 0; ck < g.Nz; m.advance(cx, cj, ck), ++n) {
            const int s = n % NS;
            // the consumers have released this stage's previous tile; every
            // lane of the warp leaves the loop together on a timeout (the
            // __syncwarp below needs all of them)
            if (n >= NS &&
                !__all_sync(0xffffffffu,
                            tbar_wait(s_addr(&empty[s]), (uint32_t)(n / NS - 1) & 1u))) {
                if (t == TCONS) atomicExch(&g_tma_timeout, 1);
                break;
            }
            if (t == TCONS) {
                const uint32_t bar = s_addr(&full[s]);
                if (m.staged(cj, ck))
                    tma_issue_tile<TY>(mp, s_addr(stage0 + s * G::STAGE), bar, cx * TT, cj * TY, ck, m,
                                       halos);
                else  // nothing to copy: the phase completes on the arrival
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], 0;" ::"r"(bar)
                                 : "memory");
            }
            __syncwarp();
        }
        return;
    }

    // ---------------------------------------------------- consumer warps --
    const I P = (I)g.plane;
    // stochastic rounding: one full hash per thread and launch; each tile
    // advances it by a Weyl step and one multiply, and population q's word is
    // that plus q times a constant (one add).  Every word is uniform, which is
    // what makes the rounding unbiased; words of one thread are correlated,
    // not independent.
    const uint32_t ekey =
        SR ? hash32(((uint32_t)blockIdx.x * TTHREADS + (uint32_t)t) ^
                    hash32(*(volatile const unsigned int *)&g_sr_epoch + 0x632BE5ABu))
           : 0u;
    const bool wrapx = (g.per & 1) && m.ntx == 1;  // as the producer's !halos
    int it = 0;
    bool aborted = false;
#pragma unroll 1
    for (; ck < g.Nz; m.advance(cx, cj, ck), ++it) {
        const int s = it % NS;
        const int x0 = cx * TT, k = ck;
        const int iA = x0 + 2 * t;
        const bool live = iA < g.Nx;  // Nx even: both nodes of the pair or neither
        if (!tbar_wait(s_addr(&full[s]), (uint32_t)(it / NS) & 1u)) {
            atomicExch(&g_tma_timeout, 1);
            aborted = true;
            break;
        }
        const bool staged = m.staged(cj, k);
        const R *stage = stage0 + s * G::STAGE;
        // one row of the tile: rows one after the other (round to nearest) or
        // unrolled (the stochastic-rounding loop spills at 128 registers unless
        // unrolled)
        const auto row = [&](const int r) {
            const int j = cj * TY + r;
            const size_t cA = (size_t)g.Nx * ((size_t)j + (size_t)g.Ny * k) + iA;
            uchar2 cl = make_uchar2(0, 0);  // LINKS: the pair's class bytes
            float2 d[19];
            if (staged) {
                if (LINKS)
                    cl = *reinterpret_cast<const uchar2 *>(
                        reinterpret_cast<const unsigned char *>(stage + G::CLS) + r * TT + 2 * t);
                const R *st = stage + r * TT + 2 * t;
                const DevLoad<R> ld;
#pragma unroll
                for (int q = 0; q < 19; ++q) {
                    const R *rq = st + q * TY * TT;  // reads at -1 / +256 fall in the neighbouring rows
                    if (CX[q] == 0) d[q] = Vec2<R>::ld(rq);
                    else if (CX[q] > 0) d[q] = make_float2(ld(rq[-1]), ld(rq[0]));
                    else d[q] = make_float2(ld(rq[1]), ld(rq[2]));
                }
                // the tile ends take the halo slots (the thread holding the
                // tile's last node: local index min(TT, Nx - x0) - 1, odd), or,
                // when the tile is a whole periodic row, the other end of the
                // staged row itself (x = Nx - 1 feeds node 0, x = 0 feeds Nx - 1)
                const R *h = stage + 19 * TY * TT + r * THALO;
                const R *rows = stage + r * TT;
                if (t == 0) {
                    if (wrapx) {
#pragma unroll
                        for (int e = 0; e < 5; ++e) d[kQP[e]].x = ld(rows[kQP[e] * TY * TT + g.Nx - 1]);
                    } else {
                        const int pl = (x0 == 0 && !(g.per & 1)) ? 0 : 7;
#pragma unroll
                        for (int e = 0; e < 5; ++e) d[kQP[e]].x = ld(h[e * TY * THALO + pl]);
                    }
                }
                if (t == (min(TT, g.Nx - x0) - 2) >> 1) {
                    if (wrapx) {
#pragma unroll
                        for (int e = 0; e < 5; ++e) d[kQM[e]].y = ld(rows[kQM[e] * TY * TT]);
                    } else {
                        const int pr = (x0 + TT >= g.Nx && !(g.per & 1)) ? 7 : 0;
#pragma unroll
                        for (int e = 0; e < 5; ++e) d[kQM[e]].y = ld(h[(5 + e) * TY * THALO + pr]);
                    }
                }
            } else if (live) {
                // rows at a y or z wall: direct pull of both nodes
                if (LINKS) cl = *reinterpret_cast<const uchar2 *>(L.cls + cA);
                float a[19], b[19];
                pull19_at(fi + cA, P, pull_geometry<I>(g, iA, j, k), a, DevLoad<R>());
                pull19_at(fi + cA + 1, P, pull_geometry<I>(g, iA + 1, j, k), b, DevLoad<R>());
#pragma unroll
                for (int q = 0; q < 19; ++q) d[q] = make_float2(a[q], b[q]);
            }
            if (r == TY - 1) {
                __syncwarp();
                if ((t & 31) == 0) tbar_arrive(s_addr(&empty[s]));  // this warp is done with stage s
            }
            if (!live) return;
            uchar2 sm2 = make_uchar2(0, 0);
            if (LINKS) {
                sm2 = make_uchar2(cl.x == 1, cl.y == 1);
            } else if (SOLID) {
                sm2 = *reinterpret_cast<const uchar2 *>(solid + cA);
            }
            // the rates pass through opaque moves each tile so the collision's
            // rate-derived constants are formed here, not held across the loop
            float spl, sml;
            asm volatile("mov.b32 %0, %1;" : "=f"(spl) : "f"(sp));
            asm volatile("mov.b32 %0, %1;" : "=f"(sml) : "f"(sm));
            float2 o[19], rho, ux, uy, uz;
            trt_dev_collide(d, o, rho, ux, uy, uz, spl, sml);
            // solid nodes store rest equilibrium (d = 0) and rho = 1, u = 0; only
            // warps that hold one pay for the selects
            if (HS && __any_sync(__activemask(), (sm2.x | sm2.y) != 0)) {
#pragma unroll
                for (int q = 0; q < 19; ++q) o[q] = make_float2(sm2.x ? 0.f : o[q].x, sm2.y ? 0.f : o[q].y);
                rho = make_float2(sm2.x ? 1.f : rho.x, sm2.y ? 1.f : rho.y);
                ux = make_float2(sm2.x ? 0.f : ux.x, sm2.y ? 0.f : ux.y);
                uy = make_float2(sm2.x ? 0.f : uy.x, sm2.y ? 0.f : uy.y);
                uz = make_float2(sm2.x ? 0.f : uz.x, sm2.y ? 0.f : uz.y);
            }
            // likewise the plane stride, so the 19 plane offsets are not hoisted
            I Pl;
            if constexpr (sizeof(I) == 4) asm volatile("mov.b32 %0, %1;" : "=r"(Pl) : "r"((int)P));
            else asm volatile("mov.b64 %0, %1;" : "=l"(Pl) : "l"((long long)P));
            R *o0 = fo + cA;
            if (LINKS && (cl.x == 2 || cl.y == 2)) {
                // a pair with a cut node: trt_dev_cut_k writes that node (it runs
                // beside this kernel), so only the other node is stored here
                const bool wA = cl.x != 2, wB = cl.y != 2;
                const uint32_t key = SR ? (ekey + (uint32_t)(it * TY + r) * 0x9E3779B9u) * 0x7FEB352Du : 0u;
#pragma unroll
                for (int q = 0; q < 19; ++q) {
                    const float vA = o[q].x, vB = o[q].y;
                    unsigned short *w = reinterpret_cast<unsigned short *>(o0 + (I)q * Pl);
                    if (SR) {
                        const uint32_t v = SRPack<R>::pack(vA, vB, key + (uint32_t)q * 0x2C1B3C6Du);
                        if (wA) w[0] = (unsigned short)(v & 0xFFFFu);
                        if (wB) w[1] = (unsigned short)(v >> 16);
                    } else {
                        if (wA) o0[(I)q * Pl] = Dev<R>::st(vA);
                        if (wB) o0[(I)q * Pl + 1] = Dev<R>::st(vB);
                    }
                }
                if (MOM) {
                    if (wA) { rho_o[cA] = rho.x; ux_o[cA] = ux.x; uy_o[cA] = uy.x; uz_o[cA] = uz.x; }
                    if (wB) { rho_o[cA + 1] = rho.y; ux_o[cA + 1] = ux.y; uy_o[cA + 1] = uy.y; uz_o[cA + 1] = uz.y; }
                }
                return;
            }
            if (SR) {
                const uint32_t key = (ekey + (uint32_t)(it * TY + r) * 0x9E3779B9u) * 0x7FEB352Du;
#pragma unroll
                for (int q = 0; q < 19; ++q) {
                    const uint32_t v = SRPack<R>::pack(o[q].x, o[q].y, key + (uint32_t)q * 0x2C1B3C6Du);
                    *reinterpret_cast<uint32_t *>(o0 + (I)q * Pl) = v;
                }
            } else {
#pragma unroll
                for (int q = 0; q < 19; ++q)
                    Vec2<R>::st(o0 + (I)q * Pl, o[q]);
            }
            if (MOM) {
                *reinterpret_cast<float2 *>(rho_o + cA) = rho;
                *reinterpret_cast<float2 *>(ux_o + cA) = ux;
                *reinterpret_cast<float2 *>(uy_o + cA) = uy;
                *reinterpret_cast<float2 *>(uz_o + cA) = uz;
            }
        };
        if constexpr (SR) {
#pragma unroll
            for (int r = 0; r < TY; ++r) row(r);
        } else {
#pragma unroll 1
            for (int r = 0; r < TY; ++r) row(r);
        }
    }
    // after a timeout: wait (bounded) for copies the producer may still have
    // in flight, so none lands in shared memory after the block has exited
    if (aborted && (t & 31) == 0) {
        for (int n = 0; n < NS && ck < g.Nz; ++n, m.advance(cx, cj, ck)) {
            const int i2 = it + n;
            tbar_wait(s_addr(&full[i2 % NS]), (uint32_t)(i2 / NS) & 1u);
        }
    }
    // stochastic rounding: this launch's last consumer warp advances the
    // epoch (the cut-link step keeps sr_advance_k, after its side kernel)
    if (SR && !LINKS) {
        __syncwarp();
        if ((t & 31) == 0) sr_epoch_done(gridDim.x * (TCONS / 32));
    }
}

static PFN_cuTensorMapEncodeTiled_v12000 tma_encode_fn() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// The staged kernel's layout and alignment rules: Nx % 8 == 0 (16-byte
// row pitch of the tensor map), 16-byte aligned input populations, 4-byte
// aligned output pairs, 8-byte aligned moment pairs, 2-byte aligned mask
// pairs, tile count within int.
static bool tma_eligible(const Grid3 &g, const void *f_out, const void *f_in, const float *rho,
                         const float *ux, const float *uy, const float *uz, const uint8_t *solid) {
    const auto al = [](const void *p, uintptr_t a) { return ((uintptr_t)p & (a - 1)) == 0; };
    const double tiles = (double)((g.Nx + TT - 1) / TT) * g.Ny * g.Nz;
    return g.Nx % 8 == 0 && al(f_in, 16) && al(f_out, 4) && al(rho, 8) && al(ux, 8) &&
           al(uy, 8) && al(uz, 8) && al(solid, 2) && tiles < 2147483647.0 &&
           tma_encode_fn() != nullptr;
}

// Maps of one population buffer: [0..2] 256-element runs of TY rows of 1, 2
// and 3 consecutive planes, [3] 8-element halo runs of one row of one plane,
// [4] class bytes of a cut-link table (x, y, z) 256-byte runs of TY rows,
// [5] one row of [0] (the copies of wrapped row groups).
struct TmaMaps {
    CUtensorMap m[6];
};

template <typename R, bool MOM, bool SOLID, typename I, bool SR, bool LINKS = false, int TY = 1>
static int launch_tma_k(const TmaMaps &mp, R *fo, const R *fi, float *rho, float *ux, float *uy,
                        float *uz, const uint8_t *solid, const Grid3 &g, float sp, float sm,
                        cudaStream_t s, const LinkTable3 &L = LinkTable3{}) {
    constexpr size_t smem = TileGeom<TY>::SMEM;
    const auto kern = trt_dev_tma_k<R, MOM, SOLID, I, SR, LINKS, TY>;
    // resident blocks per SM of this instantiation, per device (the shared
    // memory opt-in below is a per-device attribute too)
    static int occ_dev[64] = {};
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return set_error(KB_ERR_CUDA, "kb_fused_trt_step_3d: no usable current device");
    int &occ = occ_dev[dev];
    if (occ <= 0) {
        int n = 0;
        // the stage ring may exceed the 48 KB default of dynamic shared memory
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return set_error(KB_ERR_CUDA, "kb_fused_trt_step_3d: %zu bytes of shared memory per "
                             "block refused", smem);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, TTHREADS, smem) != cudaSuccess ||
            n < 1) {
            cudaGetLastError();
            n = 1;
        }
        occ = n;
    }
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long tiles = (long long)((g.Nx + TT - 1) / TT) * (g.Ny / TY) * g.Nz;
    const int blocks = (int)std::min<long long>(tiles, (long long)sms * occ);
    kern<<<blocks, TTHREADS, smem, s>>>(mp.m[0], mp.m[1], mp.m[2], mp.m[3], mp.m[4], mp.m[5], fo, fi,
                                        rho, ux, uy, uz, solid, g, sp, sm, L);
    return KB_OK;
}

// ty: rows per tile, 0 automatic (2 where Ny is even and the offsets fit in
// int; else 1).
template <typename R, typename I, bool SR>
static int launch_tma(void *f_out, const void *f_in, float *rho, float *ux, float *uy, float *uz,
                      const uint8_t *solid, const Grid3 &g, float sp, float sm, cudaStream_t s,
                      const LinkTable3 *links = nullptr, int ty = 0) {
    constexpr bool I32 = sizeof(I) == 4;
    if (ty == 0) ty = (I32 && g.Ny % 2 == 0) ? 2 : 1;
    if (ty != 1 && !(ty == 2 && I32 && g.Ny % 2 == 0))
        return set_error(KB_ERR_ARG, "kb_fused_trt_step_3d: two-row tiles need an even Ny");
    // the populations as a 4-D tensor (x, y, z, q) of 16-bit words over the
    // whole allocation (a z-range starts at its plane g.zoff)
    TmaMaps mp;
    const size_t nxy = (size_t)g.Nx * (size_t)g.Ny;
    const void *fbase = (const char *)f_in - (size_t)g.zoff * nxy * 2;
    const cuuint64_t dims[4] = {(cuuint64_t)g.Nx, (cuuint64_t)g.Ny, (cuuint64_t)(g.plane / nxy), 19};
    const cuuint64_t strides[3] = {(cuuint64_t)g.Nx * 2, (cuuint64_t)g.Nx * g.Ny * 2,
                                   (cuuint64_t)g.plane * 2};
    const cuuint32_t y = (cuuint32_t)ty;
    const cuuint32_t boxes[5][4] = {{TT, y, 1, 1}, {TT, y, 1, 2}, {TT, y, 1, 3}, {8, 1, 1, 1},
                                    {TT, 1, 1, 1}};
    const int slot[5] = {0, 1, 2, 3, 5};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    for (int n = 0; n < 5; ++n) {
        const CUresult r = tma_encode_fn()(&mp.m[slot[n]], CU_TENSOR_MAP_DATA_TYPE_UINT16, 4,
                                           const_cast<void *>(fbase), dims, strides, boxes[n], es,
                                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS)
            return set_error(KB_ERR_CUDA, "kb_fused_trt_step_3d: cuTensorMapEncodeTiled failed (%d)",
                             (int)r);
    }
    mp.m[4] = mp.m[3];  // unused placeholder unless a cut-link table is staged
    if (links) {
        const cuuint64_t cd[3] = {(cuuint64_t)g.Nx, (cuuint64_t)g.Ny, (cuuint64_t)g.Nz};
        const cuuint64_t cs[2] = {(cuuint64_t)g.Nx, (cuuint64_t)g.Nx * g.Ny};
        const cuuint32_t cb[3] = {TT, (cuuint32_t)ty, 1};
        const CUresult r = tma_encode_fn()(&mp.m[4], CU_TENSOR_MAP_DATA_TYPE_UINT8, 3,
                                           const_cast<uint8_t *>(links->cls), cd, cs, cb, es,
                                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS)
            return set_error(KB_ERR_CUDA, "kb_fused_trt_libb_links_step_3d: cuTensorMapEncodeTiled "
                             "failed (%d)", (int)r);
    }
    R *fo = (R *)f_out;
    const R *fi = (const R *)f_in;
    if constexpr (I32) {
        if (ty == 2 && links) {
            if (rho) return launch_tma_k<R, true, false, I, SR, true, 2>(mp, fo, fi, rho, ux, uy, uz, nullptr, g, sp, sm, s, *links);
            return launch_tma_k<R, false, false, I, SR, true, 2>(mp, fo, fi, rho, ux, uy, uz, nullptr, g, sp, sm, s, *links);
        }
    }
    if (links) {
        if (rho) return launch_tma_k<R, true, false, I, SR, true>(mp, fo, fi, rho, ux, uy, uz, nullptr, g, sp, sm, s, *links);
        return launch_tma_k<R, false, false, I, SR, true>(mp, fo, fi, rho, ux, uy, uz, nullptr, g, sp, sm, s, *links);
    }
    if constexpr (I32) {
        if (ty == 2) {
            if (rho) {
                if (solid) return launch_tma_k<R, true, true, I, SR, false, 2>(mp, fo, fi, rho, ux, uy, uz, solid, g, sp, sm, s);
                return launch_tma_k<R, true, false, I, SR, false, 2>(mp, fo, fi, rho, ux, uy, uz, solid, g, sp, sm, s);
            }
            if (solid) return launch_tma_k<R, false, true, I, SR, false, 2>(mp, fo, fi, rho, ux, uy, uz, solid, g, sp, sm, s);
            return launch_tma_k<R, false, false, I, SR, false, 2>(mp, fo, fi, rho, ux, uy, uz, solid, g, sp, sm, s);
        }
    }
    if (rho) {
        if (solid) return launch_tma_k<R, true, true, I, SR>(mp, fo, fi, rho, ux, uy, uz, solid, g, sp, sm, s);
        return launch_tma_k<R, true, false, I, SR>(mp, fo, fi, rho, ux, uy, uz, solid, g, sp, sm, s);
    }
    if (solid) return launch_tma_k<R, false, true, I, SR>(mp, fo, fi, rho, ux, uy, uz, solid, g, sp, sm, s);
    return launch_tma_k<R, false, false, I, SR>(mp, fo, fi, rho, ux, uy, uz, solid, g, sp, sm, s);
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
static int launch_r(void *f_out, const void *f_in, float *rho, float *ux, float *uy, float *uz,
                    const uint8_t *solid, const Grid3 &g, float sp, float sm, cudaStream_t s,
                    int kind) {
    if constexpr (sizeof(R) == 2) {
        if (kind == 5 || kind == 6) {
            const int ty = kind == 6 ? 1 : 0;  // 6: one-row tiles
            const int rc = offsets_fit_int(g, 19)
                               ? launch_tma<R, int, SR>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, nullptr, ty)
                               : launch_tma<R, long long, SR>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, nullptr, ty);
            // (the staged kernel advances the stochastic-rounding epoch itself)
            return rc;
        }
    }
    if (offsets_fit_int(g, 19))
        launch_ri<R, int, SR>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, kind);
    else
        launch_ri<R, long long, SR>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, kind);
    if (SR) sr_advance_k<<<1, 1, 0, s>>>();
    return KB_OK;
}

int launch_trt3d_dev(int dtype, void *f_out, const void *f_in, float *rho, float *ux, float *uy,
                     float *uz, const uint8_t *solid, const Grid3 &g, float sp, float sm,
                     cudaStream_t s, int variant) {
    // variant: 0 automatic, 1 one node per thread, 2 nodes x and x+32 per
    // thread, 3 adjacent node pairs with vector accesses (even Nx only),
    // 4 adjacent node quads with 8-byte accesses (16-bit storages, Nx % 4 == 0),
    // 5 row tiles staged by the tensor memory accelerator (16-bit storages,
    // Nx % 8 == 0, aligned buffers; two rows per tile where Ny is even), 6
    // the same with one row per tile.
    if (variant == 3 && g.Nx % 2 != 0)
        return set_error(KB_ERR_ARG, "kb_fused_trt_step_3d: the vector-pair kernel needs an even Nx");
    if (variant == 4 && (g.Nx % 4 != 0 || dtype == KB_F32_DEV))
        return set_error(KB_ERR_ARG,
                         "kb_fused_trt_step_3d: the quad kernel needs Nx %% 4 == 0 and 16-bit storage");
    if ((variant == 5 || variant == 6) &&
        (dtype == KB_F32_DEV || !tma_eligible(g, f_out, f_in, rho, ux, uy, uz, solid)))
        return set_error(KB_ERR_ARG,
                         "kb_fused_trt_step_3d: the staged kernel needs 16-bit storage, Nx %% 8 == 0 "
                         "and 16-byte aligned populations");
    // automatic choice, from measurements at 256^3 on B200: FP32 deviations
    // run fastest as vector pairs (44.5 GLUPS); FP16/BF16 as staged row
    // tiles (78.7 GLUPS) where the rows fill the 256-node tiles to 90 % or
    // more, else as x / x+32 pairs (65.2 GLUPS at 256^3)
    int kind = variant;
    if (variant == 0) {
        const int ntx = (g.Nx + TT - 1) / TT;
        if (dtype == KB_F32_DEV) kind = g.Nx % 2 == 0 ? 3 : 1;
        else if (10 * g.Nx >= 9 * ntx * TT && tma_eligible(g, f_out, f_in, rho, ux, uy, uz, solid))
            kind = 5;
        else kind = g.Nx >= 64 ? 2 : 1;
    }
    // the x / x+32 stores of the stochastic-rounding variant scatter 16-bit
    // halves; the vector-pair kernel stores each packed pair whole
    const int pairs = kind;
    int rc = KB_OK;
    switch (dtype) {
        case KB_F32_DEV: rc = launch_r<float>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, pairs); break;
        case KB_F16_DEV: rc = launch_r<__half>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, pairs); break;
        case KB_BF16_DEV: rc = launch_r<__nv_bfloat16>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, pairs); break;
        case KB_F16_DEV_SR: rc = launch_r<__half, true>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, pairs); break;
        case KB_BF16_DEV_SR: rc = launch_r<__nv_bfloat16, true>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, pairs); break;
        default: return set_error(KB_ERR_UNSUPPORTED, "kb_fused_trt_step_3d: unknown dtype %d", dtype);
    }
    if (rc != KB_OK) return rc;
    return check_launch("kb_fused_trt_step_3d");
}

// The side stream of a cut-link step (declared beside LinkTable3).
SideStream *side_stream() {
    static std::mutex mu;
    static SideStream per_dev[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    SideStream &ss = per_dev[dev];
    if (!ss.ok) {
        if (cudaStreamCreateWithFlags(&ss.side, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ss.join, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        ss.ok = true;
    }
    return &ss;
}

template <typename R, bool SR>
static int launch_links_r(void *f_out, const void *f_in, float *rho, float *ux, float *uy,
                          float *uz, const LinkTable3 &L, const Grid3 &g, float sp, float sm,
                          cudaStream_t s, int variant) {
    // the staged row tiles with the table (16-bit storages, under the rules
    // of the plain step; the class-byte map needs a 16-byte row pitch:
    // Nx % 16 == 0), else adjacent node pairs with vector accesses (even Nx),
    // else one node per thread (odd Nx, or variant 1).  The first two leave
    // the cut nodes to trt_dev_cut_k.
    bool staged = false;
    if constexpr (sizeof(R) == 2) {
        const int ntx = (g.Nx + TT - 1) / TT;
        const bool fill = 10 * g.Nx >= 9 * ntx * TT;
        staged = (variant == 5 || variant == 6 || (variant == 0 && fill)) && g.Nx % 16 == 0 &&
                 ((uintptr_t)L.cls & 15) == 0 && tma_eligible(g, f_out, f_in, rho, ux, uy, uz, L.cls);
    }
    const auto al = [](const void *q, uintptr_t n) { return ((uintptr_t)q & (n - 1)) == 0; };
    const bool pairs = !staged && (variant == 0 || variant == 3) && g.Nx % 2 == 0 &&
                       al(f_out, 2 * sizeof(R)) && al(f_in, 2 * sizeof(R)) && al(rho, 8) &&
                       al(ux, 8) && al(uy, 8) && al(uz, 8) && al(L.cls, 2);
    const bool i32 = offsets_fit_int(g, 19);
    R *fo = (R *)f_out;
    const R *fi = (const R *)f_in;
    if (staged || pairs) {
        // the cut nodes on the side stream (forked from s, joined back
        // before anything that follows on s), or on s itself
        SideStream *ss = L.n_rec > 0 ? side_stream() : nullptr;
        cudaStream_t cs = s;
        if (ss && cudaEventRecord(ss->fork, s) == cudaSuccess &&
            cudaStreamWaitEvent(ss->side, ss->fork, 0) == cudaSuccess)
            cs = ss->side;
        else
            cudaGetLastError();
        if (L.n_rec > 0) {
            const unsigned nb = (unsigned)((L.n_rec + BX - 1) / BX);
            if (i32) {
                if (rho) trt_dev_cut_k<R, true, int, SR><<<nb, BX, 0, cs>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
                else trt_dev_cut_k<R, false, int, SR><<<nb, BX, 0, cs>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
            } else {
                if (rho) trt_dev_cut_k<R, true, long long, SR><<<nb, BX, 0, cs>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
                else trt_dev_cut_k<R, false, long long, SR><<<nb, BX, 0, cs>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
            }
        }
        int rc = KB_OK;
        if (staged) {
            if constexpr (sizeof(R) == 2) {
                const int ty = variant == 6 ? 1 : 0;  // 6: one-row tiles
                rc = i32 ? launch_tma<R, int, SR>(f_out, f_in, rho, ux, uy, uz, nullptr, g, sp, sm, s, &L, ty)
                         : launch_tma<R, long long, SR>(f_out, f_in, rho, ux, uy, uz, nullptr, g, sp, sm, s, &L, ty);
            }
        } else {
            const dim3 grid((g.Nx / 2 + BX - 1) / BX, g.Ny, g.Nz);
            if (i32) {
                if (rho) trt_dev_v2_k<R, true, false, int, SR, true><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, L.cls, g, sp, sm);
                else trt_dev_v2_k<R, false, false, int, SR, true><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, L.cls, g, sp, sm);
            } else {
                if (rho) trt_dev_v2_k<R, true, false, long long, SR, true><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, L.cls, g, sp, sm);
                else trt_dev_v2_k<R, false, false, long long, SR, true><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, L.cls, g, sp, sm);
            }
        }
        if (cs != s && (cudaEventRecord(ss->join, cs) != cudaSuccess ||
                        cudaStreamWaitEvent(s, ss->join, 0) != cudaSuccess))
            return set_error(KB_ERR_CUDA, "kb_fused_trt_libb_links_step_3d: joining the cut-node stream failed");
        if (rc != KB_OK) return rc;
        if (SR) sr_advance_k<<<1, 1, 0, s>>>();
        return KB_OK;
    }
    const dim3 grid((g.Nx + BX - 1) / BX, g.Ny, g.Nz);
    if (i32) {
        if (rho) trt_dev_links_k<R, true, int, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
        else trt_dev_links_k<R, false, int, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
    } else {
        if (rho) trt_dev_links_k<R, true, long long, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
        else trt_dev_links_k<R, false, long long, SR><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
    }
    if (SR) sr_advance_k<<<1, 1, 0, s>>>();
    return KB_OK;
}

int launch_trt3d_dev_links(int dtype, void *f_out, const void *f_in, float *rho, float *ux,
                           float *uy, float *uz, const LinkTable3 &L, const Grid3 &g, float sp,
                           float sm, cudaStream_t s, int variant) {
    int rc = KB_OK;
    switch (dtype) {
        case KB_F32_DEV: rc = launch_links_r<float, false>(f_out, f_in, rho, ux, uy, uz, L, g, sp, sm, s, variant); break;
        case KB_F16_DEV: rc = launch_links_r<__half, false>(f_out, f_in, rho, ux, uy, uz, L, g, sp, sm, s, variant); break;
        case KB_BF16_DEV: rc = launch_links_r<__nv_bfloat16, false>(f_out, f_in, rho, ux, uy, uz, L, g, sp, sm, s, variant); break;
        case KB_F16_DEV_SR: rc = launch_links_r<__half, true>(f_out, f_in, rho, ux, uy, uz, L, g, sp, sm, s, variant); break;
        case KB_BF16_DEV_SR: rc = launch_links_r<__nv_bfloat16, true>(f_out, f_in, rho, ux, uy, uz, L, g, sp, sm, s, variant); break;
        default: return set_error(KB_ERR_UNSUPPORTED, "kb_fused_trt_libb_links_step_3d: unknown dtype %d", dtype);
    }
    if (rc != KB_OK) return rc;
    return check_launch("kb_fused_trt_libb_links_step_3d");
}

// ---------------------------------------------------------------------------
// Thermal DDF natural convection on deviation storage: the fused step of
// src/kernels/fused_thermal_2d.jl:37-151, 178-238 (pull with half-way
// bounce-back of f and g, anti-bounce-back hot west / cold east walls for g,
// temperature, Boussinesq force fy = beta_g (T - T_ref), thermal BGK of g,
// Guo-forced BGK of f) with f stored as d = f - w_q and g as
// e = g - w_q T_ref, and every step computed in FP32 on those deviations:
//   T = T_ref + sum e,   fy = beta_g sum e,   rho = 1 + sum d,
//   u = (sum c d + (0, fy / 2)) / rho
//   e* = e - wT (e - w (dT + 3 T c.u))                 [g_eq - w T_ref]
//   d* = d - w_f (d - w (drho + rho (3 c.u + 4.5 (c.u)^2 - 1.5 u^2)))
//        + (1 - w_f / 2) S_q                            [f_eq - w]
//   anti-bounce-back: e_q = -e_qb + 2 w_q (T_wall - T_ref)
// so neither the O(w) background of f nor the w T_ref background of g is
// rounded.  D2Q9 order: 0 rest, 1 +x, 2 +y, 3 -x, 4 -y, 5 +x+y, 6 -x+y,
// 7 -x-y, 8 +x-y.  VT: the temperature-dependent viscosity of
// fused_natconv_vt_step! (nu = nu_ref exp(a (T - T0)), :155-161).
template <typename R, bool VT, bool SR>
__global__ void __launch_bounds__(BX) natconv_dev_k(R *__restrict__ fo, const R *__restrict__ fi,
                                                     R *__restrict__ go, const R *__restrict__ gi,
                                                     float *__restrict__ Temp, int Nx, int Ny,
                                                     float w_f, float w_T, float beta_g,
                                                     float T_ref, float T_hot, float T_cold,
                                                     float nu_ref, float T0_visc, float a_visc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= Nx) return;
    const size_t P = (size_t)Nx * Ny;
    const size_t c = (size_t)i + (size_t)Nx * j;
    const bool w = i > 0, e = i < Nx - 1, s = j > 0, n = j < Ny - 1;
    // pull with half-way bounce-back; source offsets per population (the
    // opposite population of the node itself at a wall)
    const size_t src[9] = {c,
                           w ? c - 1 + 1 * P : c + 3 * P,
                           s ? c - Nx + 2 * P : c + 4 * P,
                           e ? c + 1 + 3 * P : c + 1 * P,
                           n ? c + Nx + 4 * P : c + 2 * P,
                           (w && s) ? c - 1 - Nx + 5 * P : c + 7 * P,
                           (e && s) ? c + 1 - Nx + 6 * P : c + 8 * P,
                           (e && n) ? c + 1 + Nx + 7 * P : c + 5 * P,
                           (w && n) ? c - 1 + Nx + 8 * P : c + 6 * P};
    float d[9], t[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        d[q] = Dev<R>::ld(fi[src[q]]);
        t[q] = Dev<R>::ld(gi[src[q]]);
    }
    const float wa = 1.0f / 9.0f, wd = 1.0f / 36.0f;
    if (i == 0) {  // hot wall (thermal_bc, fused_thermal_2d.jl:37-52)
        const float h = 2.0f * (T_hot - T_ref);
        t[1] = -t[1] + wa * h;
        t[5] = -t[5] + wd * h;
        t[8] = -t[8] + wd * h;
    }
    if (i == Nx - 1) {  // cold wall
        const float h = 2.0f * (T_cold - T_ref);
        t[3] = -t[3] + wa * h;
        t[6] = -t[6] + wd * h;
        t[7] = -t[7] + wd * h;
    }
    const float dT = ((t[0] + t[1]) + (t[2] + t[3])) + ((t[4] + t[5]) + ((t[6] + t[7]) + t[8]));
    const float Tl = T_ref + dT;
    Temp[c] = Tl;
    const float fy = beta_g * dT;
    const float drho = ((d[0] + d[1]) + (d[2] + d[3])) + ((d[4] + d[5]) + ((d[6] + d[7]) + d[8]));
    const float rho = 1.0f + drho;
    const float inv = vrcp_fast(rho);
    const float ux = (((d[1] - d[3]) + (d[5] - d[6])) + (d[8] - d[7])) * inv;
    const float uy = ((((d[2] - d[4]) + (d[5] + d[6])) - (d[7] + d[8])) + 0.5f * fy) * inv;
    // velocity projections c_q . u
    const float cu[9] = {0.f, ux, uy, -ux, -uy, ux + uy, uy - ux, -ux - uy, ux - uy};
    const float wq[9] = {4.0f / 9.0f, wa, wa, wa, wa, wd, wd, wd, wd};
    // thermal BGK on e
    float eo[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const float eeq = wq[q] * fmaf(3.0f * Tl, cu[q], dT);
        eo[q] = t[q] - w_T * (t[q] - eeq);
    }
    float wf = w_f;
    if (VT) wf = 1.0f / (3.0f * (nu_ref * expf(a_visc * (Tl - T0_visc))) + 0.5f);
    // Guo-forced BGK on d (collide_guo with fx = 0): the source
    // S_q = w_q (3 (c_q - u) . F + 9 (c_q . u)(c_q . F)), F = (0, fy)
    const float usq15 = 1.5f * fmaf(ux, ux, uy * uy);
    const float cy[9] = {0.f, 0.f, 1.f, 0.f, -1.f, 1.f, 1.f, -1.f, -1.f};
    const float gsrc = 1.0f - 0.5f * wf;
    float dout[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const float deq = wq[q] * fmaf(rho, fmaf(cu[q], fmaf(4.5f, cu[q], 3.0f), -usq15), drho);
        const float S = wq[q] * fy * fmaf(9.0f * cu[q], cy[q], 3.0f * (cy[q] - uy));
        dout[q] = d[q] - wf * (d[q] - deq) + gsrc * S;
    }
    if (SR) {
        const uint32_t key =
            hash32((uint32_t)c ^ hash32(*(volatile const unsigned int *)&g_sr_epoch + 0x632BE5ABu));
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const uint32_t v = SRPack<R>::pack(dout[q], eo[q], sr_bits(key, q));
            reinterpret_cast<unsigned short *>(fo)[c + q * P] = (unsigned short)(v & 0xFFFFu);
            reinterpret_cast<unsigned short *>(go)[c + q * P] = (unsigned short)(v >> 16);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            fo[c + q * P] = Dev<R>::st(dout[q]);
            go[c + q * P] = Dev<R>::st(eo[q]);
        }
    }
}

template <typename R, bool SR>
static void launch_natconv_dev_r(bool vt, void *f_out, const void *f_in, void *g_out,
                                 const void *g_in, float *Temp, int Nx, int Ny, float w_f,
                                 float w_T, float beta_g, float T_ref, float T_hot, float T_cold,
                                 float nu_ref, float T0_visc, float a_visc, cudaStream_t s) {
    const dim3 grid((Nx + BX - 1) / BX, Ny);
    R *fo = (R *)f_out, *go = (R *)g_out;
    const R *fi = (const R *)f_in, *gi = (const R *)g_in;
    if (vt)
        natconv_dev_k<R, true, SR><<<grid, BX, 0, s>>>(fo, fi, go, gi, Temp, Nx, Ny, w_f, w_T, beta_g,
                                                      T_ref, T_hot, T_cold, nu_ref, T0_visc, a_visc);
    else
        natconv_dev_k<R, false, SR><<<grid, BX, 0, s>>>(fo, fi, go, gi, Temp, Nx, Ny, w_f, w_T, beta_g,
                                                       T_ref, T_hot, T_cold, nu_ref, T0_visc, a_visc);
    if (SR) sr_advance_k<<<1, 1, 0, s>>>();
}

int launch_natconv_dev(int dtype, bool vt, void *f_out, const void *f_in, void *g_out,
                       const void *g_in, float *Temp, int Nx, int Ny, double w_f, double w_T,
                       double beta_g, double T_ref, double T_hot, double T_cold, double nu_ref,
                       double T0_visc, double a_visc, cudaStream_t s) {
    const float a[10] = {(float)w_f, (float)w_T, (float)beta_g, (float)T_ref, (float)T_hot,
                         (float)T_cold, (float)nu_ref, (float)T0_visc, (float)a_visc, 0.f};
#define KB_NATCONV_DEV(R, SR)                                                                   \
    launch_natconv_dev_r<R, SR>(vt, f_out, f_in, g_out, g_in, Temp, Nx, Ny, a[0], a[1], a[2], a[3], \
                                a[4], a[5], a[6], a[7], a[8], s)
    switch (dtype) {
        case KB_F32_DEV: KB_NATCONV_DEV(float, false); break;
        case KB_F16_DEV: KB_NATCONV_DEV(__half, false); break;
        case KB_BF16_DEV: KB_NATCONV_DEV(__nv_bfloat16, false); break;
        case KB_F16_DEV_SR: KB_NATCONV_DEV(__half, true); break;
        case KB_BF16_DEV_SR: KB_NATCONV_DEV(__nv_bfloat16, true); break;
        default:
            return set_error(KB_ERR_UNSUPPORTED, "kb_fused_natconv_step: unknown dtype %d", dtype);
    }
#undef KB_NATCONV_DEV
    return check_launch("kb_fused_natconv_step");
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
    const unsigned int zero = 0u;
    if (cudaMemcpyToSymbolAsync(kb::d3::g_sr_epoch, &seed, sizeof(seed), 0, cudaMemcpyHostToDevice,
                                kb::as_stream(stream)) != cudaSuccess ||
        cudaMemcpyToSymbolAsync(kb::d3::g_sr_done, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice,
                                kb::as_stream(stream)) != cudaSuccess)
        return kb::check_launch("kb_set_stochastic_seed");
    // the host value must outlive the asynchronous copy
    if (cudaStreamSynchronize(kb::as_stream(stream)) != cudaSuccess)
        return kb::check_launch("kb_set_stochastic_seed");
    return 0;
}

extern "C" int kb_get_stochastic_seed(unsigned int *seed, void *stream) {
    KB_REQUIRE(seed, "kb_get_stochastic_seed: null argument");
    unsigned int v = 0u;
    if (cudaMemcpyFromSymbolAsync(&v, kb::d3::g_sr_epoch, sizeof(v), 0, cudaMemcpyDeviceToHost,
                                  kb::as_stream(stream)) != cudaSuccess ||
        cudaStreamSynchronize(kb::as_stream(stream)) != cudaSuccess)
        return kb::check_launch("kb_get_stochastic_seed");
    *seed = v;
    return 0;
}

extern "C" int kb_staged_step_status(int *timed_out, void *stream) {
    KB_REQUIRE(timed_out, "kb_staged_step_status: null argument");
    cudaStream_t s = kb::as_stream(stream);
    int v = 0;
    if (cudaMemcpyFromSymbolAsync(&v, kb::d3::g_tma_timeout, sizeof(int), 0, cudaMemcpyDeviceToHost,
                                  s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return kb::check_launch("kb_staged_step_status");
    if (v) {
        const int zero = 0;
        if (cudaMemcpyToSymbolAsync(kb::d3::g_tma_timeout, &zero, sizeof(int), 0,
                                    cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return kb::check_launch("kb_staged_step_status");
    }
    *timed_out = v;
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
