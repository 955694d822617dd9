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

// Opposite pairs (q, qb) of D3Q19; c_qb = -c_q.  Indexed only with
// compile-time constants (fully unrolled loops), so d[] stays in registers.
__device__ constexpr int kPairQ[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16};
__device__ constexpr int kPairQb[9] = {2, 4, 6, 10, 9, 14, 13, 18, 17};

template <typename R, bool MOM, bool SOLID>
__global__ void __launch_bounds__(BX) trt_dev_k(R *__restrict__ fo, const R *__restrict__ fi,
                                                 float *__restrict__ rho_o, float *__restrict__ ux_o,
                                                 float *__restrict__ uy_o, float *__restrict__ uz_o,
                                                 const uint8_t *__restrict__ solid, Grid3 g,
                                                 float sp, float sm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= g.Nx) return;
    const size_t c = (size_t)i + (size_t)g.Nx * ((size_t)j + (size_t)g.Ny * k);
    const size_t P = g.plane;
    if (SOLID && solid[c]) {
#pragma unroll
        for (int q = 0; q < 19; ++q) fo[c + q * P] = Dev<R>::st(0.0f);
        if (MOM) { rho_o[c] = 1.0f; ux_o[c] = 0.0f; uy_o[c] = 0.0f; uz_o[c] = 0.0f; }
        return;
    }
    float d[19];
    pull19(fi, P, c, pull_geometry(g, i, j, k), d, DevLoad<R>());

    float drho = 0.f;
#pragma unroll
    for (int q = 0; q < 19; ++q) drho += d[q];
    const float jx = (d[1] - d[2]) + (d[7] - d[8]) + (d[9] - d[10]) + (d[11] - d[12]) + (d[13] - d[14]);
    const float jy = (d[3] - d[4]) + (d[7] + d[8]) - (d[9] + d[10]) + (d[15] - d[16]) + (d[17] - d[18]);
    const float jz = (d[5] - d[6]) + (d[11] + d[12]) - (d[13] + d[14]) + (d[15] + d[16]) - (d[17] + d[18]);
    const float rho = 1.0f + drho;
    const float inv = 1.0f / rho;
    const float ux = jx * inv, uy = jy * inv, uz = jz * inv;
    const float usq15 = 1.5f * (ux * ux + uy * uy + uz * uz);

    // rest population: only the even mode
    const float w0 = float(1.0 / 3.0);
    const float deq0 = w0 * (drho - rho * usq15);
    fo[c] = Dev<R>::st(d[0] - sp * (d[0] - deq0));

#pragma unroll
    for (int m = 0; m < 9; ++m) {
        const int q = kPairQ[m], qb = kPairQb[m];
        const float w = m < 3 ? float(1.0 / 18.0) : float(1.0 / 36.0);
        const float cu = float(cx19(q)) * ux + float(cy19(q)) * uy + float(cz19(q)) * uz;
        const float deq_p = w * (drho + rho * (4.5f * cu * cu - usq15));
        const float deq_m = w * rho * 3.0f * cu;
        const float dq = d[q], dqb = d[qb];
        const float np = 0.5f * (dq + dqb) - deq_p;
        const float nm = 0.5f * (dq - dqb) - deq_m;
        const float even = sp * np, odd = sm * nm;
        fo[c + q * P] = Dev<R>::st(dq - even - odd);
        fo[c + qb * P] = Dev<R>::st(dqb - even + odd);
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

template <typename R, bool MOM, bool SOLID>
__global__ void __launch_bounds__(BX) trt_dev_x2_k(R *__restrict__ fo, const R *__restrict__ fi,
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
    const size_t P = g.plane;
    const size_t row = (size_t)g.Nx * ((size_t)j + (size_t)g.Ny * k);
    const size_t cA = row + iA, cB = row + (vB ? iB : iA);
    float a[19], b[19];
    pull19(fi, P, cA, pull_geometry(g, iA, j, k), a, DevLoad<R>());
    pull19(fi, P, cB, pull_geometry(g, vB ? iB : iA, j, k), b, DevLoad<R>());
    float2 d[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) d[q] = make_float2(a[q], b[q]);

    float2 drho = d[0];
#pragma unroll
    for (int q = 1; q < 19; ++q) drho = add2(drho, d[q]);
    const float2 jx = add2(add2(add2(sub2(d[1], d[2]), sub2(d[7], d[8])), add2(sub2(d[9], d[10]), sub2(d[11], d[12]))), sub2(d[13], d[14]));
    const float2 jy = add2(add2(add2(sub2(d[3], d[4]), add2(d[7], d[8])), sub2(add2(d[15], d[17]), add2(d[9], d[10]))), sub2(sub2(f2(0.f), d[16]), d[18]));
    const float2 jz = add2(add2(add2(sub2(d[5], d[6]), add2(d[11], d[12])), sub2(add2(d[15], d[16]), add2(d[13], d[14]))), sub2(sub2(f2(0.f), d[17]), d[18]));
    const float2 rho = add2(f2(1.0f), drho);
    const float2 inv = make_float2(__frcp_rn(rho.x), __frcp_rn(rho.y));
    const float2 ux = mul2(jx, inv), uy = mul2(jy, inv), uz = mul2(jz, inv);
    const float2 usq15 = mul2(f2(1.5f), fma2(ux, ux, fma2(uy, uy, mul2(uz, uz))));
    const float2 vsp = f2(sp), vsm = f2(sm);
    uchar2 sm2 = make_uchar2(0, 0);
    if (SOLID) sm2 = make_uchar2(solid[cA], vB ? solid[cB] : 0);
    float2 o[19];
    {
        const float2 deq0 = mul2(f2(float(1.0 / 3.0)), sub2(drho, mul2(rho, usq15)));
        o[0] = sub2(d[0], mul2(vsp, sub2(d[0], deq0)));
    }
#pragma unroll
    for (int m = 0; m < 9; ++m) {
        const int q = kPairQ[m], qb = kPairQb[m];
        const float w = m < 3 ? float(1.0 / 18.0) : float(1.0 / 36.0);
        float2 cu = f2(0.f);
        if (cx19(q) == 1) cu = add2(cu, ux); else if (cx19(q) == -1) cu = sub2(cu, ux);
        if (cy19(q) == 1) cu = add2(cu, uy); else if (cy19(q) == -1) cu = sub2(cu, uy);
        if (cz19(q) == 1) cu = add2(cu, uz); else if (cz19(q) == -1) cu = sub2(cu, uz);
        const float2 deq_p = mul2(f2(w), fma2(rho, fma2(mul2(f2(4.5f), cu), cu, make_float2(-usq15.x, -usq15.y)), drho));
        const float2 deq_m = mul2(mul2(f2(3.0f * w), rho), cu);
        const float2 np = fma2(f2(0.5f), add2(d[q], d[qb]), make_float2(-deq_p.x, -deq_p.y));
        const float2 nm = fma2(f2(0.5f), sub2(d[q], d[qb]), make_float2(-deq_m.x, -deq_m.y));
        const float2 ev = mul2(vsp, np), od = mul2(vsm, nm);
        o[q] = sub2(sub2(d[q], ev), od);
        o[qb] = add2(sub2(d[qb], ev), od);
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        fo[cA + q * P] = Dev<R>::st(SOLID && sm2.x ? 0.f : o[q].x);
        if (vB) fo[cB + q * P] = Dev<R>::st(SOLID && sm2.y ? 0.f : o[q].y);
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

template <typename R>
static void launch_r(void *f_out, const void *f_in, float *rho, float *ux, float *uy, float *uz,
                     const uint8_t *solid, const Grid3 &g, float sp, float sm, cudaStream_t s,
                     bool pairs) {
    R *fo = (R *)f_out;
    const R *fi = (const R *)f_in;
    if (pairs) {
        const int threads_x = (g.Nx + 63) / 64 * 32;  // one warp per 64 nodes of a row
        const dim3 grid((threads_x + BX - 1) / BX, g.Ny, g.Nz);
        if (rho) {
            if (solid) trt_dev_x2_k<R, true, true><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
            else trt_dev_x2_k<R, true, false><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
        } else {
            if (solid) trt_dev_x2_k<R, false, true><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
            else trt_dev_x2_k<R, false, false><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
        }
        return;
    }
    const dim3 grid = nodes_grid(g.Nx, g.Ny, g.Nz);
    if (rho) {
        if (solid) trt_dev_k<R, true, true><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
        else trt_dev_k<R, true, false><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
    } else {
        if (solid) trt_dev_k<R, false, true><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
        else trt_dev_k<R, false, false><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, solid, g, sp, sm);
    }
}

int launch_trt3d_dev(int dtype, void *f_out, const void *f_in, float *rho, float *ux, float *uy,
                     float *uz, const uint8_t *solid, const Grid3 &g, float sp, float sm,
                     cudaStream_t s, int variant) {
    // variant: 0 automatic (two nodes per thread for 16-bit storages when a
    // row holds at least 64 nodes), 1 one node per thread, 2 two nodes per
    // thread
    const bool pairs = variant == 2 ||
                       (variant == 0 && dtype != KB_F32_DEV && g.Nx >= 64);
    switch (dtype) {
        case KB_F32_DEV: launch_r<float>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, pairs); break;
        case KB_F16_DEV: launch_r<__half>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, pairs); break;
        case KB_BF16_DEV: launch_r<__nv_bfloat16>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s, pairs); break;
        default: return set_error(KB_ERR_UNSUPPORTED, "kb_fused_trt_step_3d: unknown dtype %d", dtype);
    }
    return check_launch("kb_fused_trt_step_3d");
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
