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

// Pair table: (q, qb) and the velocity of q.
struct PairC {
    int q, qb, cx, cy, cz;
};
__device__ __constant__ PairC kPairs[9] = {
    {1, 2, 1, 0, 0},    {3, 4, 0, 1, 0},    {5, 6, 0, 0, 1},
    {7, 10, 1, 1, 0},   {8, 9, -1, 1, 0},   {11, 14, 1, 0, 1},
    {12, 13, -1, 0, 1}, {15, 18, 0, 1, 1},  {16, 17, 0, -1, 1},
};

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
        const PairC pc = kPairs[m];
        const float w = m < 3 ? float(1.0 / 18.0) : float(1.0 / 36.0);
        const float cu = float(pc.cx) * ux + float(pc.cy) * uy + float(pc.cz) * uz;
        const float deq_p = w * (drho + rho * (4.5f * cu * cu - usq15));
        const float deq_m = w * rho * 3.0f * cu;
        const float dq = d[pc.q], dqb = d[pc.qb];
        const float np = 0.5f * (dq + dqb) - deq_p;
        const float nm = 0.5f * (dq - dqb) - deq_m;
        const float even = sp * np, odd = sm * nm;
        fo[c + pc.q * P] = Dev<R>::st(dq - even - odd);
        fo[c + pc.qb * P] = Dev<R>::st(dqb - even + odd);
    }
    if (MOM) { rho_o[c] = rho; ux_o[c] = ux; uy_o[c] = uy; uz_o[c] = uz; }
}

template <typename R>
static void launch_r(void *f_out, const void *f_in, float *rho, float *ux, float *uy, float *uz,
                     const uint8_t *solid, const Grid3 &g, float sp, float sm, cudaStream_t s) {
    const dim3 grid = nodes_grid(g.Nx, g.Ny, g.Nz);
    R *fo = (R *)f_out;
    const R *fi = (const R *)f_in;
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
                     cudaStream_t s) {
    switch (dtype) {
        case KB_F32_DEV: launch_r<float>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s); break;
        case KB_F16_DEV: launch_r<__half>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s); break;
        case KB_BF16_DEV: launch_r<__nv_bfloat16>(f_out, f_in, rho, ux, uy, uz, solid, g, sp, sm, s); break;
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
