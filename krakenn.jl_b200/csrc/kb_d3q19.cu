// kb_d3q19.cu -- D3Q19 kernels with the reference's arithmetic.
//
// Compiled with --fmad=false so double (float) runs round exactly as the
// reference's CPU Float64 (Float32) path.  The deviation-storage variants of
// the fused TRT step live in kb_d3q19_dev.cu.
#include <vector>

#include "kb_d3q19.cuh"

namespace kb {
namespace d3 {

template <typename T>
__device__ __forceinline__ T feq_poly(T w, T rho, T cu, T usq) {
    return w * rho * (T(1) + T(3) * cu + T(4.5) * cu * cu - T(1.5) * usq);
}

// feq_3d: src/kernels/equilibrium_helpers_3d.jl:26-100 (the same expressions
// as collide_3d_kernel!, collide_stream_3d.jl:76-100).
template <typename T>
__device__ __forceinline__ void feq_all(T rho, T ux, T uy, T uz, T usq, T *feq) {
    const T wr = T(1.0 / 3.0), wa = T(1.0 / 18.0), we = T(1.0 / 36.0);
    feq[0] = wr * rho * (T(1) - T(1.5) * usq);
    feq[1] = feq_poly(wa, rho, ux, usq);
    feq[2] = feq_poly(wa, rho, -ux, usq);
    feq[3] = feq_poly(wa, rho, uy, usq);
    feq[4] = feq_poly(wa, rho, -uy, usq);
    feq[5] = feq_poly(wa, rho, uz, usq);
    feq[6] = feq_poly(wa, rho, -uz, usq);
    feq[7] = feq_poly(we, rho, ux + uy, usq);
    feq[8] = feq_poly(we, rho, -ux + uy, usq);
    feq[9] = feq_poly(we, rho, ux - uy, usq);
    feq[10] = feq_poly(we, rho, -ux - uy, usq);
    feq[11] = feq_poly(we, rho, ux + uz, usq);
    feq[12] = feq_poly(we, rho, -ux + uz, usq);
    feq[13] = feq_poly(we, rho, ux - uz, usq);
    feq[14] = feq_poly(we, rho, -ux - uz, usq);
    feq[15] = feq_poly(we, rho, uy + uz, usq);
    feq[16] = feq_poly(we, rho, -uy + uz, usq);
    feq[17] = feq_poly(we, rho, uy - uz, usq);
    feq[18] = feq_poly(we, rho, -uy - uz, usq);
}

// moments_3d: src/kernels/equilibrium_helpers_3d.jl:102-112
template <typename T>
__device__ __forceinline__ void moments(const T *p, T &rho, T &ux, T &uy, T &uz) {
    rho = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8] + p[9] + p[10] + p[11] +
          p[12] + p[13] + p[14] + p[15] + p[16] + p[17] + p[18];
    const T inv = T(1) / rho;
    ux = (p[1] - p[2] + p[7] - p[8] + p[9] - p[10] + p[11] - p[12] + p[13] - p[14]) * inv;
    uy = (p[3] - p[4] + p[7] + p[8] - p[9] - p[10] + p[15] - p[16] + p[17] - p[18]) * inv;
    uz = (p[5] - p[6] + p[11] + p[12] - p[13] - p[14] + p[15] + p[16] - p[17] - p[18]) * inv;
}

template <typename T>
__device__ __forceinline__ void swap_pairs(T *p) {
    const int a[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16};
    const int b[9] = {2, 4, 6, 10, 9, 14, 13, 18, 17};
#pragma unroll
    for (int n = 0; n < 9; ++n) { T t = p[a[n]]; p[a[n]] = p[b[n]]; p[b[n]] = t; }
}

struct Ident {
    template <typename V> __device__ __forceinline__ V operator()(V v) const { return v; }
};

#define NODE3                                                     \
    const int i = blockIdx.x * blockDim.x + threadIdx.x;          \
    const int j = blockIdx.y, k = blockIdx.z;                     \
    if (i >= g.Nx) return;                                        \
    const size_t c = (size_t)i + (size_t)g.Nx * ((size_t)j + (size_t)g.Ny * k); \
    const size_t P = g.plane;

// stream_3d_kernel!: src/kernels/collide_stream_3d.jl:5-42
template <typename T>
__global__ void __launch_bounds__(BX) stream_k(T *__restrict__ fo, const T *__restrict__ fi, Grid3 g) {
    NODE3
    T p[19];
    pull19(fi, P, c, pull_geometry(g, i, j, k), p, Ident());
#pragma unroll
    for (int q = 0; q < 19; ++q) fo[c + q * P] = p[q];
}

// collide_3d_kernel!: src/kernels/collide_stream_3d.jl:46-103
template <typename T>
__global__ void __launch_bounds__(BX) collide_k(T *__restrict__ f, const uint8_t *__restrict__ solid,
                                                 Grid3 g, T omega) {
    NODE3
    T p[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) p[q] = f[c + q * P];
    if (solid && solid[c]) {
        swap_pairs(p);
    } else {
        T rho, ux, uy, uz, feq[19];
        moments(p, rho, ux, uy, uz);
        const T usq = ux * ux + uy * uy + uz * uz;
        feq_all(rho, ux, uy, uz, usq, feq);
#pragma unroll
        for (int q = 0; q < 19; ++q) p[q] = p[q] - omega * (p[q] - feq[q]);
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) f[c + q * P] = p[q];
}

// compute_macroscopic_3d_kernel!: src/kernels/macroscopic.jl:42-61
template <typename T>
__global__ void __launch_bounds__(BX) macroscopic_k(T *__restrict__ rho, T *__restrict__ ux,
                                                     T *__restrict__ uy, T *__restrict__ uz,
                                                     const T *__restrict__ f, Grid3 g) {
    NODE3
    T p[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) p[q] = f[c + q * P];
    T r, a, b, d;
    moments(p, r, a, b, d);
    rho[c] = r; ux[c] = a; uy[c] = b; uz[c] = d;
}

// compute_macroscopic_forced_3d_kernel! (src/kernels/macroscopic.jl:121-141;
// FIELD false, constant force) and compute_macroscopic_forced_field_3d_kernel!
// (:164-192; FIELD true, per-node force).
template <typename T, bool FIELD>
__global__ void __launch_bounds__(BX) macroscopic_forced_k(T *__restrict__ rho, T *__restrict__ ux,
                                                            T *__restrict__ uy, T *__restrict__ uz,
                                                            const T *__restrict__ f, Grid3 g,
                                                            T Fx, T Fy, T Fz,
                                                            const T *__restrict__ Fxf,
                                                            const T *__restrict__ Fyf,
                                                            const T *__restrict__ Fzf) {
    NODE3
    T p[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) p[q] = f[c + q * P];
    T r = p[0];
#pragma unroll
    for (int q = 1; q < 19; ++q) r = r + p[q];
    const T inv = T(1) / r;
    const T fx = FIELD ? Fxf[c] : Fx, fy = FIELD ? Fyf[c] : Fy, fz = FIELD ? Fzf[c] : Fz;
    rho[c] = r;
    ux[c] = ((p[1] - p[2] + p[7] - p[8] + p[9] - p[10] + p[11] - p[12] + p[13] - p[14]) + fx / T(2)) * inv;
    uy[c] = ((p[3] - p[4] + p[7] + p[8] - p[9] - p[10] + p[15] - p[16] + p[17] - p[18]) + fy / T(2)) * inv;
    uz[c] = ((p[5] - p[6] + p[11] + p[12] - p[13] - p[14] + p[15] + p[16] - p[17] - p[18]) + fz / T(2)) * inv;
}

// Fused TRT step with the reference arithmetic (PullHalfwayBB_3D +
// SolidInert_3D + Moments_3D + CollideTRTDirect_3D + WriteMoments_3D,
// src/kernels/dsl/bricks_3d.jl:64-230, 476-483).  I: element-offset type.
template <typename T, typename I>
__global__ void __launch_bounds__(BX) fused_trt_k(T *__restrict__ fo, const T *__restrict__ fi,
                                                   T *__restrict__ rho, T *__restrict__ ux,
                                                   T *__restrict__ uy, T *__restrict__ uz,
                                                   const uint8_t *__restrict__ solid, Grid3 g, T sp,
                                                   T sm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= g.Nx) return;
    const size_t c = (size_t)i + (size_t)g.Nx * ((size_t)j + (size_t)g.Ny * k);
    const I P = (I)g.plane;
    T *__restrict__ o0 = fo + c;
    T p[19];
    pull19_at(fi + c, P, pull_geometry<I>(g, i, j, k), p, Ident());
    if (solid && solid[c]) {
        T feq[19];
        feq_all(T(1), T(0), T(0), T(0), T(0), feq);
#pragma unroll
        for (int q = 0; q < 19; ++q) o0[q * P] = feq[q];
        if (rho) { rho[c] = T(1); ux[c] = T(0); uy[c] = T(0); uz[c] = T(0); }
        return;
    }
    T r, a_, b_, d_, feq[19];
    moments(p, r, a_, b_, d_);
    const T usq = a_ * a_ + b_ * b_ + d_ * d_;
    feq_all(r, a_, b_, d_, usq, feq);
    const T a = (sp + sm) * T(0.5), b = (sp - sm) * T(0.5);
    const int pa[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16};
    const int pb[9] = {2, 4, 6, 10, 9, 14, 13, 18, 17};
    o0[0] = p[0] - sp * (p[0] - feq[0]);
#pragma unroll
    for (int m = 0; m < 9; ++m) {
        const int x = pa[m], y = pb[m];
        o0[x * P] = p[x] - a * (p[x] - feq[x]) - b * (p[y] - feq[y]);
        o0[y * P] = p[y] - a * (p[y] - feq[y]) - b * (p[x] - feq[x]);
    }
    if (rho) { rho[c] = r; ux[c] = a_; uy[c] = b_; uz[c] = d_; }
}

// fused_trt_libb_v2_step_3d! (src/kernels/li_bb_3d_v2.jl:13-42): the fused
// TRT step above with ApplyLiBBPrePhase_3D on fluid nodes.
template <typename T, typename I>
__global__ void __launch_bounds__(BX) fused_trt_libb_k(T *__restrict__ fo, const T *__restrict__ fi,
                                                        T *__restrict__ rho, T *__restrict__ ux,
                                                        T *__restrict__ uy, T *__restrict__ uz,
                                                        const uint8_t *__restrict__ solid,
                                                        const T *__restrict__ qw,
                                                        const T *__restrict__ wx,
                                                        const T *__restrict__ wy,
                                                        const T *__restrict__ wz, Grid3 g, T sp,
                                                        T sm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= g.Nx) return;
    const size_t c = (size_t)i + (size_t)g.Nx * ((size_t)j + (size_t)g.Ny * k);
    const I P = (I)g.plane;
    T *__restrict__ o0 = fo + c;
    T feq[19];
    if (solid && solid[c]) {
        feq_all(T(1), T(0), T(0), T(0), T(0), feq);
#pragma unroll
        for (int q = 0; q < 19; ++q) o0[q * P] = feq[q];
        if (rho) { rho[c] = T(1); ux[c] = T(0); uy[c] = T(0); uz[c] = T(0); }
        return;
    }
    T p[19];
    pull19_at(fi + c, P, pull_geometry<I>(g, i, j, k), p, Ident());
    libb_prephase_3d(fi + c, P, LinkDense<T, I>{qw + c, wx + c, wy + c, wz + c, P}, p);
    T r, a_, b_, d_;
    moments(p, r, a_, b_, d_);
    const T usq = a_ * a_ + b_ * b_ + d_ * d_;
    feq_all(r, a_, b_, d_, usq, feq);
    const T a = (sp + sm) * T(0.5), b = (sp - sm) * T(0.5);
    const int pa[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16};
    const int pb[9] = {2, 4, 6, 10, 9, 14, 13, 18, 17};
    o0[0] = p[0] - sp * (p[0] - feq[0]);
#pragma unroll
    for (int m = 0; m < 9; ++m) {
        const int x = pa[m], y = pb[m];
        o0[x * P] = p[x] - a * (p[x] - feq[x]) - b * (p[y] - feq[y]);
        o0[y * P] = p[y] - a * (p[y] - feq[y]) - b * (p[x] - feq[x]);
    }
    if (rho) { rho[c] = r; ux[c] = a_; uy[c] = b_; uz[c] = d_; }
}

// The same step with the compact cut-link table: one class byte per node
// replaces the solid mask and the 18 q_wall reads; link data are read only
// at nodes with cut links.  Bit-identical to fused_trt_libb_k.  The update
// of node c = (i, j, k) of class cl, shared by the node kernel and the
// cut-node kernel so that both compute the same bits.
template <typename T, typename I>
__device__ __forceinline__ void trt_links_node(T *__restrict__ fo, const T *__restrict__ fi,
                                               T *__restrict__ rho, T *__restrict__ ux,
                                               T *__restrict__ uy, T *__restrict__ uz,
                                               const LinkTable3 &L, const Grid3 &g, T sp, T sm,
                                               size_t c, int i, int j, int k, uint8_t cl) {
    const I P = (I)g.plane;
    T *__restrict__ o0 = fo + c;
    T feq[19];
    if (cl == 1) {
        feq_all(T(1), T(0), T(0), T(0), T(0), feq);
#pragma unroll
        for (int q = 0; q < 19; ++q) o0[q * P] = feq[q];
        if (rho) { rho[c] = T(1); ux[c] = T(0); uy[c] = T(0); uz[c] = T(0); }
        return;
    }
    T p[19];
    pull19_at(fi + c, P, pull_geometry<I>(g, i, j, k), p, Ident());
    if (cl == 2) libb_prephase_3d(fi + c, P, link_record<T>(L, L.rec[c]), p);
    T r, a_, b_, d_;
    moments(p, r, a_, b_, d_);
    const T usq = a_ * a_ + b_ * b_ + d_ * d_;
    feq_all(r, a_, b_, d_, usq, feq);
    const T a = (sp + sm) * T(0.5), b = (sp - sm) * T(0.5);
    const int pa[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16};
    const int pb[9] = {2, 4, 6, 10, 9, 14, 13, 18, 17};
    o0[0] = p[0] - sp * (p[0] - feq[0]);
#pragma unroll
    for (int m = 0; m < 9; ++m) {
        const int x = pa[m], y = pb[m];
        o0[x * P] = p[x] - a * (p[x] - feq[x]) - b * (p[y] - feq[y]);
        o0[y * P] = p[y] - a * (p[y] - feq[y]) - b * (p[x] - feq[x]);
    }
    if (rho) { rho[c] = r; ux[c] = a_; uy[c] = b_; uz[c] = d_; }
}

// SKIP_CUT: class 2 nodes are left to fused_trt_cut_k, which runs beside
// this kernel (the two write disjoint nodes and read only f_in), so this
// kernel carries no link code.
template <typename T, typename I, bool SKIP_CUT>
__global__ void __launch_bounds__(BX) fused_trt_links_k(T *__restrict__ fo, const T *__restrict__ fi,
                                                         T *__restrict__ rho, T *__restrict__ ux,
                                                         T *__restrict__ uy, T *__restrict__ uz,
                                                         LinkTable3 L, Grid3 g, T sp, T sm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= g.Nx) return;
    const size_t c = (size_t)i + (size_t)g.Nx * ((size_t)j + (size_t)g.Ny * k);
    const uint8_t cl = L.cls[c];
    if (SKIP_CUT) {
        if (cl == 2) return;
        trt_links_node<T, I>(fo, fi, rho, ux, uy, uz, L, g, sp, sm, c, i, j, k, cl == 1 ? 1 : 0);
    } else {
        trt_links_node<T, I>(fo, fi, rho, ux, uy, uz, L, g, sp, sm, c, i, j, k, cl);
    }
}

// The cut nodes (class 2) of a compact table, one thread per record.
template <typename T, typename I>
__global__ void __launch_bounds__(BX) fused_trt_cut_k(T *__restrict__ fo, const T *__restrict__ fi,
                                                       T *__restrict__ rho, T *__restrict__ ux,
                                                       T *__restrict__ uy, T *__restrict__ uz,
                                                       LinkTable3 L, Grid3 g, T sp, T sm) {
    const long long r = (long long)blockIdx.x * BX + threadIdx.x;
    if (r >= L.n_rec) return;
    const size_t c = (size_t)L.node[r];
    const size_t row = c / (size_t)g.Nx;
    const int i = (int)(c - row * (size_t)g.Nx), j = (int)(row % (size_t)g.Ny),
              k = (int)(row / (size_t)g.Ny);
    trt_links_node<T, I>(fo, fi, rho, ux, uy, uz, L, g, sp, sm, c, i, j, k, 2);
}

// Cut-link table construction.  Pass 1 classifies every node and counts the
// nodes with cut links per block of LT nodes; the host scans the counts;
// pass 2 ranks the nodes inside each block, so records follow node order.
constexpr int LT = 1024;

template <typename T>
__device__ __forceinline__ uint8_t link_class(const uint8_t *solid, const T *qw, size_t n,
                                              size_t nodes) {
    if (solid && solid[n]) return 1;
    bool any = false;
    for (int q = 1; q < 19; ++q) any |= qw[q * nodes + n] > T(0);
    return any ? 2 : 0;
}

template <typename T>
__global__ void __launch_bounds__(LT) links_count_k(uint8_t *cls, int *counts, const uint8_t *solid,
                                                    const T *qw, size_t nodes) {
    __shared__ int total;
    if (threadIdx.x == 0) total = 0;
    __syncthreads();
    const size_t n = (size_t)blockIdx.x * LT + threadIdx.x;
    int mine = 0;
    if (n < nodes) {
        const uint8_t c = link_class(solid, qw, n, nodes);
        cls[n] = c;
        mine = c == 2;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, mine);
    if ((threadIdx.x & 31) == 0 && bal) atomicAdd(&total, __popc(bal));
    __syncthreads();
    if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

template <typename T>
__global__ void __launch_bounds__(LT) links_fill_k(int *rec, int *node, T *tq, T *tx, T *ty, T *tz,
                                                   const uint8_t *cls, const int *offsets,
                                                   const T *qw, const T *wx, const T *wy,
                                                   const T *wz, size_t nodes, long long n_rec) {
    __shared__ int warp_base[LT / 32];
    const size_t n = (size_t)blockIdx.x * LT + threadIdx.x;
    const int mine = n < nodes && cls[n] == 2;
    const unsigned bal = __ballot_sync(0xffffffffu, mine);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) warp_base[warp] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int w = 0; w < LT / 32; ++w) { const int v = warp_base[w]; warp_base[w] = acc; acc += v; }
    }
    __syncthreads();
    if (!mine) return;
    const long long r = (long long)offsets[blockIdx.x] + warp_base[warp] +
                        __popc(bal & ((1u << lane) - 1u));
    rec[n] = (int)r;
    node[r] = (int)n;
    for (int q = 1; q < 19; ++q) {
        const long long t = (long long)(q - 1) * n_rec + r;
        tq[t] = qw[q * nodes + n];
        tx[t] = wx[q * nodes + n];
        ty[t] = wy[q * nodes + n];
        tz[t] = wz[q * nodes + n];
    }
}

// Zou-He face descriptors: src/kernels/boundary_3d.jl:39-137 (0-based).
struct Face {
    int normal_axis, sign, q_axis, q_axis_opp, q_diag[4], q_diag_opp[4];
    int t1p, t1m, t2p, t2m, parallel[9], outgoing[5];
};

static const Face kFaces[6] = {
    {1, -1, 1, 2, {7, 9, 11, 13}, {10, 8, 14, 12}, 3, 4, 5, 6, {0, 3, 4, 5, 6, 15, 16, 17, 18}, {2, 8, 10, 12, 14}},
    {1, 1, 2, 1, {8, 10, 12, 14}, {9, 7, 13, 11}, 3, 4, 5, 6, {0, 3, 4, 5, 6, 15, 16, 17, 18}, {1, 7, 9, 11, 13}},
    {2, -1, 3, 4, {7, 8, 15, 17}, {10, 9, 18, 16}, 1, 2, 5, 6, {0, 1, 2, 5, 6, 11, 12, 13, 14}, {4, 9, 10, 16, 18}},
    {2, 1, 4, 3, {9, 10, 16, 18}, {8, 7, 17, 15}, 1, 2, 5, 6, {0, 1, 2, 5, 6, 11, 12, 13, 14}, {3, 7, 8, 15, 17}},
    {3, -1, 5, 6, {11, 12, 15, 16}, {14, 13, 18, 17}, 1, 2, 3, 4, {0, 1, 2, 3, 4, 7, 8, 9, 10}, {6, 13, 14, 17, 18}},
    {3, 1, 6, 5, {13, 14, 17, 18}, {12, 11, 16, 15}, 1, 2, 3, 4, {0, 1, 2, 3, 4, 7, 8, 9, 10}, {5, 11, 12, 15, 16}},
};

__device__ __forceinline__ size_t face_node(const Face &F, const Grid3 &g, int a, int b, int fixed) {
    int i, j, k;
    if (F.normal_axis == 1) { i = fixed; j = a; k = b; }
    else if (F.normal_axis == 2) { i = a; j = fixed; k = b; }
    else { i = a; j = b; k = fixed; }
    return (size_t)i + (size_t)g.Nx * ((size_t)j + (size_t)g.Ny * k);
}

// zou_he_velocity_3d_kernel!: src/kernels/boundary_3d.jl:154-223
template <typename T>
__global__ void zou_he_velocity_k(T *__restrict__ f, Grid3 g, Face F, int fixed, int N1, int N2,
                                  T u_n, T u_t1, T u_t2) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y;
    if (a >= N1 || b >= N2) return;
    const size_t c = face_node(F, g, a, b, fixed), P = g.plane;
    T sum_par = T(0), sum_out = T(0);
#pragma unroll
    for (int n = 0; n < 9; ++n) sum_par += f[c + F.parallel[n] * P];
#pragma unroll
    for (int n = 0; n < 5; ++n) sum_out += f[c + F.outgoing[n] * P];
    const T sg = T(F.sign);
    const T denom = T(1) + sg * u_n;
    const T rw = (sum_par + T(2) * sum_out) / denom;
    f[c + F.q_axis * P] = f[c + F.q_axis_opp * P] - sg * T(1.0 / 3.0) * rw * u_n;
    const T d1 = f[c + F.parallel[5] * P], d2 = f[c + F.parallel[6] * P];
    const T d3 = f[c + F.parallel[7] * P], d4 = f[c + F.parallel[8] * P];
    const T t1 = (f[c + F.t1p * P] - f[c + F.t1m * P]) + (d1 - d2 + d3 - d4);
    const T t2 = (f[c + F.t2p * P] - f[c + F.t2m * P]) + (d1 + d2 - d3 - d4);
    const T s6 = sg * T(1.0 / 6.0);
    f[c + F.q_diag[0] * P] = f[c + F.q_diag_opp[0] * P] - T(0.5) * t1 + T(0.5) * rw * u_t1 - s6 * rw * u_n;
    f[c + F.q_diag[1] * P] = f[c + F.q_diag_opp[1] * P] + T(0.5) * t1 - T(0.5) * rw * u_t1 - s6 * rw * u_n;
    f[c + F.q_diag[2] * P] = f[c + F.q_diag_opp[2] * P] - T(0.5) * t2 + T(0.5) * rw * u_t2 - s6 * rw * u_n;
    f[c + F.q_diag[3] * P] = f[c + F.q_diag_opp[3] * P] + T(0.5) * t2 - T(0.5) * rw * u_t2 - s6 * rw * u_n;
}

// zou_he_pressure_3d_kernel!: src/kernels/boundary_3d.jl:232-288
template <typename T>
__global__ void zou_he_pressure_k(T *__restrict__ f, Grid3 g, Face F, int fixed, int N1, int N2,
                                  T rho_out) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y;
    if (a >= N1 || b >= N2) return;
    const size_t c = face_node(F, g, a, b, fixed), P = g.plane;
    T sum_par = T(0), sum_out = T(0);
#pragma unroll
    for (int n = 0; n < 9; ++n) sum_par += f[c + F.parallel[n] * P];
#pragma unroll
    for (int n = 0; n < 5; ++n) sum_out += f[c + F.outgoing[n] * P];
    const T sg = T(F.sign);
    const T u_n = -sg * (T(1) - (sum_par + T(2) * sum_out) / rho_out);
    f[c + F.q_axis * P] = f[c + F.q_axis_opp * P] - sg * T(1.0 / 3.0) * rho_out * u_n;
    const T t1 = f[c + F.t1p * P] - f[c + F.t1m * P];
    const T t2 = f[c + F.t2p * P] - f[c + F.t2m * P];
    const T s6 = sg * T(1.0 / 6.0);
    f[c + F.q_diag[0] * P] = f[c + F.q_diag_opp[0] * P] - T(0.5) * t1 - s6 * rho_out * u_n;
    f[c + F.q_diag[1] * P] = f[c + F.q_diag_opp[1] * P] + T(0.5) * t1 - s6 * rho_out * u_n;
    f[c + F.q_diag[2] * P] = f[c + F.q_diag_opp[2] * P] - T(0.5) * t2 - s6 * rho_out * u_n;
    f[c + F.q_diag[3] * P] = f[c + F.q_diag_opp[3] * P] + T(0.5) * t2 - s6 * rho_out * u_n;
}

// stream_periodic_xz_movingwall_y_3d_kernel!: src/kernels/stream_periodic_3d.jl:106-166
template <typename T>
__global__ void __launch_bounds__(BX) movingwall_k(T *__restrict__ fo, const T *__restrict__ fi, Grid3 g,
                                                    T Ub, T Ut, T rho_w) {
    NODE3
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz;
    const long long sy = Nx, sz = (long long)Nx * Ny;
    const long long im = (i > 0 ? -1 : Nx - 1), ip = (i < Nx - 1 ? 1 : -(Nx - 1));
    const long long km = (k > 0 ? -1 : Nz - 1) * sz, kp = (k < Nz - 1 ? 1 : -(Nz - 1)) * sz;
    const bool lo = j == 0, hi = j == Ny - 1;
    const long long jm = (j > 0 ? -1 : 0) * sy, jp = (j < Ny - 1 ? 1 : 0) * sy;
    const T cbot = T(1.0 / 6.0) * rho_w * Ub, ctop = T(1.0 / 6.0) * rho_w * Ut;
    const T *f0 = fi + c;
    fo[c] = f0[0];
    fo[c + 1 * P] = f0[im + 1 * P];
    fo[c + 2 * P] = f0[ip + 2 * P];
    fo[c + 3 * P] = lo ? f0[4 * P] : f0[jm + 3 * P];
    fo[c + 4 * P] = hi ? f0[3 * P] : f0[jp + 4 * P];
    fo[c + 5 * P] = f0[km + 5 * P];
    fo[c + 6 * P] = f0[kp + 6 * P];
    fo[c + 7 * P] = lo ? f0[10 * P] + cbot : f0[im + jm + 7 * P];
    fo[c + 8 * P] = lo ? f0[9 * P] - cbot : f0[ip + jm + 8 * P];
    fo[c + 9 * P] = hi ? f0[8 * P] + ctop : f0[im + jp + 9 * P];
    fo[c + 10 * P] = hi ? f0[7 * P] - ctop : f0[ip + jp + 10 * P];
    fo[c + 11 * P] = f0[im + km + 11 * P];
    fo[c + 12 * P] = f0[ip + km + 12 * P];
    fo[c + 13 * P] = f0[im + kp + 13 * P];
    fo[c + 14 * P] = f0[ip + kp + 14 * P];
    fo[c + 15 * P] = lo ? f0[18 * P] : f0[jm + km + 15 * P];
    fo[c + 16 * P] = hi ? f0[17 * P] : f0[jp + km + 16 * P];
    fo[c + 17 * P] = lo ? f0[16 * P] : f0[jm + kp + 17 * P];
    fo[c + 18 * P] = hi ? f0[15 * P] : f0[jp + kp + 18 * P];
}

// ------------------------------------------------- unfused thermal DDF (3D) --
// D3Q19 velocities in the reference order (0-based q = reference q - 1).
__device__ constexpr int kCx[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
__device__ constexpr int kCy[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
__device__ constexpr int kCz[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};

// c_q . v written as the reference writes it: the signed first component,
// then the second added or subtracted (one component for the axis links).
template <typename T>
__device__ __forceinline__ T cdot(int q, T x, T y, T z) {
    const T v[3] = {x, y, z};
    const int cc[3] = {kCx[q], kCy[q], kCz[q]};
    T r = T(0);
    bool first = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (cc[a] == 0) continue;
        if (first) { r = cc[a] > 0 ? v[a] : -v[a]; first = false; }
        else r = cc[a] > 0 ? r + v[a] : r - v[a];
    }
    return r;
}

// collide_thermal_3d_kernel!: src/kernels/thermal_3d.jl:12-104
template <typename T>
__global__ void __launch_bounds__(BX) collide_thermal_k(T *__restrict__ gg, const T *__restrict__ ux,
                                                         const T *__restrict__ uy,
                                                         const T *__restrict__ uz, Grid3 g, T wT) {
    NODE3
    T p[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) p[q] = gg[c + q * P];
    T Tm = p[0];
#pragma unroll
    for (int q = 1; q < 19; ++q) Tm = Tm + p[q];
    const T a = ux[c], b = uy[c], d = uz[c], t3 = T(3);
    gg[c] = p[0] - wT * (p[0] - T(1.0 / 3.0) * Tm);
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        const T w = q < 7 ? T(1.0 / 18.0) : T(1.0 / 36.0);
        const T geq = w * Tm * (T(1) + t3 * cdot(q, a, b, d));
        gg[c + q * P] = p[q] - wT * (p[q] - geq);
    }
}

// compute_temperature_3d_kernel!: src/kernels/thermal_3d.jl:128-135
template <typename T>
__global__ void __launch_bounds__(BX) temperature_k(T *__restrict__ Temp, const T *__restrict__ gg, Grid3 g) {
    NODE3
    T s = gg[c];
#pragma unroll
    for (int q = 1; q < 19; ++q) s = s + gg[c + q * P];
    Temp[c] = s;
}

// Half-way anti-bounce-back on one face: _fixed_temp_{west,...,top}_3d!
// (src/kernels/thermal_3d.jl:154-480).  Per face: the main slot, and four
// edge slots, each on the edge where the link also leaves through the
// neighbouring face (order: the face's first in-plane axis low / high, then
// the second low / high).  An edge slot uses the edge temperature and is left
// alone when its skip bit is set.
template <typename T>
struct FixedTempFace3 {
    int face;      // 0 west, 1 east, 2 south, 3 north, 4 bottom, 5 top
    T T_wall;
    T T_e[4];
    unsigned skip;  // bit n: edge slot n is owned by the adjacent face
};

template <typename T>
struct FixedTempSet3 {
    int n;
    FixedTempFace3<T> f[6];
};

template <typename T>
__global__ void fixed_temp_k(T *__restrict__ gg, Grid3 g, FixedTempSet3<T> S) {
    const FixedTempFace3<T> F = S.f[blockIdx.z];
    const int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y;
    const int axis = F.face >> 1, high = F.face & 1;
    // in-plane axes: (y, z) for x-faces, (x, z) for y-faces, (x, y) for z-faces
    const int Na = axis == 0 ? g.Ny : g.Nx, Nb = axis == 2 ? g.Ny : g.Nz;
    if (a >= Na || b >= Nb) return;
    int i, j, k;
    if (axis == 0) { i = high ? g.Nx - 1 : 0; j = a; k = b; }
    else if (axis == 1) { i = a; j = high ? g.Ny - 1 : 0; k = b; }
    else { i = a; j = b; k = high ? g.Nz - 1 : 0; }
    const size_t c = (size_t)i + (size_t)g.Nx * ((size_t)j + (size_t)g.Ny * k), P = g.plane;
    const int qm[6] = {1, 2, 3, 4, 5, 6};
    const int qe[6][4] = {{7, 9, 11, 13}, {8, 10, 12, 14}, {7, 8, 15, 17},
                          {9, 10, 16, 18}, {11, 12, 15, 16}, {13, 14, 17, 18}};
    const bool on[4] = {a == 0, a == Na - 1, b == 0, b == Nb - 1};
    const T wa = T(2) * T(1.0 / 18.0), we = T(2) * T(1.0 / 36.0);
    T *m = gg + c + qm[F.face] * P;
    *m = -*m + wa * F.T_wall;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        T *s = gg + c + qe[F.face][e] * P;
        const T T_link = on[e] ? F.T_e[e] : F.T_wall;
        if (!(on[e] && ((F.skip >> e) & 1u))) *s = -*s + we * T_link;
    }
}

// The forced BGK update of one node (or two lanes) in place, force (fx, fy,
// fz): the body of collide_boussinesq_3d_kernel! / collide_guo_3d_kernel!
// after the force is known.
template <typename T>
__device__ __forceinline__ void forced_bgk_node(T *p, T w, T fx, T fy, T fz) {
    T rho = p[0];
#pragma unroll
    for (int q = 1; q < 19; ++q) rho = rho + p[q];
    const T inv = T(1) / rho;
    const T ux = ((p[1] - p[2] + p[7] - p[8] + p[9] - p[10] + p[11] - p[12] + p[13] - p[14]) +
                  fx / T(2)) * inv;
    const T uy = ((p[3] - p[4] + p[7] + p[8] - p[9] - p[10] + p[15] - p[16] + p[17] - p[18]) +
                  fy / T(2)) * inv;
    const T uz = ((p[5] - p[6] + p[11] + p[12] - p[13] - p[14] + p[15] + p[16] - p[17] - p[18]) +
                  fz / T(2)) * inv;
    const T usq = ux * ux + uy * uy + uz * uz;
    const T gpf = T(1) - w / T(2), t3 = T(3), t9 = T(9);
    T feq[19];
    feq_all(rho, ux, uy, uz, usq, feq);
    // Guo source S_q = w_q ((c_q - u) . F) 3 + w_q (c_q . u)(c_q . F) 9
    {
        const T wr = T(1.0 / 3.0);
        const T S0 = wr * ((-ux) * fx + (-uy) * fy + (-uz) * fz) * t3;
        p[0] = p[0] - w * (p[0] - feq[0]) + gpf * S0;
    }
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        const T wq = q < 7 ? T(1.0 / 18.0) : T(1.0 / 36.0);
        const T ax = kCx[q] > 0 ? T(1) - ux : (kCx[q] < 0 ? -T(1) - ux : -ux);
        const T ay = kCy[q] > 0 ? T(1) - uy : (kCy[q] < 0 ? -T(1) - uy : -uy);
        const T az = kCz[q] > 0 ? T(1) - uz : (kCz[q] < 0 ? -T(1) - uz : -uz);
        const T S = wq * (ax * fx + ay * fy + az * fz) * t3 +
                    wq * cdot(q, ux, uy, uz) * cdot(q, fx, fy, fz) * t9;
        p[q] = p[q] - w * (p[q] - feq[q]) + gpf * S;
    }
}

// BGK with the Guo source of a body force: MODE 0 collide_boussinesq_3d_kernel!
// (src/kernels/thermal_3d.jl:559-722, F = (0, beta_g (T - T_ref), 0)),
// MODE 1 collide_guo_3d_kernel! (src/kernels/collide_guo_3d.jl:5-186, constant
// F), MODE 2 collide_guo_field_3d_kernel! (:199-323, per-node F).  The three
// share the reference's operation order.  I: the element offset type (int
// where the 19 planes fit in 32 bits).  FP64 is bounded to 4 blocks per SM
// (128 registers instead of 166 at 3 blocks).
template <typename T, int MODE, typename I>
__global__ void __launch_bounds__(BX, sizeof(T) == 8 ? 4 : 1) boussinesq_k(T *__restrict__ f, const T *__restrict__ Temp,
                                                    const uint8_t *__restrict__ solid, Grid3 g, T w,
                                                    T beta_g, T T_ref, const T *__restrict__ Fxf,
                                                    const T *__restrict__ Fyf,
                                                    const T *__restrict__ Fzf, T Fx, T Fy, T Fz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= g.Nx) return;
    const I c = (I)i + (I)g.Nx * ((I)j + (I)g.Ny * (I)k);
    const I P = (I)g.plane;
    T p[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) p[q] = f[c + q * P];
    if (solid && solid[c]) {
        swap_pairs(p);
    } else {
        const T fx = MODE == 0 ? T(0) : (MODE == 1 ? Fx : Fxf[c]);
        const T fy = MODE == 0 ? beta_g * (Temp[c] - T_ref) : (MODE == 1 ? Fy : Fyf[c]);
        const T fz = MODE == 0 ? T(0) : (MODE == 1 ? Fz : Fzf[c]);
        forced_bgk_node(p, w, fx, fy, fz);
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) f[c + q * P] = p[q];
}

// FP32, even Nx, 8-byte aligned fields: thread t updates the adjacent nodes
// 2t, 2t + 1 of its row as two lanes (Lanes2), each as boussinesq_k does to
// within 3 ulp; a solid node of the pair swaps its opposite populations.
// Bounded to 4 blocks per SM (128 registers): 3 blocks at 164 registers ran
// slower, 5 blocks spill 170-220 B.
template <int MODE, typename I>
__global__ void __launch_bounds__(BX, 4) boussinesq2_k(float *__restrict__ f, const float *__restrict__ Temp,
                                                     const uint8_t *__restrict__ solid, Grid3 g,
                                                     float w, float beta_g, float T_ref,
                                                     const float *__restrict__ Fxf,
                                                     const float *__restrict__ Fyf,
                                                     const float *__restrict__ Fzf, float Fx,
                                                     float Fy, float Fz) {
    const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= g.Nx) return;
    const I c = (I)i + (I)g.Nx * ((I)j + (I)g.Ny * (I)k);
    const I P = (I)g.plane;
    Lanes2 p[19], o[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) p[q].v = *reinterpret_cast<const float2 *>(f + c + q * P);
    const uchar2 sd = solid ? *reinterpret_cast<const uchar2 *>(solid + c) : make_uchar2(0, 0);
    const auto ld2 = [&](const float *a) { return Lanes2::of(*reinterpret_cast<const float2 *>(a + c)); };
#pragma unroll
    for (int q = 0; q < 19; ++q) o[q] = p[q];
    if (!(sd.x && sd.y)) {
        const Lanes2 fx = MODE == 0 ? Lanes2(0.0) : (MODE == 1 ? Lanes2::of(make_float2(Fx, Fx)) : ld2(Fxf));
        const Lanes2 fy = MODE == 0 ? Lanes2::of(make_float2(beta_g, beta_g)) * (ld2(Temp) - Lanes2::of(make_float2(T_ref, T_ref)))
                                    : (MODE == 1 ? Lanes2::of(make_float2(Fy, Fy)) : ld2(Fyf));
        const Lanes2 fz = MODE == 0 ? Lanes2(0.0) : (MODE == 1 ? Lanes2::of(make_float2(Fz, Fz)) : ld2(Fzf));
        forced_bgk_node(o, Lanes2::of(make_float2(w, w)), fx, fy, fz);
    }
    if (sd.x || sd.y) {
        swap_pairs(p);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            if (sd.x) o[q].v.x = p[q].v.x;
            if (sd.y) o[q].v.y = p[q].v.y;
        }
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) *reinterpret_cast<float2 *>(f + c + q * P) = o[q].v;
}

}  // namespace d3
}  // namespace kb

// ----------------------------------------------------------- host wrappers --
namespace {

using namespace kb::d3;

Grid3 grid3(int Nx, int Ny, int Nz, int per = 0) {
    Grid3 g;
    g.Nx = Nx; g.Ny = Ny; g.Nz = Nz; g.per = per;
    g.plane = (size_t)Nx * (size_t)Ny * (size_t)Nz;
    return g;
}

int plain_dtype(const char *what, int dtype) {
    if (dtype != KB_F64 && dtype != KB_F32)
        return kb::set_error(KB_ERR_UNSUPPORTED,
                             "%s: dtype %d not supported (reference-arithmetic kernels take "
                             "KB_F64 or KB_F32)", what, dtype);
    return KB_OK;
}

#define KB3_DISPATCH_PLAIN(what, dtype, BODY)             \
    do {                                                  \
        int _e = plain_dtype(what, dtype);                \
        if (_e) return _e;                                \
        if (dtype == KB_F64) {                            \
            using T = double;                             \
            BODY;                                         \
        } else {                                          \
            using T = float;                              \
            BODY;                                         \
        }                                                 \
        return kb::check_launch(what);                    \
    } while (0)

void face_extent(const Face &F, int Nx, int Ny, int Nz, int *N1, int *N2) {
    if (F.normal_axis == 1) { *N1 = Ny; *N2 = Nz; }
    else if (F.normal_axis == 2) { *N1 = Nx; *N2 = Nz; }
    else { *N1 = Nx; *N2 = Ny; }
}

int face_fixed(const Face &F, int Nx, int Ny, int Nz) {
    const int n = F.normal_axis == 1 ? Nx : (F.normal_axis == 2 ? Ny : Nz);
    return F.sign > 0 ? n - 1 : 0;
}

}  // namespace

namespace {
int g_trt3d_dev_variant = 0;  // see kb_set_kernel_variant

template <typename T>
void launch_trt_libb_3d(void *f_out, const void *f_in, void *rho, void *ux, void *uy, void *uz,
                        const uint8_t *solid, const void *qw, const void *wx, const void *wy,
                        const void *wz, const Grid3 &g, double sp, double sm, cudaStream_t s) {
    const dim3 grid = nodes_grid(g.Nx, g.Ny, g.Nz);
    if (offsets_fit_int(g, 19))
        fused_trt_libb_k<T, int><<<grid, BX, 0, s>>>(
            (T *)f_out, (const T *)f_in, (T *)rho, (T *)ux, (T *)uy, (T *)uz, solid, (const T *)qw,
            (const T *)wx, (const T *)wy, (const T *)wz, g, (T)sp, (T)sm);
    else
        fused_trt_libb_k<T, long long><<<grid, BX, 0, s>>>(
            (T *)f_out, (const T *)f_in, (T *)rho, (T *)ux, (T *)uy, (T *)uz, solid, (const T *)qw,
            (const T *)wx, (const T *)wy, (const T *)wz, g, (T)sp, (T)sm);
}
}
namespace kb {
namespace umma {
void set_engine(int e);  // kb_umma.cu
}
}

extern "C" {

int kb_set_kernel_variant(int kernel, int variant) {
    KB_REQUIRE(kernel == 1 || kernel == 2, "kb_set_kernel_variant: unknown kernel id %d", kernel);
    if (kernel == 2) {
        KB_REQUIRE(variant >= 0 && variant <= 2, "kb_set_kernel_variant: engine %d not in 0..2", variant);
        kb::umma::set_engine(variant);
        return KB_OK;
    }
    KB_REQUIRE(variant >= 0 && variant <= 6, "kb_set_kernel_variant: variant %d not in 0..6", variant);
    g_trt3d_dev_variant = variant;
    return KB_OK;
}

int kb_stream_3d(void *f_out, const void *f_in, int Nx, int Ny, int Nz, int dtype, void *stream) {
    KB_REQUIRE(f_out && f_in, "kb_stream_3d: null population pointer");
    KB_REQUIRE(f_out != f_in, "kb_stream_3d: f_out and f_in must differ");
    if (int e = check_dims("kb_stream_3d", Nx, Ny, Nz)) return e;
    KB3_DISPATCH_PLAIN("kb_stream_3d", dtype,
        (stream_k<T><<<nodes_grid(Nx, Ny, Nz), BX, 0, kb::as_stream(stream)>>>(
            (T *)f_out, (const T *)f_in, grid3(Nx, Ny, Nz))));
}

int kb_collide_3d(void *f, const uint8_t *is_solid, int Nx, int Ny, int Nz, double omega,
                  int dtype, void *stream) {
    KB_REQUIRE(f, "kb_collide_3d: null population pointer");
    if (int e = check_dims("kb_collide_3d", Nx, Ny, Nz)) return e;
    KB3_DISPATCH_PLAIN("kb_collide_3d", dtype,
        (collide_k<T><<<nodes_grid(Nx, Ny, Nz), BX, 0, kb::as_stream(stream)>>>(
            (T *)f, is_solid, grid3(Nx, Ny, Nz), (T)omega)));
}

int kb_apply_zou_he_velocity_3d(void *f, int Nx, int Ny, int Nz, int face, double u_normal,
                                double u_tang1, double u_tang2, int dtype, void *stream) {
    KB_REQUIRE(f, "kb_apply_zou_he_velocity_3d: null population pointer");
    KB_REQUIRE(face >= 0 && face < 6, "kb_apply_zou_he_velocity_3d: face %d not in 0..5", face);
    if (int e = check_dims("kb_apply_zou_he_velocity_3d", Nx, Ny, Nz)) return e;
    const Face &F = kFaces[face];
    int N1, N2;
    face_extent(F, Nx, Ny, Nz, &N1, &N2);
    const int fixed = face_fixed(F, Nx, Ny, Nz);
    dim3 grid((N1 + BX - 1) / BX, N2);
    KB3_DISPATCH_PLAIN("kb_apply_zou_he_velocity_3d", dtype,
        (zou_he_velocity_k<T><<<grid, BX, 0, kb::as_stream(stream)>>>(
            (T *)f, grid3(Nx, Ny, Nz), F, fixed, N1, N2, (T)u_normal, (T)u_tang1, (T)u_tang2)));
}

int kb_apply_zou_he_top_3d(void *f, double u_wall_x, int Nx, int Ny, int Nz, int dtype,
                           void *stream) {
    // apply_zou_he_top_3d!: normal z, sign +1, u_n = 0, tangent x = u_wall_x
    return kb_apply_zou_he_velocity_3d(f, Nx, Ny, Nz, 5, 0.0, u_wall_x, 0.0, dtype, stream);
}

int kb_apply_zou_he_pressure_3d(void *f, int Nx, int Ny, int Nz, int face, double rho_out,
                                int dtype, void *stream) {
    KB_REQUIRE(f, "kb_apply_zou_he_pressure_3d: null population pointer");
    KB_REQUIRE(face >= 0 && face < 6, "kb_apply_zou_he_pressure_3d: face %d not in 0..5", face);
    if (int e = check_dims("kb_apply_zou_he_pressure_3d", Nx, Ny, Nz)) return e;
    const Face &F = kFaces[face];
    int N1, N2;
    face_extent(F, Nx, Ny, Nz, &N1, &N2);
    const int fixed = face_fixed(F, Nx, Ny, Nz);
    dim3 grid((N1 + BX - 1) / BX, N2);
    KB3_DISPATCH_PLAIN("kb_apply_zou_he_pressure_3d", dtype,
        (zou_he_pressure_k<T><<<grid, BX, 0, kb::as_stream(stream)>>>(
            (T *)f, grid3(Nx, Ny, Nz), F, fixed, N1, N2, (T)rho_out)));
}

int kb_compute_macroscopic_3d(void *rho, void *ux, void *uy, void *uz, const void *f, int Nx,
                              int Ny, int Nz, int dtype, void *stream) {
    KB_REQUIRE(rho && ux && uy && uz && f, "kb_compute_macroscopic_3d: null pointer");
    if (int e = check_dims("kb_compute_macroscopic_3d", Nx, Ny, Nz)) return e;
    KB3_DISPATCH_PLAIN("kb_compute_macroscopic_3d", dtype,
        (macroscopic_k<T><<<nodes_grid(Nx, Ny, Nz), BX, 0, kb::as_stream(stream)>>>(
            (T *)rho, (T *)ux, (T *)uy, (T *)uz, (const T *)f, grid3(Nx, Ny, Nz))));
}

}  // extern "C"

namespace {
// One fused TRT step over the grid g; the pointers address node (0, 0, 0)
// of g, the population stride is g.plane.
int trt3d_step(const char *what, void *f_out, const void *f_in, void *rho, void *ux, void *uy,
               void *uz, const uint8_t *is_solid, const Grid3 &g, double nu, double Lambda,
               int dtype, void *stream) {
    KB_REQUIRE(f_out && f_in, "%s: null population pointer", what);
    KB_REQUIRE(f_out != f_in, "%s: f_out and f_in must differ", what);
    const int nm = (rho != nullptr) + (ux != nullptr) + (uy != nullptr) + (uz != nullptr);
    KB_REQUIRE(nm == 0 || nm == 4, "%s: pass all four moment arrays or none", what);
    double sp, sm;
    if (int e = kb_trt_rates(nu, Lambda, &sp, &sm)) return e;
    cudaStream_t s = kb::as_stream(stream);
    const bool i32 = offsets_fit_int(g, 19);
    const dim3 grid = nodes_grid(g.Nx, g.Ny, g.Nz);
    if (dtype == KB_F64) {
        if (i32)
            fused_trt_k<double, int><<<grid, BX, 0, s>>>(
                (double *)f_out, (const double *)f_in, (double *)rho, (double *)ux, (double *)uy,
                (double *)uz, is_solid, g, sp, sm);
        else
            fused_trt_k<double, long long><<<grid, BX, 0, s>>>(
                (double *)f_out, (const double *)f_in, (double *)rho, (double *)ux, (double *)uy,
                (double *)uz, is_solid, g, sp, sm);
    } else if (dtype == KB_F32) {
        if (i32)
            fused_trt_k<float, int><<<grid, BX, 0, s>>>(
                (float *)f_out, (const float *)f_in, (float *)rho, (float *)ux, (float *)uy,
                (float *)uz, is_solid, g, (float)sp, (float)sm);
        else
            fused_trt_k<float, long long><<<grid, BX, 0, s>>>(
                (float *)f_out, (const float *)f_in, (float *)rho, (float *)ux, (float *)uy,
                (float *)uz, is_solid, g, (float)sp, (float)sm);
    } else if (dtype == KB_F32_DEV || dtype == KB_F16_DEV || dtype == KB_BF16_DEV ||
               dtype == KB_F16_DEV_SR || dtype == KB_BF16_DEV_SR) {
        return launch_trt3d_dev(dtype, f_out, f_in, (float *)rho, (float *)ux, (float *)uy,
                                (float *)uz, is_solid, g, (float)sp, (float)sm, s, g_trt3d_dev_variant);
    } else {
        return kb::set_error(KB_ERR_UNSUPPORTED, "%s: unknown dtype %d", what, dtype);
    }
    return kb::check_launch(what);
}

// bytes of one population word and of one moment value per storage
size_t pop_bytes(int dtype) {
    switch (dtype) {
        case KB_F64: return 8;
        case KB_F32: case KB_F32_DEV: return 4;
        case KB_F16_DEV: case KB_BF16_DEV: case KB_F16_DEV_SR: case KB_BF16_DEV_SR: return 2;
        default: return 0;
    }
}
}  // namespace

extern "C" {

int kb_fused_trt_step_3d(void *f_out, const void *f_in, void *rho, void *ux, void *uy, void *uz,
                         const uint8_t *is_solid, int Nx, int Ny, int Nz, double nu,
                         double Lambda, int periodic, int dtype, void *stream) {
    const char *what = "kb_fused_trt_step_3d";
    KB_REQUIRE(periodic >= 0 && periodic < 8, "%s: periodic mask %d not in 0..7", what, periodic);
    if (int e = check_dims(what, Nx, Ny, Nz)) return e;
    return trt3d_step(what, f_out, f_in, rho, ux, uy, uz, is_solid, grid3(Nx, Ny, Nz, periodic),
                      nu, Lambda, dtype, stream);
}

int kb_fused_trt_step_3d_zrange(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                                void *uz, const uint8_t *is_solid, int Nx, int Ny, int Nz_alloc,
                                int k_begin, int k_end, double nu, double Lambda,
                                int periodic_xy, int dtype, void *stream) {
    const char *what = "kb_fused_trt_step_3d_zrange";
    KB_REQUIRE(periodic_xy >= 0 && periodic_xy < 4, "%s: periodic mask %d not in 0..3", what,
               periodic_xy);
    if (int e = check_dims(what, Nx, Ny, Nz_alloc)) return e;
    KB_REQUIRE(k_begin >= 1 && k_begin < k_end && k_end <= Nz_alloc - 1,
               "%s: plane range [%d, %d) must lie in [1, %d) (the first and last allocated planes "
               "are halo planes)", what, k_begin, k_end, Nz_alloc - 1);
    const size_t eb = pop_bytes(dtype);
    KB_REQUIRE(eb != 0, "%s: unknown dtype %d", what, dtype);
    const size_t mb = (dtype == KB_F64 || dtype == KB_F32) ? eb : 4;  // moment bytes
    const size_t off = (size_t)k_begin * (size_t)Nx * (size_t)Ny;     // nodes before the range
    Grid3 g = grid3(Nx, Ny, Nz_alloc, (periodic_xy & 3) | KB_ZHALO);
    g.Nz = k_end - k_begin;
    g.zoff = k_begin;
    const auto at = [off](void *p, size_t b) { return p ? (void *)((char *)p + off * b) : p; };
    return trt3d_step(what, at(f_out, eb), (const char *)f_in + off * eb, at(rho, mb), at(ux, mb),
                      at(uy, mb), at(uz, mb), is_solid ? is_solid + off : nullptr, g, nu, Lambda,
                      dtype, stream);
}

int kb_fused_trt_libb_step_3d(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                              void *uz, const uint8_t *is_solid, const void *q_wall,
                              const void *uw_link_x, const void *uw_link_y, const void *uw_link_z,
                              int Nx, int Ny, int Nz, double nu, double Lambda, int periodic,
                              int dtype, void *stream) {
    const char *what = "kb_fused_trt_libb_step_3d";
    KB_REQUIRE(f_out && f_in, "%s: null population pointer", what);
    KB_REQUIRE(q_wall && uw_link_x && uw_link_y && uw_link_z, "%s: null q_wall / uw_link pointer",
               what);
    KB_REQUIRE(f_out != f_in, "%s: f_out and f_in must differ", what);
    const int nm = (rho != nullptr) + (ux != nullptr) + (uy != nullptr) + (uz != nullptr);
    KB_REQUIRE(nm == 0 || nm == 4, "%s: pass all four moment arrays or none", what);
    KB_REQUIRE(periodic >= 0 && periodic < 8, "%s: periodic mask %d not in 0..7", what, periodic);
    if (int e = check_dims(what, Nx, Ny, Nz)) return e;
    double sp, sm;
    if (int e = kb_trt_rates(nu, Lambda, &sp, &sm)) return e;
    const Grid3 g = grid3(Nx, Ny, Nz, periodic);
    cudaStream_t s = kb::as_stream(stream);
    KB3_DISPATCH_PLAIN(what, dtype,
        launch_trt_libb_3d<T>(f_out, f_in, rho, ux, uy, uz, is_solid, q_wall, uw_link_x,
                              uw_link_y, uw_link_z, g, sp, sm, s));
}

int kb_stream_periodic_xz_movingwall_y_3d(void *f_out, const void *f_in, double Ub, double Ut,
                                          double rho_w, int Nx, int Ny, int Nz, int dtype,
                                          void *stream) {
    KB_REQUIRE(f_out && f_in, "kb_stream_periodic_xz_movingwall_y_3d: null population pointer");
    KB_REQUIRE(f_out != f_in, "kb_stream_periodic_xz_movingwall_y_3d: f_out and f_in must differ");
    if (int e = check_dims("kb_stream_periodic_xz_movingwall_y_3d", Nx, Ny, Nz)) return e;
    KB3_DISPATCH_PLAIN("kb_stream_periodic_xz_movingwall_y_3d", dtype,
        (movingwall_k<T><<<nodes_grid(Nx, Ny, Nz), BX, 0, kb::as_stream(stream)>>>(
            (T *)f_out, (const T *)f_in, grid3(Nx, Ny, Nz), (T)Ub, (T)Ut, (T)rho_w)));
}

int kb_collide_thermal_3d(void *g, const void *ux, const void *uy, const void *uz, int Nx, int Ny,
                          int Nz, double omega_T, int dtype, void *stream) {
    KB_REQUIRE(g && ux && uy && uz, "kb_collide_thermal_3d: null pointer");
    if (int e = check_dims("kb_collide_thermal_3d", Nx, Ny, Nz)) return e;
    KB3_DISPATCH_PLAIN("kb_collide_thermal_3d", dtype,
        (collide_thermal_k<T><<<nodes_grid(Nx, Ny, Nz), BX, 0, kb::as_stream(stream)>>>(
            (T *)g, (const T *)ux, (const T *)uy, (const T *)uz, grid3(Nx, Ny, Nz), (T)omega_T)));
}

int kb_compute_temperature_3d(void *Temp, const void *g, int Nx, int Ny, int Nz, int dtype,
                              void *stream) {
    KB_REQUIRE(Temp && g, "kb_compute_temperature_3d: null pointer");
    if (int e = check_dims("kb_compute_temperature_3d", Nx, Ny, Nz)) return e;
    KB3_DISPATCH_PLAIN("kb_compute_temperature_3d", dtype,
        (temperature_k<T><<<nodes_grid(Nx, Ny, Nz), BX, 0, kb::as_stream(stream)>>>(
            (T *)Temp, (const T *)g, grid3(Nx, Ny, Nz))));
}

}  // extern "C"

namespace {

template <typename T, int MODE>
void launch_boussinesq_3d(T *f, const T *Temp, const uint8_t *solid, const Grid3 &g, T w, T beta_g,
                          T T_ref, const T *Fxf, const T *Fyf, const T *Fzf, T Fx, T Fy, T Fz,
                          cudaStream_t s) {
    const bool i32 = offsets_fit_int(g, 19);
    if constexpr (sizeof(T) == 4) {
        // two nodes per thread where the rows pair up and the fields allow
        // 8-byte accesses (the solid mask 2-byte)
        const auto al = [](const void *p, uintptr_t n) { return ((uintptr_t)p & (n - 1)) == 0; };
        if (g.Nx % 2 == 0 && al(f, 8) && al(Temp, 8) && al(Fxf, 8) && al(Fyf, 8) && al(Fzf, 8) &&
            al(solid, 2)) {
            const dim3 grid((unsigned)((g.Nx / 2 + BX - 1) / BX), (unsigned)g.Ny, (unsigned)g.Nz);
            if (i32)
                boussinesq2_k<MODE, int><<<grid, BX, 0, s>>>(f, Temp, solid, g, w, beta_g, T_ref, Fxf, Fyf,
                                                             Fzf, Fx, Fy, Fz);
            else
                boussinesq2_k<MODE, size_t><<<grid, BX, 0, s>>>(f, Temp, solid, g, w, beta_g, T_ref, Fxf,
                                                                Fyf, Fzf, Fx, Fy, Fz);
            return;
        }
    }
    const dim3 grid = nodes_grid(g.Nx, g.Ny, g.Nz);
    if (i32)
        boussinesq_k<T, MODE, int><<<grid, BX, 0, s>>>(f, Temp, solid, g, w, beta_g, T_ref, Fxf, Fyf,
                                                       Fzf, Fx, Fy, Fz);
    else
        boussinesq_k<T, MODE, size_t><<<grid, BX, 0, s>>>(f, Temp, solid, g, w, beta_g, T_ref, Fxf,
                                                          Fyf, Fzf, Fx, Fy, Fz);
}

}  // namespace

extern "C" {

int kb_collide_boussinesq_3d(void *f, const void *Temp, const uint8_t *is_solid, int Nx, int Ny,
                             int Nz, double omega, double beta_g, double T_ref, int dtype,
                             void *stream) {
    KB_REQUIRE(f && Temp, "kb_collide_boussinesq_3d: null pointer");
    if (int e = check_dims("kb_collide_boussinesq_3d", Nx, Ny, Nz)) return e;
    KB3_DISPATCH_PLAIN("kb_collide_boussinesq_3d", dtype,
        (launch_boussinesq_3d<T, 0>((T *)f, (const T *)Temp, is_solid, grid3(Nx, Ny, Nz), (T)omega,
                                    (T)beta_g, (T)T_ref, nullptr, nullptr, nullptr, T(0), T(0), T(0),
                                    kb::as_stream(stream))));
}

int kb_collide_guo_3d(void *f, const uint8_t *is_solid, int Nx, int Ny, int Nz, double omega,
                      double Fx, double Fy, double Fz, int dtype, void *stream) {
    KB_REQUIRE(f, "kb_collide_guo_3d: null population pointer");
    if (int e = check_dims("kb_collide_guo_3d", Nx, Ny, Nz)) return e;
    KB3_DISPATCH_PLAIN("kb_collide_guo_3d", dtype,
        (launch_boussinesq_3d<T, 1>((T *)f, nullptr, is_solid, grid3(Nx, Ny, Nz), (T)omega, T(0), T(0),
                                    nullptr, nullptr, nullptr, (T)Fx, (T)Fy, (T)Fz,
                                    kb::as_stream(stream))));
}

int kb_collide_guo_field_3d(void *f, const uint8_t *is_solid, const void *Fx_field,
                            const void *Fy_field, const void *Fz_field, int Nx, int Ny, int Nz,
                            double omega, int dtype, void *stream) {
    KB_REQUIRE(f && Fx_field && Fy_field && Fz_field, "kb_collide_guo_field_3d: null pointer");
    if (int e = check_dims("kb_collide_guo_field_3d", Nx, Ny, Nz)) return e;
    KB3_DISPATCH_PLAIN("kb_collide_guo_field_3d", dtype,
        (launch_boussinesq_3d<T, 2>((T *)f, nullptr, is_solid, grid3(Nx, Ny, Nz), (T)omega, T(0), T(0),
                                    (const T *)Fx_field, (const T *)Fy_field, (const T *)Fz_field,
                                    T(0), T(0), T(0), kb::as_stream(stream))));
}

}  // extern "C"

namespace {

template <typename T>
int launch_fixed_temp_3d(T *g, int Nx, int Ny, int Nz, const FixedTempSet3<T> &S, cudaStream_t s,
                         const char *what) {
    if (S.n == 0) return KB_OK;
    int Na = 1, Nb = 1;
    for (int n = 0; n < S.n; ++n) {
        const int axis = S.f[n].face >> 1;
        const int a = axis == 0 ? Ny : Nx, b = axis == 2 ? Ny : Nz;
        Na = a > Na ? a : Na;
        Nb = b > Nb ? b : Nb;
    }
    fixed_temp_k<T><<<dim3((Na + BX - 1) / BX, Nb, S.n), BX, 0, s>>>(g, grid3(Nx, Ny, Nz), S);
    return kb::check_launch(what);
}

template <typename T>
T edge_temp(double Ta, bool has_b, double Tb) {
    // _corner_temp (thermal_2d.jl:356-357): the mean of the two wall temperatures
    return has_b ? (T(Ta) + T(Tb)) / T(2) : T(Ta);
}

// _apply_fixed_temp_faces_3d! (thermal_3d.jl:494-533): x-faces apply all
// their edge slots (mean temperature where the other face is Dirichlet);
// y-faces skip the edges they share with a Dirichlet x-face; z-faces skip
// every edge shared with a Dirichlet face.  No slot is written twice, so all
// faces run in one launch.
template <typename T>
int fixed_temp_all_3d(T *g, int Nx, int Ny, int Nz, unsigned faces, const double *Tf,
                      cudaStream_t s) {
    bool h[6];
    for (int n = 0; n < 6; ++n) h[n] = (faces >> n) & 1u;
    FixedTempSet3<T> S{};
    S.n = 0;
    for (int face = 0; face < 6; ++face) {
        if (!h[face]) continue;
        FixedTempFace3<T> F{};
        F.face = face;
        F.T_wall = T(Tf[face]);
        if (face < 2) {
            F.T_e[0] = edge_temp<T>(Tf[face], h[2], Tf[2]);
            F.T_e[1] = edge_temp<T>(Tf[face], h[3], Tf[3]);
            F.T_e[2] = edge_temp<T>(Tf[face], h[4], Tf[4]);
            F.T_e[3] = edge_temp<T>(Tf[face], h[5], Tf[5]);
            F.skip = 0u;
        } else if (face < 4) {
            F.T_e[0] = F.T_e[1] = T(Tf[face]);
            F.T_e[2] = edge_temp<T>(Tf[face], h[4], Tf[4]);
            F.T_e[3] = edge_temp<T>(Tf[face], h[5], Tf[5]);
            F.skip = (h[0] ? 1u : 0u) | (h[1] ? 2u : 0u);
        } else {
            F.T_e[0] = F.T_e[1] = F.T_e[2] = F.T_e[3] = T(Tf[face]);
            F.skip = (h[0] ? 1u : 0u) | (h[1] ? 2u : 0u) | (h[2] ? 4u : 0u) | (h[3] ? 8u : 0u);
        }
        S.f[S.n++] = F;
    }
    return launch_fixed_temp_3d(g, Nx, Ny, Nz, S, s, "kb_apply_fixed_temp_3d");
}

}  // namespace

extern "C" {

int kb_apply_fixed_temp_face_3d(void *g, int Nx, int Ny, int Nz, int face, double T_wall,
                                const double *T_edge, unsigned skip_edges, int dtype,
                                void *stream) {
    KB_REQUIRE(g, "kb_apply_fixed_temp_face_3d: null population pointer");
    KB_REQUIRE(face >= 0 && face < 6, "kb_apply_fixed_temp_face_3d: face %d not in 0..5", face);
    KB_REQUIRE(skip_edges < 16u, "kb_apply_fixed_temp_face_3d: skip mask 0x%x beyond 4 edges",
               skip_edges);
    if (int e = check_dims("kb_apply_fixed_temp_face_3d", Nx, Ny, Nz)) return e;
    KB3_DISPATCH_PLAIN("kb_apply_fixed_temp_face_3d", dtype, {
        FixedTempSet3<T> S{};
        S.n = 1;
        S.f[0].face = face;
        S.f[0].T_wall = (T)T_wall;
        for (int n = 0; n < 4; ++n) S.f[0].T_e[n] = T_edge ? (T)T_edge[n] : (T)T_wall;
        S.f[0].skip = skip_edges;
        if (int r = launch_fixed_temp_3d((T *)g, Nx, Ny, Nz, S, kb::as_stream(stream),
                                         "kb_apply_fixed_temp_face_3d"))
            return r;
    });
}

int kb_apply_fixed_temp_3d(void *g, int Nx, int Ny, int Nz, unsigned faces, const double *T_faces,
                           int dtype, void *stream) {
    KB_REQUIRE(g, "kb_apply_fixed_temp_3d: null population pointer");
    KB_REQUIRE(faces < 64u, "kb_apply_fixed_temp_3d: face mask 0x%x has bits beyond 0..5", faces);
    KB_REQUIRE(faces == 0u || T_faces, "kb_apply_fixed_temp_3d: null temperature array");
    if (int e = check_dims("kb_apply_fixed_temp_3d", Nx, Ny, Nz)) return e;
    KB3_DISPATCH_PLAIN("kb_apply_fixed_temp_3d", dtype, {
        if (int r = fixed_temp_all_3d((T *)g, Nx, Ny, Nz, faces, T_faces, kb::as_stream(stream)))
            return r;
    });
}

}  // extern "C"

// ------------------------------------------------------- compact cut links --
struct kb_libb_links {
    int Nx = 0, Ny = 0, Nz = 0, dtype = KB_F64;
    uint8_t *cls = nullptr;
    int *rec = nullptr;
    int *node = nullptr;  // node of each record
    void *qw = nullptr, *wx = nullptr, *wy = nullptr, *wz = nullptr;
    long long n_rec = 0;
};

namespace {

kb::d3::LinkTable3 table_view(const kb_libb_links *L) {
    return kb::d3::LinkTable3{L->cls, L->rec, L->qw, L->wx, L->wy, L->wz, L->n_rec, L->node};
}

template <typename T>
int build_links(kb_libb_links *L, const uint8_t *solid, const T *qw, const T *wx, const T *wy,
                const T *wz, cudaStream_t s) {
    const size_t nodes = (size_t)L->Nx * L->Ny * L->Nz;
    const size_t nblk = (nodes + kb::d3::LT - 1) / kb::d3::LT;
    int *counts = nullptr;
    cudaError_t e = cudaMalloc(&L->cls, nodes);
    if (e == cudaSuccess) e = cudaMalloc(&L->rec, nodes * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&counts, nblk * sizeof(int));
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(counts);
        return kb::set_error(KB_ERR_NOMEM, "kb_libb_links_create: device allocation failed: %s",
                             cudaGetErrorString(e));
    }
    kb::d3::links_count_k<T><<<(unsigned)nblk, kb::d3::LT, 0, s>>>(L->cls, counts, solid, qw, nodes);
    std::vector<int> h(nblk);
    e = cudaMemcpyAsync(h.data(), counts, nblk * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaFree(counts);
        return kb::set_error(KB_ERR_CUDA, "kb_libb_links_create: %s", cudaGetErrorString(e));
    }
    long long acc = 0;
    for (size_t b = 0; b < nblk; ++b) { const int v = h[b]; h[b] = (int)acc; acc += v; }
    if (acc > 2147483647LL) {
        cudaFree(counts);
        return kb::set_error(KB_ERR_ARG, "kb_libb_links_create: %lld nodes with cut links "
                             "exceed the 2^31 record limit", acc);
    }
    L->n_rec = acc;
    e = cudaMemcpyAsync(counts, h.data(), nblk * sizeof(int), cudaMemcpyHostToDevice, s);
    if (acc > 0 && e == cudaSuccess) {
        const size_t bytes = (size_t)acc * 18 * sizeof(T);
        e = cudaMalloc(&L->node, (size_t)acc * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&L->qw, bytes);
        if (e == cudaSuccess) e = cudaMalloc(&L->wx, bytes);
        if (e == cudaSuccess) e = cudaMalloc(&L->wy, bytes);
        if (e == cudaSuccess) e = cudaMalloc(&L->wz, bytes);
        if (e == cudaSuccess)
            kb::d3::links_fill_k<T><<<(unsigned)nblk, kb::d3::LT, 0, s>>>(
                L->rec, L->node, (T *)L->qw, (T *)L->wx, (T *)L->wy, (T *)L->wz, L->cls, counts, qw, wx,
                wy, wz, nodes, acc);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(counts);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return kb::set_error(KB_ERR_NOMEM, "kb_libb_links_create: %s", cudaGetErrorString(e));
    }
    return kb::check_launch("kb_libb_links_create");
}

template <typename T, typename I>
int launch_links_3d_i(T *fo, const T *fi, T *rho, T *ux, T *uy, T *uz,
                       const kb::d3::LinkTable3 &L, const Grid3 &g, T sp, T sm, cudaStream_t s) {
    const dim3 grid = nodes_grid(g.Nx, g.Ny, g.Nz);
    kb::d3::SideStream *ss = L.n_rec > 0 ? kb::d3::side_stream() : nullptr;
    if (!ss) {  // no cut nodes, or no side stream: one kernel for every node
        fused_trt_links_k<T, I, false><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
        return KB_OK;
    }
    // the cut nodes on the side stream, forked from s and joined back
    // before anything that follows on s
    cudaStream_t cs = s;
    if (cudaEventRecord(ss->fork, s) == cudaSuccess && cudaStreamWaitEvent(ss->side, ss->fork, 0) == cudaSuccess)
        cs = ss->side;
    else
        cudaGetLastError();
    const unsigned nb = (unsigned)((L.n_rec + BX - 1) / BX);
    fused_trt_cut_k<T, I><<<nb, BX, 0, cs>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
    fused_trt_links_k<T, I, true><<<grid, BX, 0, s>>>(fo, fi, rho, ux, uy, uz, L, g, sp, sm);
    if (cs != s && (cudaEventRecord(ss->join, cs) != cudaSuccess || cudaStreamWaitEvent(s, ss->join, 0) != cudaSuccess))
        return kb::set_error(KB_ERR_CUDA, "kb_fused_trt_libb_links_step_3d: joining the cut-node stream failed");
    return KB_OK;
}

template <typename T>
int launch_links_3d(void *f_out, const void *f_in, void *rho, void *ux, void *uy, void *uz,
                    const kb::d3::LinkTable3 &L, const Grid3 &g, double sp, double sm,
                    cudaStream_t s) {
    if (offsets_fit_int(g, 19))
        return launch_links_3d_i<T, int>((T *)f_out, (const T *)f_in, (T *)rho, (T *)ux, (T *)uy, (T *)uz, L, g,
                                  (T)sp, (T)sm, s);
    return launch_links_3d_i<T, long long>((T *)f_out, (const T *)f_in, (T *)rho, (T *)ux, (T *)uy, (T *)uz, L,
                                        g, (T)sp, (T)sm, s);
}

}  // namespace

extern "C" {

int kb_libb_links_destroy(kb_libb_links *L) {
    if (!L) return KB_OK;
    cudaFree(L->cls); cudaFree(L->rec); cudaFree(L->node);
    cudaFree(L->qw); cudaFree(L->wx); cudaFree(L->wy); cudaFree(L->wz);
    delete L;
    return KB_OK;
}

int kb_libb_links_create(kb_libb_links **out, const uint8_t *is_solid, const void *q_wall,
                         const void *uw_link_x, const void *uw_link_y, const void *uw_link_z,
                         int Nx, int Ny, int Nz, int dtype, void *stream) {
    const char *what = "kb_libb_links_create";
    KB_REQUIRE(out, "%s: null handle pointer", what);
    *out = nullptr;
    KB_REQUIRE(q_wall && uw_link_x && uw_link_y && uw_link_z, "%s: null q_wall / uw_link pointer",
               what);
    KB_REQUIRE(dtype == KB_F64 || dtype == KB_F32,
               "%s: link arrays must be KB_F64 or KB_F32 (dtype %d)", what, dtype);
    if (int e = check_dims(what, Nx, Ny, Nz)) return e;
    kb_libb_links *L = new kb_libb_links();
    L->Nx = Nx; L->Ny = Ny; L->Nz = Nz; L->dtype = dtype;
    cudaStream_t s = kb::as_stream(stream);
    const int r = dtype == KB_F64
        ? build_links(L, is_solid, (const double *)q_wall, (const double *)uw_link_x,
                      (const double *)uw_link_y, (const double *)uw_link_z, s)
        : build_links(L, is_solid, (const float *)q_wall, (const float *)uw_link_x,
                      (const float *)uw_link_y, (const float *)uw_link_z, s);
    if (r) { kb_libb_links_destroy(L); return r; }
    *out = L;
    return KB_OK;
}

int kb_libb_links_info(const kb_libb_links *L, long long *nodes_with_links, int *dtype) {
    KB_REQUIRE(L, "kb_libb_links_info: null handle");
    if (nodes_with_links) *nodes_with_links = L->n_rec;
    if (dtype) *dtype = L->dtype;
    return KB_OK;
}

int kb_fused_trt_libb_links_step_3d(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                                    void *uz, const kb_libb_links *L, double nu, double Lambda,
                                    int periodic, int dtype, void *stream) {
    const char *what = "kb_fused_trt_libb_links_step_3d";
    KB_REQUIRE(f_out && f_in, "%s: null population pointer", what);
    KB_REQUIRE(L, "%s: null cut-link table", what);
    KB_REQUIRE(f_out != f_in, "%s: f_out and f_in must differ", what);
    const int nm = (rho != nullptr) + (ux != nullptr) + (uy != nullptr) + (uz != nullptr);
    KB_REQUIRE(nm == 0 || nm == 4, "%s: pass all four moment arrays or none", what);
    KB_REQUIRE(periodic >= 0 && periodic < 8, "%s: periodic mask %d not in 0..7", what, periodic);
    double sp, sm;
    if (int e = kb_trt_rates(nu, Lambda, &sp, &sm)) return e;
    const Grid3 g = grid3(L->Nx, L->Ny, L->Nz, periodic);
    cudaStream_t s = kb::as_stream(stream);
    const kb::d3::LinkTable3 T3 = table_view(L);
    if (dtype == KB_F64 || dtype == KB_F32) {
        if (L->dtype != dtype)
            return kb::set_error(KB_ERR_UNSUPPORTED, "%s: populations of dtype %d need a cut-link "
                                 "table of the same dtype (table has %d)", what, dtype, L->dtype);
        const int rc = dtype == KB_F64 ? launch_links_3d<double>(f_out, f_in, rho, ux, uy, uz, T3, g, sp, sm, s)
                                       : launch_links_3d<float>(f_out, f_in, rho, ux, uy, uz, T3, g, sp, sm, s);
        if (rc != KB_OK) return rc;
        return kb::check_launch(what);
    }
    if (dtype == KB_F32_DEV || dtype == KB_F16_DEV || dtype == KB_BF16_DEV ||
        dtype == KB_F16_DEV_SR || dtype == KB_BF16_DEV_SR) {
        if (L->dtype != KB_F32)
            return kb::set_error(KB_ERR_UNSUPPORTED, "%s: deviation storages collide in FP32 and "
                                 "need a KB_F32 cut-link table", what);
        return kb::d3::launch_trt3d_dev_links(dtype, f_out, f_in, (float *)rho, (float *)ux,
                                              (float *)uy, (float *)uz, T3, g, (float)sp,
                                              (float)sm, s, g_trt3d_dev_variant);
    }
    return kb::set_error(KB_ERR_UNSUPPORTED, "%s: unknown dtype %d", what, dtype);
}

}  // extern "C"

extern "C" {

int kb_compute_macroscopic_forced_3d(void *rho, void *ux, void *uy, void *uz, const void *f,
                                     int Nx, int Ny, int Nz, double Fx, double Fy, double Fz,
                                     int dtype, void *stream) {
    KB_REQUIRE(rho && ux && uy && uz && f, "kb_compute_macroscopic_forced_3d: null pointer");
    if (int e = check_dims("kb_compute_macroscopic_forced_3d", Nx, Ny, Nz)) return e;
    KB3_DISPATCH_PLAIN("kb_compute_macroscopic_forced_3d", dtype,
        (macroscopic_forced_k<T, false><<<nodes_grid(Nx, Ny, Nz), BX, 0, kb::as_stream(stream)>>>(
            (T *)rho, (T *)ux, (T *)uy, (T *)uz, (const T *)f, grid3(Nx, Ny, Nz), (T)Fx, (T)Fy,
            (T)Fz, nullptr, nullptr, nullptr)));
}

int kb_compute_macroscopic_forced_field_3d(void *rho, void *ux, void *uy, void *uz, const void *f,
                                           const void *Fx_field, const void *Fy_field,
                                           const void *Fz_field, int Nx, int Ny, int Nz,
                                           int dtype, void *stream) {
    KB_REQUIRE(rho && ux && uy && uz && f && Fx_field && Fy_field && Fz_field,
               "kb_compute_macroscopic_forced_field_3d: null pointer");
    if (int e = check_dims("kb_compute_macroscopic_forced_field_3d", Nx, Ny, Nz)) return e;
    KB3_DISPATCH_PLAIN("kb_compute_macroscopic_forced_field_3d", dtype,
        (macroscopic_forced_k<T, true><<<nodes_grid(Nx, Ny, Nz), BX, 0, kb::as_stream(stream)>>>(
            (T *)rho, (T *)ux, (T *)uy, (T *)uz, (const T *)f, grid3(Nx, Ny, Nz), T(0), T(0),
            T(0), (const T *)Fx_field, (const T *)Fy_field, (const T *)Fz_field)));
}

int kb_stream_periodic_xz_wall_y_3d(void *f_out, const void *f_in, int Nx, int Ny, int Nz,
                                    int dtype, void *stream) {
    KB_REQUIRE(f_out && f_in, "kb_stream_periodic_xz_wall_y_3d: null population pointer");
    KB_REQUIRE(f_out != f_in, "kb_stream_periodic_xz_wall_y_3d: f_out and f_in must differ");
    if (int e = check_dims("kb_stream_periodic_xz_wall_y_3d", Nx, Ny, Nz)) return e;
    // the pull of stream_3d with x and z wrapped (periodic mask x | z)
    KB3_DISPATCH_PLAIN("kb_stream_periodic_xz_wall_y_3d", dtype,
        (stream_k<T><<<nodes_grid(Nx, Ny, Nz), BX, 0, kb::as_stream(stream)>>>(
            (T *)f_out, (const T *)f_in, grid3(Nx, Ny, Nz, 5))));
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Ghost planes of a z-slab whose neighbours are itself (one rank on a
// periodic z axis): the five c_z = +1 populations of the top real plane go
// to the bottom ghost plane, the five c_z = -1 populations of the first real
// plane to the top ghost plane; blockIdx.y picks one of the ten planes.
namespace kb {
namespace d3 {

template <typename W>
__global__ void slab_ghosts_k(W *f, size_t plane, size_t pop, int nz_alloc, int lo, int hi) {
    constexpr int CZP[5] = {5, 11, 12, 15, 16}, CZM[5] = {6, 13, 14, 17, 18};
    const int p = blockIdx.y;
    if (p < 5 ? !lo : !hi) return;
    const int q = p < 5 ? CZP[p] : CZM[p - 5];
    const size_t dst = (size_t)q * pop + (p < 5 ? 0 : (size_t)(nz_alloc - 1) * plane);
    const size_t src = (size_t)q * pop + (size_t)(p < 5 ? nz_alloc - 1 - hi : lo) * plane;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < plane;
         i += (size_t)gridDim.x * blockDim.x)
        f[dst + i] = f[src + i];
}

}  // namespace d3
}  // namespace kb

extern "C" int kb_slab_fill_ghosts_3d(void *f, int Nx, int Ny, int nz_alloc, int lo, int hi,
                                      int dtype, void *stream) {
    using namespace kb::d3;
    KB_REQUIRE(f, "kb_slab_fill_ghosts_3d: null population pointer");
    if (int e = check_dims("kb_slab_fill_ghosts_3d", Nx, Ny, nz_alloc)) return e;
    KB_REQUIRE(nz_alloc >= 1 + (lo != 0) + (hi != 0),
               "kb_slab_fill_ghosts_3d: %d planes hold no real plane besides the ghosts", nz_alloc);
    const size_t plane = (size_t)Nx * Ny, pop = plane * (size_t)nz_alloc;
    const size_t b = kb::dtype_bytes(dtype);
    KB_REQUIRE(b != 0, "kb_slab_fill_ghosts_3d: unknown dtype %d", dtype);
    const dim3 grid((unsigned)std::min<size_t>((plane + 255) / 256, 1024), 10);
    cudaStream_t s = kb::as_stream(stream);
    const int l = lo != 0, h = hi != 0;
    if (b == 8) slab_ghosts_k<unsigned long long><<<grid, 256, 0, s>>>((unsigned long long *)f, plane, pop, nz_alloc, l, h);
    else if (b == 4) slab_ghosts_k<unsigned int><<<grid, 256, 0, s>>>((unsigned int *)f, plane, pop, nz_alloc, l, h);
    else slab_ghosts_k<unsigned short><<<grid, 256, 0, s>>>((unsigned short *)f, plane, pop, nz_alloc, l, h);
    return kb::check_launch("kb_slab_fill_ghosts_3d");
}
