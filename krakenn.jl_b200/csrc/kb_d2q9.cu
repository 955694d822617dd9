// kb_d2q9.cu -- D2Q9 kernels with the reference's arithmetic.
//
// Compiled with --fmad=false: every multiply and add rounds separately, in
// the order Kraken.jl writes them, so a double run reproduces the
// reference's CPU Float64 path bit for bit (and a float run its Float32
// path).  Each kernel names the reference kernel it restates.
//
// Thread mapping: one thread per node, blockDim.x along x (the unit-stride
// axis of every population plane), so each population load/store of a warp
// is one contiguous run of 32 elements (shifted by one for the x-pulls).
#include "kb_common.cuh"

namespace kb {
namespace d3 {
// The deviation-storage form of the fused thermal DDF step lives in the
// precision-tier unit (kb_d3q19_dev.cu, compiled with FMA contraction).
int launch_natconv_dev(int dtype, bool vt, void *f_out, const void *f_in, void *g_out,
                       const void *g_in, float *Temp, int Nx, int Ny, double w_f, double w_T,
                       double beta_g, double T_ref, double T_hot, double T_cold, double nu_ref,
                       double T0_visc, double a_visc, cudaStream_t s);
}  // namespace d3
}  // namespace kb

namespace kb {
namespace d2 {

constexpr int BX = 128;

template <typename T>
struct Grid2 {
    int Nx, Ny;
    size_t plane;  // Nx*Ny
    __device__ __forceinline__ size_t at(int i, int j) const { return (size_t)i + (size_t)Nx * j; }
};

// feq_2d(Val(q), rho, ux, uy, usq): src/kernels/equilibrium_helpers.jl:8-50
template <typename T>
__device__ __forceinline__ T feq_poly(T w, T rho, T cu, T usq) {
    return w * rho * (T(1) + T(3) * cu + T(4.5) * cu * cu - T(1.5) * usq);
}

template <typename T>
__device__ __forceinline__ void feq_all(T rho, T ux, T uy, T usq, T *feq) {
    const T w0 = T(4.0 / 9.0), w1 = T(1.0 / 9.0), w5 = T(1.0 / 36.0);
    feq[0] = w0 * rho * (T(1) - T(1.5) * usq);
    feq[1] = feq_poly(w1, rho, ux, usq);
    feq[2] = feq_poly(w1, rho, uy, usq);
    feq[3] = feq_poly(w1, rho, -ux, usq);
    feq[4] = feq_poly(w1, rho, -uy, usq);
    feq[5] = feq_poly(w5, rho, ux + uy, usq);
    feq[6] = feq_poly(w5, rho, -ux + uy, usq);
    feq[7] = feq_poly(w5, rho, -ux - uy, usq);
    feq[8] = feq_poly(w5, rho, ux - uy, usq);
}

// moments_2d: src/kernels/equilibrium_helpers.jl:54-61
template <typename T>
__device__ __forceinline__ void moments(const T *p, T &rho, T &ux, T &uy) {
    rho = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8];
    T inv = T(1) / rho;
    ux = (p[1] - p[3] + p[5] - p[6] - p[7] + p[8]) * inv;
    uy = (p[2] - p[4] + p[5] + p[6] - p[7] - p[8]) * inv;
}

// Pull with half-way bounce-back on the four edges:
// src/kernels/collide_stream_2d.jl:12-23 (same in fused_bgk_2d.jl:13-24).
template <typename T>
__device__ __forceinline__ void pull_bb(const T *__restrict__ f, const Grid2<T> &g, int i, int j,
                                        T *fp) {
    const int Nx = g.Nx, Ny = g.Ny;
    const size_t P = g.plane;
    const bool w = i > 0, e = i < Nx - 1, s = j > 0, n = j < Ny - 1;
    const size_t c = g.at(i, j);
    fp[0] = f[c];
    fp[1] = w ? f[c - 1 + 1 * P] : f[c + 3 * P];
    fp[2] = s ? f[c - Nx + 2 * P] : f[c + 4 * P];
    fp[3] = e ? f[c + 1 + 3 * P] : f[c + 1 * P];
    fp[4] = n ? f[c + Nx + 4 * P] : f[c + 2 * P];
    fp[5] = (w && s) ? f[c - 1 - Nx + 5 * P] : f[c + 7 * P];
    fp[6] = (e && s) ? f[c + 1 - Nx + 6 * P] : f[c + 8 * P];
    fp[7] = (e && n) ? f[c + 1 + Nx + 7 * P] : f[c + 5 * P];
    fp[8] = (w && n) ? f[c - 1 + Nx + 8 * P] : f[c + 6 * P];
}

template <typename T>
__device__ __forceinline__ void swap_pairs(T *p) {
    T t;
    t = p[1]; p[1] = p[3]; p[3] = t;
    t = p[2]; p[2] = p[4]; p[4] = t;
    t = p[5]; p[5] = p[7]; p[7] = t;
    t = p[6]; p[6] = p[8]; p[8] = t;
}

template <typename T>
__device__ __forceinline__ void bgk(T *p, T omega, T &rho, T &ux, T &uy) {
    T feq[9];
    moments(p, rho, ux, uy);
    T usq = ux * ux + uy * uy;
    feq_all(rho, ux, uy, usq, feq);
#pragma unroll
    for (int q = 0; q < 9; ++q) p[q] = p[q] - omega * (p[q] - feq[q]);
}

#define NODE2                                              \
    const int i = blockIdx.x * blockDim.x + threadIdx.x;   \
    const int j = blockIdx.y;                              \
    if (i >= g.Nx) return;                                 \
    const size_t c = g.at(i, j);                           \
    const size_t P = g.plane;

// equilibrium(::D2Q9, rho, ux, uy, q) (src/lattice/d2q9.jl:60-67) at every
// node, as the reference's initialisers fill f (src/drivers/basic.jl:265).
// Fields may be FP32 for FP64 populations (a warm start from a prediction).
template <typename T, typename F>
__global__ void __launch_bounds__(BX) equilibrium_k(T *__restrict__ f, const F *__restrict__ rho,
                                                     const F *__restrict__ ux,
                                                     const F *__restrict__ uy, Grid2<T> g) {
    NODE2
    const T r = (T)rho[c], a = (T)ux[c], b = (T)uy[c];
    const T usq = a * a + b * b;
    T feq[9];
    feq_all(r, a, b, usq, feq);
#pragma unroll
    for (int q = 0; q < 9; ++q) f[c + q * P] = feq[q];
}

// stream_2d_kernel!: src/kernels/collide_stream_2d.jl:5-31
template <typename T>
__global__ void __launch_bounds__(BX) stream_k(T *__restrict__ fo, const T *__restrict__ fi, Grid2<T> g) {
    NODE2
    T p[9];
    pull_bb(fi, g, i, j, p);
#pragma unroll
    for (int q = 0; q < 9; ++q) fo[c + q * P] = p[q];
}

// collide_2d_kernel!: src/kernels/collide_stream_2d.jl:35-61
template <typename T>
__global__ void __launch_bounds__(BX) collide_k(T *__restrict__ f, const uint8_t *__restrict__ solid,
                                                 Grid2<T> g, T omega) {
    NODE2
    T p[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) p[q] = f[c + q * P];
    if (solid && solid[c]) {
        swap_pairs(p);
    } else {
        T rho, ux, uy;
        bgk(p, omega, rho, ux, uy);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) f[c + q * P] = p[q];
}

// zou_he_velocity_north_2d_kernel!: src/kernels/boundary_2d.jl:13-42
template <typename T>
__device__ __forceinline__ void zou_he_north_node(T *p, T u) {
    T rw = (p[0] + p[1] + p[3] + T(2) * (p[2] + p[5] + p[6])) / (T(1) + u * T(0));
    T f2 = p[1], f4 = p[3], f6 = p[5], f7 = p[6];
    p[4] = p[2];
    p[8] = f7 - T(0.5) * (f2 - f4) + T(0.5) * rw * u;
    p[7] = f6 + T(0.5) * (f2 - f4) - T(0.5) * rw * u;
}

template <typename T>
__global__ void zou_he_north_k(T *__restrict__ f, Grid2<T> g, T u) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.Nx) return;
    const size_t c = g.at(i, g.Ny - 1), P = g.plane;
    T p[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) p[q] = f[c + q * P];
    zou_he_north_node(p, u);
    f[c + 4 * P] = p[4];
    f[c + 8 * P] = p[8];
    f[c + 7 * P] = p[7];
}

// zou_he_velocity_south_2d_kernel!: src/kernels/boundary_2d.jl:135-149
template <typename T>
__global__ void zou_he_south_k(T *__restrict__ f, Grid2<T> g, T u) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.Nx) return;
    const size_t c = g.at(i, 0), P = g.plane;
    T f1 = f[c], f2 = f[c + P], f4 = f[c + 3 * P], f5 = f[c + 4 * P], f8 = f[c + 7 * P],
      f9 = f[c + 8 * P];
    T rw = f1 + f2 + f4 + T(2) * (f5 + f8 + f9);
    f[c + 2 * P] = f5;
    f[c + 5 * P] = f8 - T(0.5) * (f2 - f4) + T(0.5) * rw * u;
    f[c + 6 * P] = f9 + T(0.5) * (f2 - f4) - T(0.5) * rw * u;
}

// zou_he_velocity_west_2d_kernel!: src/kernels/boundary_2d.jl:171-184
template <typename T>
__global__ void zou_he_west_k(T *__restrict__ f, Grid2<T> g, T u) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= g.Ny) return;
    const size_t c = g.at(0, j), P = g.plane;
    T f1 = f[c], f3 = f[c + 2 * P], f4 = f[c + 3 * P], f5 = f[c + 4 * P], f7 = f[c + 6 * P],
      f8 = f[c + 7 * P];
    T rw = (f1 + f3 + f5 + T(2) * (f4 + f7 + f8)) / (T(1) - u);
    f[c + 1 * P] = f4 + T(2.0 / 3.0) * rw * u;
    f[c + 5 * P] = f8 - T(0.5) * (f3 - f5) + T(1.0 / 6.0) * rw * u;
    f[c + 8 * P] = f7 + T(0.5) * (f3 - f5) + T(1.0 / 6.0) * rw * u;
}

// zou_he_pressure_east_2d_kernel!: src/kernels/boundary_2d.jl:206-223
template <typename T>
__global__ void zou_he_pressure_east_k(T *__restrict__ f, Grid2<T> g, T rho_out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= g.Ny) return;
    const size_t c = g.at(g.Nx - 1, j), P = g.plane;
    T f1 = f[c], f2 = f[c + P], f3 = f[c + 2 * P], f5 = f[c + 4 * P], f6 = f[c + 5 * P],
      f9 = f[c + 8 * P];
    T ux = -T(1) + (f1 + f3 + f5 + T(2) * (f2 + f6 + f9)) / rho_out;
    f[c + 3 * P] = f2 - T(2.0 / 3.0) * rho_out * ux;
    f[c + 6 * P] = f9 - T(0.5) * (f3 - f5) - T(1.0 / 6.0) * rho_out * ux;
    f[c + 7 * P] = f6 + T(0.5) * (f3 - f5) - T(1.0 / 6.0) * rho_out * ux;
}

// zou_he_pressure_west_2d_kernel!: src/kernels/boundary_2d.jl:264-281
template <typename T>
__global__ void zou_he_pressure_west_k(T *__restrict__ f, Grid2<T> g, T rho_in) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= g.Ny) return;
    const size_t c = g.at(0, j), P = g.plane;
    T f1 = f[c], f3 = f[c + 2 * P], f4 = f[c + 3 * P], f5 = f[c + 4 * P], f7 = f[c + 6 * P],
      f8 = f[c + 7 * P];
    T ux = T(1) - (f1 + f3 + f5 + T(2) * (f4 + f7 + f8)) / rho_in;
    f[c + 1 * P] = f4 + T(2.0 / 3.0) * rho_in * ux;
    f[c + 5 * P] = f8 - T(0.5) * (f3 - f5) + T(1.0 / 6.0) * rho_in * ux;
    f[c + 8 * P] = f7 + T(0.5) * (f3 - f5) + T(1.0 / 6.0) * rho_in * ux;
}

// extrapolate_east_2d_kernel!: src/kernels/boundary_2d.jl:303-311
template <typename T>
__global__ void extrapolate_east_k(T *__restrict__ f, Grid2<T> g) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= g.Ny) return;
    const size_t c = g.at(g.Nx - 1, j), P = g.plane;
#pragma unroll
    for (int q = 0; q < 9; ++q) f[c + q * P] = f[c - 1 + q * P];
}

// bounce_back_walls_2d_kernel!: src/kernels/boundary_2d.jl:64-90
template <typename T>
__global__ void bounce_back_wall_k(T *__restrict__ f, Grid2<T> g, int wall_id) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t P = g.plane;
    if (wall_id == 1 || wall_id == 4) {
        if (idx >= g.Nx) return;
    } else {
        if (idx >= g.Ny) return;
    }
    if (wall_id == 1) {
        const size_t c = g.at(idx, 0);
        f[c + 2 * P] = f[c + 4 * P];
        f[c + 5 * P] = f[c + 7 * P];
        f[c + 6 * P] = f[c + 8 * P];
    } else if (wall_id == 2) {
        const size_t c = g.at(0, idx);
        f[c + 1 * P] = f[c + 3 * P];
        f[c + 5 * P] = f[c + 7 * P];
        f[c + 8 * P] = f[c + 6 * P];
    } else if (wall_id == 3) {
        const size_t c = g.at(g.Nx - 1, idx);
        f[c + 3 * P] = f[c + 1 * P];
        f[c + 6 * P] = f[c + 8 * P];
        f[c + 7 * P] = f[c + 5 * P];
    } else {
        const size_t c = g.at(idx, g.Ny - 1);
        f[c + 4 * P] = f[c + 2 * P];
        f[c + 7 * P] = f[c + 5 * P];
        f[c + 8 * P] = f[c + 6 * P];
    }
}

// compute_macroscopic_2d_kernel!: src/kernels/macroscopic.jl:5-18
template <typename T>
__device__ __forceinline__ void macro_node(const T *p, T &r, T &ux, T &uy) {
    r = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8];
    T inv = T(1) / r;
    ux = (p[1] - p[3] + p[5] - p[6] - p[7] + p[8]) * inv;
    uy = (p[2] - p[4] + p[5] + p[6] - p[7] - p[8]) * inv;
}

template <typename T>
__global__ void __launch_bounds__(BX) macroscopic_k(T *__restrict__ rho, T *__restrict__ ux,
                                                     T *__restrict__ uy, const T *__restrict__ f,
                                                     Grid2<T> g) {
    NODE2
    T p[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) p[q] = f[c + q * P];
    T r, a, b;
    macro_node(p, r, a, b);
    rho[c] = r; ux[c] = a; uy[c] = b;
}

// fused_bgk_step_kernel!: src/kernels/fused_bgk_2d.jl:8-59
template <typename T>
__global__ void __launch_bounds__(BX) fused_bgk_k(T *__restrict__ fo, const T *__restrict__ fi,
                                                   T *__restrict__ rho, T *__restrict__ ux,
                                                   T *__restrict__ uy,
                                                   const uint8_t *__restrict__ solid, Grid2<T> g,
                                                   T omega) {
    NODE2
    T p[9];
    pull_bb(fi, g, i, j, p);
    T r, a, b;
    if (solid && solid[c]) {
        swap_pairs(p);
        r = T(1); a = T(0); b = T(0);
    } else {
        bgk(p, omega, r, a, b);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) fo[c + q * P] = p[q];
    rho[c] = r; ux[c] = a; uy[c] = b;
}

// fused_trt_step_kernel!: src/kernels/fused_trt_2d.jl:29-101
template <typename T>
__global__ void __launch_bounds__(BX) fused_trt_k(T *__restrict__ fo, const T *__restrict__ fi,
                                                   T *__restrict__ rho, T *__restrict__ ux,
                                                   T *__restrict__ uy,
                                                   const uint8_t *__restrict__ solid, Grid2<T> g,
                                                   T sp, T sm) {
    NODE2
    T p[9];
    pull_bb(fi, g, i, j, p);
    T r, a_, b_;
    if (solid && solid[c]) {
        swap_pairs(p);
#pragma unroll
        for (int q = 0; q < 9; ++q) fo[c + q * P] = p[q];
        rho[c] = T(1); ux[c] = T(0); uy[c] = T(0);
        return;
    }
    T feq[9];
    moments(p, r, a_, b_);
    T usq = a_ * a_ + b_ * b_;
    feq_all(r, a_, b_, usq, feq);
    const T a = (sp + sm) * T(0.5), b = (sp - sm) * T(0.5);
    fo[c + 0 * P] = p[0] - sp * (p[0] - feq[0]);
    fo[c + 1 * P] = p[1] - a * (p[1] - feq[1]) - b * (p[3] - feq[3]);
    fo[c + 3 * P] = p[3] - a * (p[3] - feq[3]) - b * (p[1] - feq[1]);
    fo[c + 2 * P] = p[2] - a * (p[2] - feq[2]) - b * (p[4] - feq[4]);
    fo[c + 4 * P] = p[4] - a * (p[4] - feq[4]) - b * (p[2] - feq[2]);
    fo[c + 5 * P] = p[5] - a * (p[5] - feq[5]) - b * (p[7] - feq[7]);
    fo[c + 7 * P] = p[7] - a * (p[7] - feq[7]) - b * (p[5] - feq[5]);
    fo[c + 6 * P] = p[6] - a * (p[6] - feq[6]) - b * (p[8] - feq[8]);
    fo[c + 8 * P] = p[8] - a * (p[8] - feq[8]) - b * (p[6] - feq[6]);
    rho[c] = r; ux[c] = a_; uy[c] = b_;
}

// _libb_branch (src/kernels/li_bb_2d.jl:70-83): Bouzidi interpolated
// bounce-back of one cut link at wall distance q_w in (0, 1].
template <typename T>
__device__ __forceinline__ T libb_branch(T q_w, T f_here, T f_back, T f_bar_here, T d) {
    if (q_w <= T(0.5)) return T(2) * q_w * f_here + (T(1) - T(2) * q_w) * f_back + d;
    const T inv = T(1) / (T(2) * q_w);
    return inv * f_here + (T(1) - inv) * f_bar_here + d * inv;
}

// ApplyLiBBPrePhase (src/kernels/dsl/bricks.jl:516-560): for each cut link q
// (q_wall[q] > 0) the pulled population of the opposite direction, which
// came from a solid node, is replaced by the Bouzidi estimate from the
// node's own previous post-collision populations.  Pairs in the reference
// order; the second link of a pair sees the first one's substitution.
// qw/ux/uy point at the node in planes of stride P.
template <typename T>
__device__ __forceinline__ void libb_prephase_2d(const T *__restrict__ f0, const T *__restrict__ qw,
                                                 const T *__restrict__ uwx,
                                                 const T *__restrict__ uwy, size_t P, T *p) {
    const T c23 = T(2.0 / 3.0), c16 = T(1.0 / 6.0);
    T q;
    if ((q = qw[1 * P]) > T(0)) p[3] = libb_branch(q, f0[1 * P], p[1], f0[3 * P], -c23 * uwx[1 * P]);
    if ((q = qw[3 * P]) > T(0)) p[1] = libb_branch(q, f0[3 * P], p[3], f0[1 * P], c23 * uwx[3 * P]);
    if ((q = qw[2 * P]) > T(0)) p[4] = libb_branch(q, f0[2 * P], p[2], f0[4 * P], -c23 * uwy[2 * P]);
    if ((q = qw[4 * P]) > T(0)) p[2] = libb_branch(q, f0[4 * P], p[4], f0[2 * P], c23 * uwy[4 * P]);
    if ((q = qw[5 * P]) > T(0))
        p[7] = libb_branch(q, f0[5 * P], p[5], f0[7 * P], -c16 * (uwx[5 * P] + uwy[5 * P]));
    if ((q = qw[7 * P]) > T(0))
        p[5] = libb_branch(q, f0[7 * P], p[7], f0[5 * P], c16 * (uwx[7 * P] + uwy[7 * P]));
    if ((q = qw[6 * P]) > T(0))
        p[8] = libb_branch(q, f0[6 * P], p[6], f0[8 * P], -c16 * (-uwx[6 * P] + uwy[6 * P]));
    if ((q = qw[8 * P]) > T(0))
        p[6] = libb_branch(q, f0[8 * P], p[8], f0[6 * P], c16 * (-uwx[8 * P] + uwy[8 * P]));
}

// fused_trt_libb_v2_step! (src/kernels/li_bb_2d_v2.jl:35-41, 104-115):
// PullHalfwayBB -> SolidInert | ApplyLiBBPrePhase -> Moments ->
// CollideTRTDirect -> WriteMoments.  Moments are written when rho != NULL.
template <typename T>
__global__ void __launch_bounds__(BX) fused_trt_libb_k(T *__restrict__ fo, const T *__restrict__ fi,
                                                        T *__restrict__ rho, T *__restrict__ ux,
                                                        T *__restrict__ uy,
                                                        const uint8_t *__restrict__ solid,
                                                        const T *__restrict__ qw,
                                                        const T *__restrict__ uwx,
                                                        const T *__restrict__ uwy, Grid2<T> g, T sp,
                                                        T sm) {
    NODE2
    T feq[9];
    if (solid && solid[c]) {
        // SolidInert (bricks.jl:133-150): rest equilibrium w_q
        feq_all(T(1), T(0), T(0), T(0), feq);
#pragma unroll
        for (int q = 0; q < 9; ++q) fo[c + q * P] = feq[q];
        if (rho) { rho[c] = T(1); ux[c] = T(0); uy[c] = T(0); }
        return;
    }
    T p[9];
    pull_bb(fi, g, i, j, p);
    libb_prephase_2d(fi + c, qw + c, uwx + c, uwy + c, P, p);
    T r, a_, b_;
    moments(p, r, a_, b_);
    const T usq = a_ * a_ + b_ * b_;
    feq_all(r, a_, b_, usq, feq);
    const T a = (sp + sm) * T(0.5), b = (sp - sm) * T(0.5);
    fo[c + 0 * P] = p[0] - sp * (p[0] - feq[0]);
    fo[c + 1 * P] = p[1] - a * (p[1] - feq[1]) - b * (p[3] - feq[3]);
    fo[c + 3 * P] = p[3] - a * (p[3] - feq[3]) - b * (p[1] - feq[1]);
    fo[c + 2 * P] = p[2] - a * (p[2] - feq[2]) - b * (p[4] - feq[4]);
    fo[c + 4 * P] = p[4] - a * (p[4] - feq[4]) - b * (p[2] - feq[2]);
    fo[c + 5 * P] = p[5] - a * (p[5] - feq[5]) - b * (p[7] - feq[7]);
    fo[c + 7 * P] = p[7] - a * (p[7] - feq[7]) - b * (p[5] - feq[5]);
    fo[c + 6 * P] = p[6] - a * (p[6] - feq[6]) - b * (p[8] - feq[8]);
    fo[c + 8 * P] = p[8] - a * (p[8] - feq[8]) - b * (p[6] - feq[6]);
    if (rho) { rho[c] = r; ux[c] = a_; uy[c] = b_; }
}

// In-place A-A streaming (one population buffer), the scheme that
// aa_even_step!/aa_odd_step! (src/kernels/aa_bgk_2d.jl:14-143) aim at.  The
// reference's two kernels read and write slots that neighbouring nodes write
// in the same launch (its even kernel pulls a neighbour's slot that the
// neighbour overwrites; its odd kernel has two writers for a wall slot), so
// their result depends on execution order.  These two kernels are race free:
// every slot is read and written by one thread only.
//   state S: slot qb(x) = post-collision f_q(x), not yet streamed
//   state P: slot q(x)  = f_q arriving at x (post-stream, pre-collision)
// aa_stream (S -> P): gather p_q from slot qb(x - c_q) (half-way bounce-back:
//   slot q(x) when x - c_q is outside), collide, scatter to slot q(x + c_q)
//   (slot qb(x) when x + c_q is outside).
// aa_local (P -> S): read slot q(x), collide, write slot qb(x).
// A buffer in the pull kernels' format F (slot q(x) = f*_q(x)) is state S
// after swapping q <-> qb; stream then local is exactly two fused pull-BGK
// steps (fused_bgk_2d.jl:8-59), bit for bit, including the solid-node swap
// and the moments (written when rho/ux/uy are given).
__device__ constexpr int kOpp9[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};

template <typename T>
__device__ __forceinline__ void aa_collide(T *p, bool is_solid, T omega, T &r, T &a, T &b) {
    if (is_solid) {
        swap_pairs(p);
        r = T(1); a = T(0); b = T(0);
    } else {
        bgk(p, omega, r, a, b);
    }
}

template <typename T>
__global__ void __launch_bounds__(BX) aa_stream_k(T *__restrict__ f, T *__restrict__ rho,
                                                   T *__restrict__ ux, T *__restrict__ uy,
                                                   const uint8_t *__restrict__ solid, Grid2<T> g,
                                                   T omega) {
    NODE2
    const int Nx = g.Nx, Ny = g.Ny;
    const bool w = i > 0, e = i < Nx - 1, s = j > 0, n = j < Ny - 1;
    // source (x - c_q) exists?  destination (x + c_q) exists?
    const bool src[9] = {true, w, s, e, n, w && s, e && s, e && n, w && n};
    const bool dst[9] = {true, e, n, w, s, e && n, w && n, w && s, e && s};
    const long long off[9] = {0, 1, (long long)Nx, -1, -(long long)Nx, 1 + (long long)Nx,
                              -1 + (long long)Nx, -1 - (long long)Nx, 1 - (long long)Nx};
    T p[9];
#pragma unroll
    for (int q = 0; q < 9; ++q)
        p[q] = src[q] ? f[c - off[q] + kOpp9[q] * P] : f[c + q * P];
    T r, a, b;
    aa_collide(p, solid && solid[c], omega, r, a, b);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        if (dst[q]) f[c + off[q] + q * P] = p[q];
        else f[c + kOpp9[q] * P] = p[q];
    }
    if (rho) { rho[c] = r; ux[c] = a; uy[c] = b; }
}

template <typename T>
__global__ void __launch_bounds__(BX) aa_local_k(T *__restrict__ f, T *__restrict__ rho,
                                                  T *__restrict__ ux, T *__restrict__ uy,
                                                  const uint8_t *__restrict__ solid, Grid2<T> g,
                                                  T omega) {
    NODE2
    T p[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) p[q] = f[c + q * P];
    T r, a, b;
    aa_collide(p, solid && solid[c], omega, r, a, b);
#pragma unroll
    for (int q = 0; q < 9; ++q) f[c + kOpp9[q] * P] = p[q];
    if (rho) { rho[c] = r; ux[c] = a; uy[c] = b; }
}

// collide_mrt_2d_kernel! node update: src/kernels/collide_mrt_2d.jl:54-106.
// With FIXED_U the equilibria use the prescribed velocity (ux_g, uy_g) and
// the momentum is reset to rho * u_g: the iteration of Mei, Luo, Lallemand
// and d'Humieres (2006, "Consistent initial conditions for lattice
// Boltzmann simulations", Computers & Fluids 35) that makes rho and the
// non-equilibrium populations consistent with a given velocity field.
// Without FIXED_U the arithmetic is the reference's, operation for operation.
template <typename T, bool FIXED_U = false>
__device__ __forceinline__ void mrt_node(T *p, T s_e, T s_eps, T s_q, T s_nu, T ux_g = T(0),
                                         T uy_g = T(0)) {
    const T f1 = p[0], f2 = p[1], f3 = p[2], f4 = p[3], f5 = p[4], f6 = p[5], f7 = p[6],
            f8 = p[7], f9 = p[8];
    T rho = f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8 + f9;
    T e = -T(4) * f1 - f2 - f3 - f4 - f5 + T(2) * (f6 + f7 + f8 + f9);
    T eps = T(4) * f1 - T(2) * (f2 + f3 + f4 + f5) + f6 + f7 + f8 + f9;
    T jx = f2 - f4 + f6 - f7 - f8 + f9;
    T qx = -T(2) * f2 + T(2) * f4 + f6 - f7 - f8 + f9;
    T jy = f3 - f5 + f6 + f7 - f8 - f9;
    T qy = -T(2) * f3 + T(2) * f5 + f6 + f7 - f8 - f9;
    T pxx = f2 - f3 + f4 - f5;
    T pxy = f6 - f7 + f8 - f9;
    T inv = T(1) / rho;
    T ux = jx * inv, uy = jy * inv;
    if (FIXED_U) {
        ux = ux_g;
        uy = uy_g;
        jx = rho * ux;
        jy = rho * uy;
    }
    T usq = ux * ux + uy * uy;
    T e_eq = -T(2) * rho + T(3) * rho * usq;
    T eps_eq = rho - T(3) * rho * usq;
    T qx_eq = -rho * ux;
    T qy_eq = -rho * uy;
    T pxx_eq = rho * (ux * ux - uy * uy);
    T pxy_eq = rho * ux * uy;
    T es = e - s_e * (e - e_eq);
    T ep = eps - s_eps * (eps - eps_eq);
    T qxs = qx - s_q * (qx - qx_eq);
    T qys = qy - s_q * (qy - qy_eq);
    T ps = pxx - s_nu * (pxx - pxx_eq);
    T pxys = pxy - s_nu * (pxy - pxy_eq);
    const T r = rho, jxs = jx, jys = jy;
    const T c9 = T(1.0 / 9.0), c36 = T(1.0 / 36.0), c18 = T(1.0 / 18.0), c6 = T(1.0 / 6.0),
            c4 = T(1.0 / 4.0), c12 = T(1.0 / 12.0);
    p[0] = c9 * r - c9 * es + c9 * ep;
    p[1] = c9 * r - c36 * es - c18 * ep + c6 * jxs - c6 * qxs + c4 * ps;
    p[2] = c9 * r - c36 * es - c18 * ep + c6 * jys - c6 * qys - c4 * ps;
    p[3] = c9 * r - c36 * es - c18 * ep - c6 * jxs + c6 * qxs + c4 * ps;
    p[4] = c9 * r - c36 * es - c18 * ep - c6 * jys + c6 * qys - c4 * ps;
    p[5] = c9 * r + c18 * es + c36 * ep + c6 * jxs + c12 * qxs + c6 * jys + c12 * qys + c4 * pxys;
    p[6] = c9 * r + c18 * es + c36 * ep - c6 * jxs - c12 * qxs + c6 * jys + c12 * qys - c4 * pxys;
    p[7] = c9 * r + c18 * es + c36 * ep - c6 * jxs - c12 * qxs - c6 * jys - c12 * qys + c4 * pxys;
    p[8] = c9 * r + c18 * es + c36 * ep + c6 * jxs + c12 * qxs - c6 * jys - c12 * qys - c4 * pxys;
}

// collide_mrt_2d_kernel!: src/kernels/collide_mrt_2d.jl:43-109
template <typename T>
__global__ void __launch_bounds__(BX) mrt_k(T *__restrict__ f, const uint8_t *__restrict__ solid,
                                             Grid2<T> g, T s_e, T s_eps, T s_q, T s_nu) {
    NODE2
    T p[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) p[q] = f[c + q * P];
    if (solid && solid[c]) swap_pairs(p);
    else mrt_node(p, s_e, s_eps, s_q, s_nu);
#pragma unroll
    for (int q = 0; q < 9; ++q) f[c + q * P] = p[q];
}

// One step of the MRT cavity loop of test/test_mrt.jl:19-25 (stream_2d! ->
// apply_zou_he_north_2d! -> collide_mrt_2d! -> compute_macroscopic_2d!) in
// one launch; node-local after the pull, so the bits are the same.
template <typename T>
__global__ void __launch_bounds__(BX) cavity_mrt_step_k(T *__restrict__ fo, const T *__restrict__ fi,
                                                         T *__restrict__ rho, T *__restrict__ ux,
                                                         T *__restrict__ uy,
                                                         const uint8_t *__restrict__ solid,
                                                         Grid2<T> g, T s_e, T s_eps, T s_q,
                                                         T s_nu, T u_lid) {
    NODE2
    T p[9];
    pull_bb(fi, g, i, j, p);
    if (j == g.Ny - 1) zou_he_north_node(p, u_lid);
    if (solid && solid[c]) swap_pairs(p);
    else mrt_node(p, s_e, s_eps, s_q, s_nu);
#pragma unroll
    for (int q = 0; q < 9; ++q) fo[c + q * P] = p[q];
    if (rho) {
        T r, a, b;
        macro_node(p, r, a, b);
        rho[c] = r; ux[c] = a; uy[c] = b;
    }
}

// One consistent-initialisation iteration of the MRT cavity: the step above
// with the collision's velocity held at the given field (mrt_node<FIXED_U>).
template <typename T, typename F>
__global__ void __launch_bounds__(BX) cavity_mrt_fixed_u_k(T *__restrict__ fo, const T *__restrict__ fi,
                                                            const F *__restrict__ ux_g,
                                                            const F *__restrict__ uy_g,
                                                            const uint8_t *__restrict__ solid,
                                                            Grid2<T> g, T s_e, T s_eps, T s_q,
                                                            T s_nu, T u_lid) {
    NODE2
    T p[9];
    pull_bb(fi, g, i, j, p);
    if (j == g.Ny - 1) zou_he_north_node(p, u_lid);
    if (solid && solid[c]) swap_pairs(p);
    else mrt_node<T, true>(p, s_e, s_eps, s_q, s_nu, (T)ux_g[c], (T)uy_g[c]);
#pragma unroll
    for (int q = 0; q < 9; ++q) fo[c + q * P] = p[q];
}

// stream_fully_periodic_2d_kernel!: src/kernels/stream_periodic_2d.jl:79-98
template <typename T>
__global__ void __launch_bounds__(BX) stream_periodic_k(T *__restrict__ fo, const T *__restrict__ fi,
                                                         Grid2<T> g) {
    NODE2
    const int Nx = g.Nx, Ny = g.Ny;
    const int ip = i > 0 ? i - 1 : Nx - 1, im = i < Nx - 1 ? i + 1 : 0;
    const int jp = j > 0 ? j - 1 : Ny - 1, jm = j < Ny - 1 ? j + 1 : 0;
    fo[c + 0 * P] = fi[g.at(i, j) + 0 * P];
    fo[c + 1 * P] = fi[g.at(ip, j) + 1 * P];
    fo[c + 2 * P] = fi[g.at(i, jp) + 2 * P];
    fo[c + 3 * P] = fi[g.at(im, j) + 3 * P];
    fo[c + 4 * P] = fi[g.at(i, jm) + 4 * P];
    fo[c + 5 * P] = fi[g.at(ip, jp) + 5 * P];
    fo[c + 6 * P] = fi[g.at(im, jp) + 6 * P];
    fo[c + 7 * P] = fi[g.at(im, jm) + 7 * P];
    fo[c + 8 * P] = fi[g.at(ip, jm) + 8 * P];
}

// stream_periodic_x_wall_y_2d_kernel!: src/kernels/stream_periodic_2d.jl:5-55
template <typename T>
__global__ void __launch_bounds__(BX) stream_px_wy_k(T *__restrict__ fo, const T *__restrict__ fi,
                                                      Grid2<T> g) {
    NODE2
    const int Nx = g.Nx, Ny = g.Ny;
    const int jm1 = j > 0 ? j - 1 : j, jp1 = j < Ny - 1 ? j + 1 : j;
    const int iw = i > 0 ? i - 1 : Nx - 1, ie = i < Nx - 1 ? i + 1 : 0;
    fo[c + 0 * P] = fi[c];
    fo[c + 1 * P] = fi[g.at(iw, j) + 1 * P];
    fo[c + 2 * P] = j > 0 ? fi[g.at(i, jm1) + 2 * P] : fi[c + 4 * P];
    fo[c + 3 * P] = fi[g.at(ie, j) + 3 * P];
    fo[c + 4 * P] = j < Ny - 1 ? fi[g.at(i, jp1) + 4 * P] : fi[c + 2 * P];
    fo[c + 5 * P] = j > 0 ? fi[g.at(iw, jm1) + 5 * P] : fi[c + 7 * P];
    fo[c + 6 * P] = j > 0 ? fi[g.at(ie, jm1) + 6 * P] : fi[c + 8 * P];
    fo[c + 7 * P] = j < Ny - 1 ? fi[g.at(ie, jp1) + 7 * P] : fi[c + 5 * P];
    fo[c + 8 * P] = j < Ny - 1 ? fi[g.at(iw, jp1) + 8 * P] : fi[c + 6 * P];
}

// One step of run_cavity_2d (src/drivers/basic.jl:121-136) in one launch.
// stream_2d -> zou_he_north (row Ny only) -> collide_2d -> macroscopic on the
// post-collision populations.  All stages after the pull touch only this node.
template <typename T>
__global__ void __launch_bounds__(BX) cavity_step_k(T *__restrict__ fo, const T *__restrict__ fi,
                                                     T *__restrict__ rho, T *__restrict__ ux,
                                                     T *__restrict__ uy,
                                                     const uint8_t *__restrict__ solid, Grid2<T> g,
                                                     T omega, T u_lid) {
    NODE2
    T p[9];
    pull_bb(fi, g, i, j, p);
    if (j == g.Ny - 1) zou_he_north_node(p, u_lid);
    if (solid && solid[c]) {
        swap_pairs(p);
    } else {
        T r, a, b;
        bgk(p, omega, r, a, b);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) fo[c + q * P] = p[q];
    T r, a, b;
    macro_node(p, r, a, b);
    rho[c] = r; ux[c] = a; uy[c] = b;
}

// Lid-driven cavity step with a moving-wall half-way bounce-back lid: the
// DSL composition PullHalfwayBB -> ApplyHalfwayBBPrePhase -> Moments ->
// CollideBGK -> WriteMoments; the lid link rule is
// src/kernels/dsl/bricks.jl:447-487 with the top row's north-pointing links
// (reference q = 3, 6, 7) cut by a wall moving at (u_lid, 0), corners
// included.  Moments are the pre-collision ones, as in fused_bgk_step!.
template <typename T>
__global__ void __launch_bounds__(BX) cavity_movingwall_k(T *__restrict__ fo, const T *__restrict__ fi,
                                                           T *__restrict__ rho, T *__restrict__ ux,
                                                           T *__restrict__ uy,
                                                           const uint8_t *__restrict__ solid,
                                                           Grid2<T> g, T omega, T u_lid) {
    NODE2
    T p[9];
    pull_bb(fi, g, i, j, p);
    T r, a, b;
    if (solid && solid[c]) {
        swap_pairs(p);
        r = T(1); a = T(0); b = T(0);
    } else {
        if (j == g.Ny - 1) {
            const T d5 = -T(2.0 / 3.0) * T(0);
            const T d8 = -T(1.0 / 6.0) * (u_lid + T(0));
            const T d9 = -T(1.0 / 6.0) * (-u_lid + T(0));
            p[4] = fi[c + 2 * P] + d5;
            p[7] = fi[c + 5 * P] + d8;
            p[8] = fi[c + 6 * P] + d9;
        }
        bgk(p, omega, r, a, b);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) fo[c + q * P] = p[q];
    if (rho) { rho[c] = r; ux[c] = a; uy[c] = b; }
}

// ------------------------------------------------------------ thermal DDF --
// src/kernels/fused_thermal_2d.jl:37-151, 178-238.
template <typename T>
__device__ __forceinline__ void thermal_bc(T *gp, int i, int Nx, T T_hot, T T_cold) {
    if (i == 0) {
        gp[1] = -gp[1] + T(2) * T(1.0 / 9.0) * T_hot;
        gp[5] = -gp[5] + T(2) * T(1.0 / 36.0) * T_hot;
        gp[8] = -gp[8] + T(2) * T(1.0 / 36.0) * T_hot;
    }
    if (i == Nx - 1) {
        gp[3] = -gp[3] + T(2) * T(1.0 / 9.0) * T_cold;
        gp[6] = -gp[6] + T(2) * T(1.0 / 36.0) * T_cold;
        gp[7] = -gp[7] + T(2) * T(1.0 / 36.0) * T_cold;
    }
}

template <typename T>
__device__ __forceinline__ void collide_thermal(T *g, T ux, T uy, T wT) {
    const T Tm = g[0] + g[1] + g[2] + g[3] + g[4] + g[5] + g[6] + g[7] + g[8];
    const T t3 = T(3), c0 = T(4.0 / 9.0), c1 = T(1.0 / 9.0), c5 = T(1.0 / 36.0);
    T geq;
    geq = c0 * Tm;                         g[0] = g[0] - wT * (g[0] - geq);
    geq = c1 * Tm * (T(1) + t3 * ux);      g[1] = g[1] - wT * (g[1] - geq);
    geq = c1 * Tm * (T(1) + t3 * uy);      g[2] = g[2] - wT * (g[2] - geq);
    geq = c1 * Tm * (T(1) - t3 * ux);      g[3] = g[3] - wT * (g[3] - geq);
    geq = c1 * Tm * (T(1) - t3 * uy);      g[4] = g[4] - wT * (g[4] - geq);
    geq = c5 * Tm * (T(1) + t3 * (ux + uy));   g[5] = g[5] - wT * (g[5] - geq);
    geq = c5 * Tm * (T(1) + t3 * (-ux + uy));  g[6] = g[6] - wT * (g[6] - geq);
    geq = c5 * Tm * (T(1) + t3 * (-ux - uy));  g[7] = g[7] - wT * (g[7] - geq);
    geq = c5 * Tm * (T(1) + t3 * (ux - uy));   g[8] = g[8] - wT * (g[8] - geq);
}

// BGK with the Guo source of the body force (fx, fy): collide_guo_2d_kernel!
// (src/kernels/collide_guo_2d.jl:5-81); with fx = 0 and fy the buoyancy it is
// collide_boussinesq_node (fused_thermal_2d.jl:115-151).  ux, uy are the
// force-corrected velocities.
template <typename T>
__device__ __forceinline__ void collide_guo(T *f, T rho, T ux, T uy, T fx, T fy, T w) {
    const T usq = ux * ux + uy * uy;
    const T gp = T(1) - w / T(2);
    const T t3 = T(3), c0 = T(4.0 / 9.0), c1 = T(1.0 / 9.0), c5 = T(1.0 / 36.0), n9 = T(9);
    T feq[9], S[9];
    feq_all(rho, ux, uy, usq, feq);
    S[0] = c0 * ((-ux) * fx + (-uy) * fy) * t3;
    S[1] = c1 * ((T(1) - ux) * fx + (-uy) * fy) * t3 + c1 * ux * fx * n9;
    S[2] = c1 * ((-ux) * fx + (T(1) - uy) * fy) * t3 + c1 * uy * fy * n9;
    S[3] = c1 * ((-T(1) - ux) * fx + (-uy) * fy) * t3 + c1 * ux * fx * n9;
    S[4] = c1 * ((-ux) * fx + (-T(1) - uy) * fy) * t3 + c1 * uy * fy * n9;
    S[5] = c5 * ((T(1) - ux) * fx + (T(1) - uy) * fy) * t3 + c5 * (ux + uy) * (fx + fy) * n9;
    S[6] = c5 * ((-T(1) - ux) * fx + (T(1) - uy) * fy) * t3 + c5 * (-ux + uy) * (-fx + fy) * n9;
    S[7] = c5 * ((-T(1) - ux) * fx + (-T(1) - uy) * fy) * t3 + c5 * (-ux - uy) * (-fx - fy) * n9;
    S[8] = c5 * ((T(1) - ux) * fx + (-T(1) - uy) * fy) * t3 + c5 * (ux - uy) * (fx - fy) * n9;
#pragma unroll
    for (int q = 0; q < 9; ++q) f[q] = f[q] - w * (f[q] - feq[q]) + gp * S[q];
}

__device__ __forceinline__ double kb_exp(double x) { return exp(x); }
__device__ __forceinline__ float kb_exp(float x) { return expf(x); }

template <typename T, bool VT>
__global__ void __launch_bounds__(BX) natconv_k(T *__restrict__ fo, const T *__restrict__ fi,
                                                 T *__restrict__ go, const T *__restrict__ gi,
                                                 T *__restrict__ Temp, Grid2<T> g, T w_f, T w_T,
                                                 T beta_g, T T_ref, T T_hot, T T_cold, T nu_ref,
                                                 T T0_visc, T a_visc) {
    NODE2
    T fp[9], gp[9];
    pull_bb(fi, g, i, j, fp);
    pull_bb(gi, g, i, j, gp);
    thermal_bc(gp, i, g.Nx, T_hot, T_cold);
    const T Tl = gp[0] + gp[1] + gp[2] + gp[3] + gp[4] + gp[5] + gp[6] + gp[7] + gp[8];
    Temp[c] = Tl;
    // macroscopic_boussinesq: fused_thermal_2d.jl:61-72
    const T fy = beta_g * (Tl - T_ref);
    const T rho = fp[0] + fp[1] + fp[2] + fp[3] + fp[4] + fp[5] + fp[6] + fp[7] + fp[8];
    const T inv = T(1) / rho;
    const T ux = (fp[1] - fp[3] + fp[5] - fp[6] - fp[7] + fp[8]) * inv;
    const T uy = ((fp[2] - fp[4] + fp[5] + fp[6] - fp[7] - fp[8]) + fy / T(2)) * inv;
    collide_thermal(gp, ux, uy, w_T);
#pragma unroll
    for (int q = 0; q < 9; ++q) go[c + q * P] = gp[q];
    T w = w_f;
    if (VT) {
        // collide_boussinesq_vt_node: fused_thermal_2d.jl:155-161
        const T nul = nu_ref * kb_exp(a_visc * (Tl - T0_visc));
        w = T(1) / (T(3) * nul + T(0.5));
    }
    collide_guo(fp, rho, ux, uy, T(0), fy, w);
#pragma unroll
    for (int q = 0; q < 9; ++q) fo[c + q * P] = fp[q];
}

// compute_temperature_2d!: src/kernels/thermal_2d.jl:113-138
template <typename T>
__global__ void __launch_bounds__(BX) temperature_k(T *__restrict__ Temp, const T *__restrict__ gg,
                                                     Grid2<T> g) {
    NODE2
    Temp[c] = gg[c] + gg[c + P] + gg[c + 2 * P] + gg[c + 3 * P] + gg[c + 4 * P] + gg[c + 5 * P] +
              gg[c + 6 * P] + gg[c + 7 * P] + gg[c + 8 * P];
}

// ------------------------------------------------- unfused thermal DDF (2D) --
// collide_thermal_2d_kernel!: src/kernels/thermal_2d.jl:16-62
template <typename T>
__global__ void __launch_bounds__(BX) collide_thermal_k(T *__restrict__ gg, const T *__restrict__ ux,
                                                         const T *__restrict__ uy, Grid2<T> g, T wT) {
    NODE2
    T p[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) p[q] = gg[c + q * P];
    collide_thermal(p, ux[c], uy[c], wT);
#pragma unroll
    for (int q = 0; q < 9; ++q) gg[c + q * P] = p[q];
}

// collide_thermal_masked_2d_kernel!: src/kernels/thermal_2d.jl:83-102.  The
// equilibrium is written per population from (w_q, c_q) as the reference's
// loop writes it; skipped nodes are left untouched.
template <typename T>
__global__ void __launch_bounds__(BX) collide_thermal_masked_k(T *__restrict__ gg,
                                                                const T *__restrict__ ux,
                                                                const T *__restrict__ uy,
                                                                const uint8_t *__restrict__ skip,
                                                                Grid2<T> g, T wT) {
    NODE2
    if (skip && skip[c]) return;
    const T a = ux[c], b = uy[c];
    T p[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) p[q] = gg[c + q * P];
    const T Tm = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8];
    const T t3 = T(3);
    const int cx[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    const int cy[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const T w = q == 0 ? T(4) / T(9) : (q <= 4 ? T(1) / T(9) : T(1) / T(36));
        const T geq = w * Tm * (T(1) + t3 * (T(cx[q]) * a + T(cy[q]) * b));
        gg[c + q * P] = p[q] - wT * (p[q] - geq);
    }
}

// Half-way anti-bounce-back on one face: _fixed_temp_{west,east,south,north}_2d!
// (src/kernels/thermal_2d.jl:151-350).  Slots are 0-based (reference q - 1).
// The face's main slot always flips; each of its two corner slots uses the
// corner temperature and is left alone when its skip flag is set.
template <typename T>
struct FixedTempFace2 {
    int face;     // 0 west, 1 east, 2 south, 3 north
    T T_wall;
    T T_c[2];     // corner temperature at the low / high end of the face
    int skip[2];  // corner slot owned by the adjacent face
};

template <typename T>
struct FixedTempSet2 {
    int n;
    FixedTempFace2<T> f[4];
};

// _abb_slot (thermal_2d.jl:163-166).  A skipped corner slot is not written
// at all: in the one-launch multi-face form the face that owns it may be
// writing it at the same time.
template <typename T>
__device__ __forceinline__ void abb_slot(T *gq, T w2, T T_face, bool on_corner, T T_corner, bool skip) {
    if (on_corner && skip) return;
    const T T_link = on_corner ? T_corner : T_face;
    *gq = -*gq + w2 * T_link;
}

template <typename T>
__global__ void fixed_temp_k(T *__restrict__ gg, Grid2<T> g, FixedTempSet2<T> S) {
    const FixedTempFace2<T> F = S.f[blockIdx.y];
    const int n = threadIdx.x + blockIdx.x * blockDim.x;
    const bool xface = F.face < 2;
    const int len = xface ? g.Ny : g.Nx;
    if (n >= len) return;
    const int i = xface ? (F.face == 0 ? 0 : g.Nx - 1) : n;
    const int j = xface ? n : (F.face == 2 ? 0 : g.Ny - 1);
    const size_t c = g.at(i, j), P = g.plane;
    // main slot, low-corner slot, high-corner slot per face
    const int qm[4] = {1, 3, 2, 4}, ql[4] = {5, 6, 5, 8}, qh[4] = {8, 7, 6, 7};
    const T wa = T(2) * T(1.0 / 9.0), we = T(2) * T(1.0 / 36.0);
    const bool lo = n == 0, hi = n == len - 1;
    T *m = gg + c + qm[F.face] * P, *l = gg + c + ql[F.face] * P, *h = gg + c + qh[F.face] * P;
    *m = -*m + wa * F.T_wall;
    abb_slot(l, we, F.T_wall, lo, F.T_c[0], F.skip[0] != 0);
    abb_slot(h, we, F.T_wall, hi, F.T_c[1], F.skip[1] != 0);
}

// collide_boussinesq_2d_kernel! (src/kernels/thermal_2d.jl:421-473) and its
// nu(T) forms: MODE 1 Arrhenius (:482-539), MODE 2 modified Arrhenius
// (:593-650).  a, b: (omega) for MODE 0, (nu_ref, T_ref, A_arr) for MODE 1,
// (nu_ref, T0_visc, alpha_visc) for MODE 2.
template <typename T, int MODE>
__global__ void __launch_bounds__(BX) boussinesq_k(T *__restrict__ f, const T *__restrict__ Temp,
                                                    const uint8_t *__restrict__ solid, Grid2<T> g,
                                                    T omega, T nu_ref, T Ta, T Aa, T beta_g,
                                                    T T_ref) {
    NODE2
    T p[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) p[q] = f[c + q * P];
    if (solid && solid[c]) {
        swap_pairs(p);
    } else {
        const T Tl = Temp[c];
        T w = omega;
        if (MODE == 1) {
            const T nul = nu_ref * kb_exp(Aa * (T(1) / Tl - T(1) / Ta));
            w = T(1) / (T(3) * nul + T(0.5));
        } else if (MODE == 2) {
            const T nul = nu_ref * kb_exp(Aa * (Tl - Ta));
            w = T(1) / (T(3) * nul + T(0.5));
        }
        const T fy = beta_g * (Tl - T_ref);
        const T fx = T(0);
        const T rho = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8];
        const T inv = T(1) / rho;
        const T a = ((p[1] - p[3] + p[5] - p[6] - p[7] + p[8]) + fx / T(2)) * inv;
        const T b = ((p[2] - p[4] + p[5] + p[6] - p[7] - p[8]) + fy / T(2)) * inv;
        collide_guo(p, rho, a, b, fx, fy, w);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) f[c + q * P] = p[q];
}

// compute_macroscopic_forced_2d_kernel! (src/kernels/macroscopic.jl:84-99):
// the velocity carries the half-force correction (sum c f + F/2) / rho.
template <typename T>
__global__ void __launch_bounds__(BX) macroscopic_forced_k(T *__restrict__ rho, T *__restrict__ ux,
                                                            T *__restrict__ uy,
                                                            const T *__restrict__ f, Grid2<T> g,
                                                            T Fx, T Fy) {
    NODE2
    T p[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) p[q] = f[c + q * P];
    const T r = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8];
    const T inv = T(1) / r;
    rho[c] = r;
    ux[c] = ((p[1] - p[3] + p[5] - p[6] - p[7] + p[8]) + Fx / T(2)) * inv;
    uy[c] = ((p[2] - p[4] + p[5] + p[6] - p[7] - p[8]) + Fy / T(2)) * inv;
}

// collide_guo_2d_kernel! (src/kernels/collide_guo_2d.jl:5-81; FIELD false,
// constant force) and collide_guo_field_2d_kernel! (:93-155; FIELD true,
// per-node force).  Solid nodes swap opposite pairs.
template <typename T, bool FIELD>
__global__ void __launch_bounds__(BX) guo_k(T *__restrict__ f, const uint8_t *__restrict__ solid,
                                             const T *__restrict__ Fxf, const T *__restrict__ Fyf,
                                             Grid2<T> g, T omega, T Fx, T Fy) {
    NODE2
    T p[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) p[q] = f[c + q * P];
    if (solid && solid[c]) {
        swap_pairs(p);
    } else {
        const T fx = FIELD ? Fxf[c] : Fx, fy = FIELD ? Fyf[c] : Fy;
        const T rho = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8];
        const T inv = T(1) / rho;
        const T a = ((p[1] - p[3] + p[5] - p[6] - p[7] + p[8]) + fx / T(2)) * inv;
        const T b = ((p[2] - p[4] + p[5] + p[6] - p[7] - p[8]) + fy / T(2)) * inv;
        collide_guo(p, rho, a, b, fx, fy, omega);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) f[c + q * P] = p[q];
}

// FP32 forced BGK of two adjacent nodes per thread (even Nx, 8-byte aligned
// fields) as two lanes (Lanes2): KIND 0 collide_boussinesq_2d (force
// (0, beta_g (T - T_ref)), omega), 1 collide_guo_2d (constant force), 2
// collide_guo_field_2d (per-node force).  Each lane evaluates the expression
// tree of boussinesq_k / guo_k, with packed round-to-nearest adds and
// multiplies, to within 3 ulp of them; a solid node of the pair swaps its
// opposite populations.  I: the element offset type.
template <int KIND, typename I>
__global__ void __launch_bounds__(BX) forced2_k(float *__restrict__ f, const float *__restrict__ Temp,
                                                 const uint8_t *__restrict__ solid,
                                                 const float *__restrict__ Fxf,
                                                 const float *__restrict__ Fyf, Grid2<float> g,
                                                 float omega, float beta_g, float T_ref, float Fx,
                                                 float Fy) {
    const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int j = blockIdx.y;
    if (i >= g.Nx) return;
    const I c = (I)i + (I)g.Nx * (I)j;
    const I P = (I)g.plane;
    Lanes2 p[9], o[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) p[q].v = *reinterpret_cast<const float2 *>(f + c + q * P);
    const uchar2 sd = solid ? *reinterpret_cast<const uchar2 *>(solid + c) : make_uchar2(0, 0);
    const auto ld2 = [&](const float *a) { return Lanes2::of(*reinterpret_cast<const float2 *>(a + c)); };
    const auto sp = [](float x) { return Lanes2::of(make_float2(x, x)); };
#pragma unroll
    for (int q = 0; q < 9; ++q) o[q] = p[q];
    if (!(sd.x && sd.y)) {
        const Lanes2 fx = KIND == 0 ? Lanes2(0.0) : (KIND == 1 ? sp(Fx) : ld2(Fxf));
        const Lanes2 fy = KIND == 0 ? sp(beta_g) * (ld2(Temp) - sp(T_ref)) : (KIND == 1 ? sp(Fy) : ld2(Fyf));
        const Lanes2 rho = o[0] + o[1] + o[2] + o[3] + o[4] + o[5] + o[6] + o[7] + o[8];
        const Lanes2 inv = Lanes2(1.0) / rho;
        const Lanes2 a = ((o[1] - o[3] + o[5] - o[6] - o[7] + o[8]) + fx / Lanes2(2.0)) * inv;
        const Lanes2 b = ((o[2] - o[4] + o[5] + o[6] - o[7] - o[8]) + fy / Lanes2(2.0)) * inv;
        collide_guo(o, rho, a, b, fx, fy, sp(omega));
    }
    if (sd.x || sd.y) {
        swap_pairs(p);
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            if (sd.x) o[q].v.x = p[q].v.x;
            if (sd.y) o[q].v.y = p[q].v.y;
        }
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) *reinterpret_cast<float2 *>(f + c + q * P) = o[q].v;
}

}  // namespace d2
}  // namespace kb

// ----------------------------------------------------------- host wrappers --
namespace {

using namespace kb::d2;

template <typename T>
Grid2<T> grid2(int Nx, int Ny) {
    Grid2<T> g;
    g.Nx = Nx; g.Ny = Ny; g.plane = (size_t)Nx * (size_t)Ny;
    return g;
}

inline dim3 nodes_grid(int Nx, int Ny) { return dim3((Nx + BX - 1) / BX, Ny); }
inline unsigned line_grid(int n) { return (unsigned)((n + BX - 1) / BX); }

// Forced BGK (KIND 0 Boussinesq, 1 constant Guo force, 2 per-node Guo force):
// FP32 on even Nx with 8-byte aligned fields takes two nodes per thread
// (forced2_k), everything else one node per thread.
template <typename T, int KIND>
void launch_forced_2d(T *f, const T *Temp, const uint8_t *solid, const T *Fxf, const T *Fyf, int Nx,
                      int Ny, T omega, T beta_g, T T_ref, T Fx, T Fy, cudaStream_t s) {
    const Grid2<T> g = grid2<T>(Nx, Ny);
    if constexpr (sizeof(T) == 4) {
        const auto al = [](const void *q, uintptr_t n) { return ((uintptr_t)q & (n - 1)) == 0; };
        if (Nx % 2 == 0 && al(f, 8) && al(Temp, 8) && al(Fxf, 8) && al(Fyf, 8) && al(solid, 2)) {
            const dim3 grid((unsigned)((Nx / 2 + BX - 1) / BX), (unsigned)Ny);
            if (9.0 * (double)g.plane < 2147483647.0)
                forced2_k<KIND, int><<<grid, BX, 0, s>>>(f, Temp, solid, Fxf, Fyf, g, omega, beta_g,
                                                         T_ref, Fx, Fy);
            else
                forced2_k<KIND, size_t><<<grid, BX, 0, s>>>(f, Temp, solid, Fxf, Fyf, g, omega, beta_g,
                                                            T_ref, Fx, Fy);
            return;
        }
    }
    if (KIND == 0)
        boussinesq_k<T, 0><<<nodes_grid(Nx, Ny), BX, 0, s>>>(f, Temp, solid, g, omega, T(0), T(0), T(0),
                                                             beta_g, T_ref);
    else if (KIND == 1)
        guo_k<T, false><<<nodes_grid(Nx, Ny), BX, 0, s>>>(f, solid, nullptr, nullptr, g, omega, Fx, Fy);
    else
        guo_k<T, true><<<nodes_grid(Nx, Ny), BX, 0, s>>>(f, solid, Fxf, Fyf, g, omega, T(0), T(0));
}

int check_dims(const char *what, int Nx, int Ny) {
    if (Nx < 1 || Ny < 1 || Ny > 65535)
        return kb::set_error(KB_ERR_ARG, "%s: bad grid %d x %d (need Nx >= 1, 1 <= Ny <= 65535)",
                             what, Nx, Ny);
    return KB_OK;
}

int plain_dtype(const char *what, int dtype) {
    if (dtype != KB_F64 && dtype != KB_F32)
        return kb::set_error(KB_ERR_UNSUPPORTED,
                             "%s: dtype %d not supported (reference-arithmetic kernels take "
                             "KB_F64 or KB_F32)", what, dtype);
    return KB_OK;
}

#define KB_DISPATCH_PLAIN(what, dtype, BODY)              \
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

}  // namespace

extern "C" {

int kb_stream_2d(void *f_out, const void *f_in, int Nx, int Ny, int dtype, void *stream) {
    KB_REQUIRE(f_out && f_in, "kb_stream_2d: null population pointer");
    KB_REQUIRE(f_out != f_in, "kb_stream_2d: f_out and f_in must differ");
    if (int e = check_dims("kb_stream_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_stream_2d", dtype,
        (stream_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f_out, (const T *)f_in, grid2<T>(Nx, Ny))));
}

int kb_collide_2d(void *f, const uint8_t *is_solid, int Nx, int Ny, double omega, int dtype,
                  void *stream) {
    KB_REQUIRE(f, "kb_collide_2d: null population pointer");
    if (int e = check_dims("kb_collide_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_collide_2d", dtype,
        (collide_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f, is_solid, grid2<T>(Nx, Ny), (T)omega)));
}

int kb_apply_zou_he_north_2d(void *f, double u_wall_x, int Nx, int Ny, int dtype, void *stream) {
    KB_REQUIRE(f, "kb_apply_zou_he_north_2d: null population pointer");
    if (int e = check_dims("kb_apply_zou_he_north_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_apply_zou_he_north_2d", dtype,
        (zou_he_north_k<T><<<line_grid(Nx), BX, 0, kb::as_stream(stream)>>>(
            (T *)f, grid2<T>(Nx, Ny), (T)u_wall_x)));
}

int kb_apply_zou_he_south_2d(void *f, double u_wall_x, int Nx, int Ny, int dtype, void *stream) {
    KB_REQUIRE(f, "kb_apply_zou_he_south_2d: null population pointer");
    if (int e = check_dims("kb_apply_zou_he_south_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_apply_zou_he_south_2d", dtype,
        (zou_he_south_k<T><<<line_grid(Nx), BX, 0, kb::as_stream(stream)>>>(
            (T *)f, grid2<T>(Nx, Ny), (T)u_wall_x)));
}

int kb_apply_zou_he_west_2d(void *f, double u_in, int Nx, int Ny, int dtype, void *stream) {
    KB_REQUIRE(f, "kb_apply_zou_he_west_2d: null population pointer");
    if (int e = check_dims("kb_apply_zou_he_west_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_apply_zou_he_west_2d", dtype,
        (zou_he_west_k<T><<<line_grid(Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f, grid2<T>(Nx, Ny), (T)u_in)));
}

int kb_apply_zou_he_pressure_east_2d(void *f, int Nx, int Ny, double rho_out, int dtype,
                                     void *stream) {
    KB_REQUIRE(f, "kb_apply_zou_he_pressure_east_2d: null population pointer");
    if (int e = check_dims("kb_apply_zou_he_pressure_east_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_apply_zou_he_pressure_east_2d", dtype,
        (zou_he_pressure_east_k<T><<<line_grid(Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f, grid2<T>(Nx, Ny), (T)rho_out)));
}

int kb_apply_zou_he_pressure_west_2d(void *f, int Nx, int Ny, double rho_in, int dtype,
                                     void *stream) {
    KB_REQUIRE(f, "kb_apply_zou_he_pressure_west_2d: null population pointer");
    if (int e = check_dims("kb_apply_zou_he_pressure_west_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_apply_zou_he_pressure_west_2d", dtype,
        (zou_he_pressure_west_k<T><<<line_grid(Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f, grid2<T>(Nx, Ny), (T)rho_in)));
}

int kb_apply_extrapolate_east_2d(void *f, int Nx, int Ny, int dtype, void *stream) {
    KB_REQUIRE(f, "kb_apply_extrapolate_east_2d: null population pointer");
    if (int e = check_dims("kb_apply_extrapolate_east_2d", Nx, Ny)) return e;
    KB_REQUIRE(Nx >= 2, "kb_apply_extrapolate_east_2d: needs Nx >= 2");
    KB_DISPATCH_PLAIN("kb_apply_extrapolate_east_2d", dtype,
        (extrapolate_east_k<T><<<line_grid(Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f, grid2<T>(Nx, Ny))));
}

int kb_apply_bounce_back_wall_2d(void *f, int Nx, int Ny, int wall_id, int dtype, void *stream) {
    KB_REQUIRE(f, "kb_apply_bounce_back_wall_2d: null population pointer");
    if (int e = check_dims("kb_apply_bounce_back_wall_2d", Nx, Ny)) return e;
    KB_REQUIRE(wall_id >= 1 && wall_id <= 4,
               "kb_apply_bounce_back_wall_2d: unknown side %d (1 south, 2 west, 3 east, 4 north)",
               wall_id);
    const int n = (wall_id == 1 || wall_id == 4) ? Nx : Ny;
    KB_DISPATCH_PLAIN("kb_apply_bounce_back_wall_2d", dtype,
        (bounce_back_wall_k<T><<<line_grid(n), BX, 0, kb::as_stream(stream)>>>(
            (T *)f, grid2<T>(Nx, Ny), wall_id)));
}

int kb_init_equilibrium_2d(void *f, const void *rho, const void *ux, const void *uy,
                           int fields_dtype, int Nx, int Ny, int dtype, void *stream) {
    KB_REQUIRE(f && rho && ux && uy, "kb_init_equilibrium_2d: null pointer");
    KB_REQUIRE(fields_dtype == KB_F64 || fields_dtype == KB_F32,
               "kb_init_equilibrium_2d: fields must be KB_F64 or KB_F32 (got %d)", fields_dtype);
    if (int e = check_dims("kb_init_equilibrium_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_init_equilibrium_2d", dtype,
        if (fields_dtype == KB_F64)
            (equilibrium_k<T, double><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
                (T *)f, (const double *)rho, (const double *)ux, (const double *)uy, grid2<T>(Nx, Ny)));
        else
            (equilibrium_k<T, float><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
                (T *)f, (const float *)rho, (const float *)ux, (const float *)uy, grid2<T>(Nx, Ny))));
}

int kb_compute_macroscopic_2d(void *rho, void *ux, void *uy, const void *f, int Nx, int Ny,
                              int dtype, void *stream) {
    KB_REQUIRE(rho && ux && uy && f, "kb_compute_macroscopic_2d: null pointer");
    if (int e = check_dims("kb_compute_macroscopic_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_compute_macroscopic_2d", dtype,
        (macroscopic_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)rho, (T *)ux, (T *)uy, (const T *)f, grid2<T>(Nx, Ny))));
}

int kb_fused_bgk_step(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                      const uint8_t *is_solid, int Nx, int Ny, double omega, int dtype,
                      void *stream) {
    KB_REQUIRE(f_out && f_in && rho && ux && uy, "kb_fused_bgk_step: null pointer");
    KB_REQUIRE(f_out != f_in, "kb_fused_bgk_step: f_out and f_in must differ");
    if (int e = check_dims("kb_fused_bgk_step", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_fused_bgk_step", dtype,
        (fused_bgk_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f_out, (const T *)f_in, (T *)rho, (T *)ux, (T *)uy, is_solid, grid2<T>(Nx, Ny),
            (T)omega)));
}

int kb_trt_rates(double nu, double Lambda, double *s_plus, double *s_minus) {
    KB_REQUIRE(s_plus && s_minus, "kb_trt_rates: null output pointer");
    KB_REQUIRE(nu > 0.0, "kb_trt_rates: nu must be positive (got %g)", nu);
    KB_REQUIRE(Lambda > 0.0, "kb_trt_rates: Lambda must be positive (got %g)", Lambda);
    // trt_rates: src/kernels/fused_trt_2d.jl:129-133
    *s_plus = 1.0 / (3.0 * nu + 0.5);
    *s_minus = 1.0 / (Lambda / (3.0 * nu) + 0.5);
    return KB_OK;
}

int kb_fused_trt_step(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                      const uint8_t *is_solid, int Nx, int Ny, double nu, double Lambda, int dtype,
                      void *stream) {
    KB_REQUIRE(f_out && f_in && rho && ux && uy, "kb_fused_trt_step: null pointer");
    KB_REQUIRE(f_out != f_in, "kb_fused_trt_step: f_out and f_in must differ");
    if (int e = check_dims("kb_fused_trt_step", Nx, Ny)) return e;
    double sp, sm;
    if (int e = kb_trt_rates(nu, Lambda, &sp, &sm)) return e;
    KB_DISPATCH_PLAIN("kb_fused_trt_step", dtype,
        (fused_trt_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f_out, (const T *)f_in, (T *)rho, (T *)ux, (T *)uy, is_solid, grid2<T>(Nx, Ny),
            (T)sp, (T)sm)));
}

int kb_fused_trt_libb_step(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                           const uint8_t *is_solid, const void *q_wall, const void *uw_link_x,
                           const void *uw_link_y, int Nx, int Ny, double nu, double Lambda,
                           int dtype, void *stream) {
    const char *what = "kb_fused_trt_libb_step";
    KB_REQUIRE(f_out && f_in, "%s: null population pointer", what);
    KB_REQUIRE(q_wall && uw_link_x && uw_link_y, "%s: null q_wall / uw_link pointer", what);
    KB_REQUIRE(f_out != f_in, "%s: f_out and f_in must differ", what);
    const int nm = (rho != nullptr) + (ux != nullptr) + (uy != nullptr);
    KB_REQUIRE(nm == 0 || nm == 3, "%s: pass all three moment arrays or none", what);
    if (int e = check_dims(what, Nx, Ny)) return e;
    double sp, sm;
    if (int e = kb_trt_rates(nu, Lambda, &sp, &sm)) return e;
    KB_DISPATCH_PLAIN(what,
        dtype, (fused_trt_libb_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
                   (T *)f_out, (const T *)f_in, (T *)rho, (T *)ux, (T *)uy, is_solid,
                   (const T *)q_wall, (const T *)uw_link_x, (const T *)uw_link_y,
                   grid2<T>(Nx, Ny), (T)sp, (T)sm)));
}

static int aa_step(bool stream_step, void *f, void *rho, void *ux, void *uy,
                   const uint8_t *is_solid, int Nx, int Ny, double omega, int dtype,
                   void *stream) {
    const char *what = stream_step ? "kb_aa_stream_step_2d" : "kb_aa_local_step_2d";
    KB_REQUIRE(f, "%s: null population pointer", what);
    const int nm = (rho != nullptr) + (ux != nullptr) + (uy != nullptr);
    KB_REQUIRE(nm == 0 || nm == 3, "%s: pass all three moment arrays or none", what);
    if (int e = check_dims(what, Nx, Ny)) return e;
    KB_DISPATCH_PLAIN(what, dtype,
        (stream_step
             ? aa_stream_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
                   (T *)f, (T *)rho, (T *)ux, (T *)uy, is_solid, grid2<T>(Nx, Ny), (T)omega)
             : aa_local_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
                   (T *)f, (T *)rho, (T *)ux, (T *)uy, is_solid, grid2<T>(Nx, Ny), (T)omega)));
}

int kb_aa_stream_step_2d(void *f, void *rho, void *ux, void *uy, const uint8_t *is_solid, int Nx,
                         int Ny, double omega, int dtype, void *stream) {
    return aa_step(true, f, rho, ux, uy, is_solid, Nx, Ny, omega, dtype, stream);
}

int kb_aa_local_step_2d(void *f, void *rho, void *ux, void *uy, const uint8_t *is_solid, int Nx,
                        int Ny, double omega, int dtype, void *stream) {
    return aa_step(false, f, rho, ux, uy, is_solid, Nx, Ny, omega, dtype, stream);
}

int kb_collide_mrt_2d(void *f, const uint8_t *is_solid, int Nx, int Ny, double nu, double s_e,
                      double s_eps, double s_q, int dtype, void *stream) {
    KB_REQUIRE(f, "kb_collide_mrt_2d: null population pointer");
    KB_REQUIRE(nu > 0.0, "kb_collide_mrt_2d: nu must be positive (got %g)", nu);
    if (int e = check_dims("kb_collide_mrt_2d", Nx, Ny)) return e;
    // s_nu = T(1.0 / (3.0 * nu + 0.5)): src/kernels/collide_mrt_2d.jl:122
    const double s_nu = 1.0 / (3.0 * nu + 0.5);
    KB_DISPATCH_PLAIN("kb_collide_mrt_2d", dtype,
        (mrt_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f, is_solid, grid2<T>(Nx, Ny), (T)s_e, (T)s_eps, (T)s_q, (T)s_nu)));
}

int kb_stream_fully_periodic_2d(void *f_out, const void *f_in, int Nx, int Ny, int dtype,
                                void *stream) {
    KB_REQUIRE(f_out && f_in, "kb_stream_fully_periodic_2d: null population pointer");
    KB_REQUIRE(f_out != f_in, "kb_stream_fully_periodic_2d: f_out and f_in must differ");
    if (int e = check_dims("kb_stream_fully_periodic_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_stream_fully_periodic_2d", dtype,
        (stream_periodic_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f_out, (const T *)f_in, grid2<T>(Nx, Ny))));
}

int kb_stream_periodic_x_wall_y_2d(void *f_out, const void *f_in, int Nx, int Ny, int dtype,
                                   void *stream) {
    KB_REQUIRE(f_out && f_in, "kb_stream_periodic_x_wall_y_2d: null population pointer");
    KB_REQUIRE(f_out != f_in, "kb_stream_periodic_x_wall_y_2d: f_out and f_in must differ");
    if (int e = check_dims("kb_stream_periodic_x_wall_y_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_stream_periodic_x_wall_y_2d", dtype,
        (stream_px_wy_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f_out, (const T *)f_in, grid2<T>(Nx, Ny))));
}

int kb_cavity_step_2d(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                      const uint8_t *is_solid, int Nx, int Ny, double omega, double u_lid,
                      int dtype, void *stream) {
    KB_REQUIRE(f_out && f_in && rho && ux && uy, "kb_cavity_step_2d: null pointer");
    KB_REQUIRE(f_out != f_in, "kb_cavity_step_2d: f_out and f_in must differ");
    if (int e = check_dims("kb_cavity_step_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_cavity_step_2d", dtype,
        (cavity_step_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f_out, (const T *)f_in, (T *)rho, (T *)ux, (T *)uy, is_solid, grid2<T>(Nx, Ny),
            (T)omega, (T)u_lid)));
}

int kb_cavity_mrt_step_2d(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                          const uint8_t *is_solid, int Nx, int Ny, double nu, double s_e,
                          double s_eps, double s_q, double u_lid, int dtype, void *stream) {
    KB_REQUIRE(f_out && f_in, "kb_cavity_mrt_step_2d: null population pointer");
    KB_REQUIRE(f_out != f_in, "kb_cavity_mrt_step_2d: f_out and f_in must differ");
    const int nm = (rho != nullptr) + (ux != nullptr) + (uy != nullptr);
    KB_REQUIRE(nm == 0 || nm == 3, "kb_cavity_mrt_step_2d: pass all three moment arrays or none");
    KB_REQUIRE(nu > 0.0, "kb_cavity_mrt_step_2d: nu must be positive (got %g)", nu);
    if (int e = check_dims("kb_cavity_mrt_step_2d", Nx, Ny)) return e;
    const double s_nu = 1.0 / (3.0 * nu + 0.5);
    KB_DISPATCH_PLAIN("kb_cavity_mrt_step_2d", dtype,
        (cavity_mrt_step_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f_out, (const T *)f_in, (T *)rho, (T *)ux, (T *)uy, is_solid, grid2<T>(Nx, Ny),
            (T)s_e, (T)s_eps, (T)s_q, (T)s_nu, (T)u_lid)));
}

int kb_cavity_mrt_init_step_2d(void *f_out, const void *f_in, const void *ux, const void *uy,
                               int fields_dtype, const uint8_t *is_solid, int Nx, int Ny, double nu,
                               double s_e, double s_eps, double s_q, double u_lid, int dtype,
                               void *stream) {
    KB_REQUIRE(f_out && f_in && ux && uy, "kb_cavity_mrt_init_step_2d: null pointer");
    KB_REQUIRE(f_out != f_in, "kb_cavity_mrt_init_step_2d: f_out and f_in must differ");
    KB_REQUIRE(fields_dtype == KB_F64 || fields_dtype == KB_F32,
               "kb_cavity_mrt_init_step_2d: fields must be KB_F64 or KB_F32 (got %d)", fields_dtype);
    if (int e = check_dims("kb_cavity_mrt_init_step_2d", Nx, Ny)) return e;
    const double s_nu = 1.0 / (3.0 * nu + 0.5);
    KB_DISPATCH_PLAIN("kb_cavity_mrt_init_step_2d", dtype,
        if (fields_dtype == KB_F64)
            (cavity_mrt_fixed_u_k<T, double><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
                (T *)f_out, (const T *)f_in, (const double *)ux, (const double *)uy, is_solid,
                grid2<T>(Nx, Ny), (T)s_e, (T)s_eps, (T)s_q, (T)s_nu, (T)u_lid));
        else
            (cavity_mrt_fixed_u_k<T, float><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
                (T *)f_out, (const T *)f_in, (const float *)ux, (const float *)uy, is_solid,
                grid2<T>(Nx, Ny), (T)s_e, (T)s_eps, (T)s_q, (T)s_nu, (T)u_lid)));
}

int kb_cavity_movingwall_step_2d(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                                 const uint8_t *is_solid, int Nx, int Ny, double omega,
                                 double u_lid, int dtype, void *stream) {
    KB_REQUIRE(f_out && f_in, "kb_cavity_movingwall_step_2d: null population pointer");
    KB_REQUIRE(f_out != f_in, "kb_cavity_movingwall_step_2d: f_out and f_in must differ");
    const int nm = (rho != nullptr) + (ux != nullptr) + (uy != nullptr);
    KB_REQUIRE(nm == 0 || nm == 3, "kb_cavity_movingwall_step_2d: pass all three moment arrays or none");
    if (int e = check_dims("kb_cavity_movingwall_step_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_cavity_movingwall_step_2d", dtype,
        (cavity_movingwall_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f_out, (const T *)f_in, (T *)rho, (T *)ux, (T *)uy, is_solid, grid2<T>(Nx, Ny),
            (T)omega, (T)u_lid)));
}

int kb_fused_natconv_step(void *f_out, const void *f_in, void *g_out, const void *g_in,
                          void *Temp, int Nx, int Ny, double omega_f, double omega_T,
                          double beta_g, double T_ref_buoy, double T_hot, double T_cold,
                          int dtype, void *stream) {
    KB_REQUIRE(f_out && f_in && g_out && g_in && Temp, "kb_fused_natconv_step: null pointer");
    KB_REQUIRE(f_out != f_in && g_out != g_in, "kb_fused_natconv_step: in and out must differ");
    if (int e = check_dims("kb_fused_natconv_step", Nx, Ny)) return e;
    if (dtype != KB_F64 && dtype != KB_F32)
        return kb::d3::launch_natconv_dev(dtype, false, f_out, f_in, g_out, g_in, (float *)Temp, Nx,
                                          Ny, omega_f, omega_T, beta_g, T_ref_buoy, T_hot, T_cold,
                                          0.0, 0.0, 0.0, kb::as_stream(stream));
    KB_DISPATCH_PLAIN("kb_fused_natconv_step", dtype,
        (natconv_k<T, false><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f_out, (const T *)f_in, (T *)g_out, (const T *)g_in, (T *)Temp, grid2<T>(Nx, Ny),
            (T)omega_f, (T)omega_T, (T)beta_g, (T)T_ref_buoy, (T)T_hot, (T)T_cold, T(0), T(0),
            T(0))));
}

int kb_fused_natconv_vt_step(void *f_out, const void *f_in, void *g_out, const void *g_in,
                             void *Temp, int Nx, int Ny, double nu_ref, double T0_visc,
                             double alpha_visc, double omega_T, double beta_g, double T_ref_buoy,
                             double T_hot, double T_cold, int dtype, void *stream) {
    KB_REQUIRE(f_out && f_in && g_out && g_in && Temp, "kb_fused_natconv_vt_step: null pointer");
    KB_REQUIRE(f_out != f_in && g_out != g_in, "kb_fused_natconv_vt_step: in and out must differ");
    if (int e = check_dims("kb_fused_natconv_vt_step", Nx, Ny)) return e;
    if (dtype != KB_F64 && dtype != KB_F32)
        return kb::d3::launch_natconv_dev(dtype, true, f_out, f_in, g_out, g_in, (float *)Temp, Nx,
                                          Ny, 0.0, omega_T, beta_g, T_ref_buoy, T_hot, T_cold,
                                          nu_ref, T0_visc, alpha_visc, kb::as_stream(stream));
    KB_DISPATCH_PLAIN("kb_fused_natconv_vt_step", dtype,
        (natconv_k<T, true><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f_out, (const T *)f_in, (T *)g_out, (const T *)g_in, (T *)Temp, grid2<T>(Nx, Ny),
            T(0), (T)omega_T, (T)beta_g, (T)T_ref_buoy, (T)T_hot, (T)T_cold, (T)nu_ref,
            (T)T0_visc, (T)alpha_visc)));
}

int kb_compute_temperature_2d(void *Temp, const void *g, int Nx, int Ny, int dtype, void *stream) {
    KB_REQUIRE(Temp && g, "kb_compute_temperature_2d: null pointer");
    if (int e = check_dims("kb_compute_temperature_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_compute_temperature_2d", dtype,
        (temperature_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)Temp, (const T *)g, grid2<T>(Nx, Ny))));
}

int kb_collide_thermal_2d(void *g, const void *ux, const void *uy, int Nx, int Ny, double omega_T,
                          int dtype, void *stream) {
    KB_REQUIRE(g && ux && uy, "kb_collide_thermal_2d: null pointer");
    if (int e = check_dims("kb_collide_thermal_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_collide_thermal_2d", dtype,
        (collide_thermal_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)g, (const T *)ux, (const T *)uy, grid2<T>(Nx, Ny), (T)omega_T)));
}

int kb_collide_thermal_masked_2d(void *g, const void *ux, const void *uy, const uint8_t *is_skip,
                                 int Nx, int Ny, double omega_T, int dtype, void *stream) {
    KB_REQUIRE(g && ux && uy, "kb_collide_thermal_masked_2d: null pointer");
    if (int e = check_dims("kb_collide_thermal_masked_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_collide_thermal_masked_2d", dtype,
        (collide_thermal_masked_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)g, (const T *)ux, (const T *)uy, is_skip, grid2<T>(Nx, Ny), (T)omega_T)));
}

}  // extern "C"

namespace {

template <typename T>
T corner_temp(double Ta, bool has_b, double Tb) {
    // _corner_temp (thermal_2d.jl:356-357): the mean of the two wall
    // temperatures, in the population type
    return has_b ? (T(Ta) + T(Tb)) / T(2) : T(Ta);
}

template <typename T>
int launch_fixed_temp_2d(T *g, int Nx, int Ny, const FixedTempSet2<T> &S, cudaStream_t s,
                         const char *what) {
    if (S.n == 0) return KB_OK;
    const int len = Nx > Ny ? Nx : Ny;
    fixed_temp_k<T><<<dim3(line_grid(len), S.n), BX, 0, s>>>(g, grid2<T>(Nx, Ny), S);
    return kb::check_launch(what);
}

// _apply_fixed_temp_faces_2d! (thermal_2d.jl:371-392) for every face in
// `faces`: the x-faces own the corner slots they share with a Dirichlet
// y-face (mean temperature), the y-faces skip them.  No slot is written by
// two faces, so all faces run in one launch.
template <typename T>
int fixed_temp_all_2d(T *g, int Nx, int Ny, unsigned faces, const double *Tf, cudaStream_t s) {
    const bool hw = faces & 1u, he = faces & 2u, hs = faces & 4u, hn = faces & 8u;
    FixedTempSet2<T> S{};
    S.n = 0;
    for (int face = 0; face < 4; ++face) {
        if (!(faces & (1u << face))) continue;
        FixedTempFace2<T> F{};
        F.face = face;
        F.T_wall = T(Tf[face]);
        if (face < 2) {
            F.T_c[0] = corner_temp<T>(Tf[face], hs, Tf[2]);
            F.T_c[1] = corner_temp<T>(Tf[face], hn, Tf[3]);
            F.skip[0] = F.skip[1] = 0;
        } else {
            F.T_c[0] = F.T_c[1] = T(Tf[face]);
            F.skip[0] = hw;
            F.skip[1] = he;
        }
        S.f[S.n++] = F;
    }
    return launch_fixed_temp_2d(g, Nx, Ny, S, s, "kb_apply_fixed_temp_2d");
}

}  // namespace

extern "C" {

int kb_apply_fixed_temp_face_2d(void *g, int Nx, int Ny, int face, double T_wall,
                                double T_corner_lo, double T_corner_hi, int skip_lo, int skip_hi,
                                int dtype, void *stream) {
    KB_REQUIRE(g, "kb_apply_fixed_temp_face_2d: null population pointer");
    KB_REQUIRE(face >= 0 && face < 4, "kb_apply_fixed_temp_face_2d: face %d not in 0..3", face);
    if (int e = check_dims("kb_apply_fixed_temp_face_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_apply_fixed_temp_face_2d", dtype, {
        FixedTempSet2<T> S{};
        S.n = 1;
        S.f[0].face = face;
        S.f[0].T_wall = (T)T_wall;
        S.f[0].T_c[0] = (T)T_corner_lo;
        S.f[0].T_c[1] = (T)T_corner_hi;
        S.f[0].skip[0] = skip_lo != 0;
        S.f[0].skip[1] = skip_hi != 0;
        if (int r = launch_fixed_temp_2d((T *)g, Nx, Ny, S, kb::as_stream(stream),
                                         "kb_apply_fixed_temp_face_2d"))
            return r;
    });
}

int kb_apply_fixed_temp_2d(void *g, int Nx, int Ny, unsigned faces, const double *T_faces,
                           int dtype, void *stream) {
    KB_REQUIRE(g, "kb_apply_fixed_temp_2d: null population pointer");
    KB_REQUIRE(faces < 16u, "kb_apply_fixed_temp_2d: face mask 0x%x has bits beyond 0..3", faces);
    KB_REQUIRE(faces == 0u || T_faces, "kb_apply_fixed_temp_2d: null temperature array");
    if (int e = check_dims("kb_apply_fixed_temp_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_apply_fixed_temp_2d", dtype, {
        if (int r = fixed_temp_all_2d((T *)g, Nx, Ny, faces, T_faces, kb::as_stream(stream)))
            return r;
    });
}

int kb_collide_boussinesq_2d(void *f, const void *Temp, const uint8_t *is_solid, int Nx, int Ny,
                             double omega, double beta_g, double T_ref, int dtype, void *stream) {
    KB_REQUIRE(f && Temp, "kb_collide_boussinesq_2d: null pointer");
    if (int e = check_dims("kb_collide_boussinesq_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_collide_boussinesq_2d", dtype,
        (launch_forced_2d<T, 0>((T *)f, (const T *)Temp, is_solid, nullptr, nullptr, Nx, Ny, (T)omega,
                                (T)beta_g, (T)T_ref, T(0), T(0), kb::as_stream(stream))));
}

int kb_collide_boussinesq_vt_2d(void *f, const void *Temp, const uint8_t *is_solid, int Nx, int Ny,
                                double nu_ref, double T_ref, double A_arr, double beta_g,
                                int dtype, void *stream) {
    KB_REQUIRE(f && Temp, "kb_collide_boussinesq_vt_2d: null pointer");
    if (int e = check_dims("kb_collide_boussinesq_vt_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_collide_boussinesq_vt_2d", dtype,
        (boussinesq_k<T, 1><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f, (const T *)Temp, is_solid, grid2<T>(Nx, Ny), T(0), (T)nu_ref, (T)T_ref,
            (T)A_arr, (T)beta_g, (T)T_ref)));
}

int kb_collide_boussinesq_vt_modified_2d(void *f, const void *Temp, const uint8_t *is_solid,
                                         int Nx, int Ny, double nu_ref, double T0_visc,
                                         double alpha_visc, double beta_g, double T_ref_buoy,
                                         int dtype, void *stream) {
    KB_REQUIRE(f && Temp, "kb_collide_boussinesq_vt_modified_2d: null pointer");
    if (int e = check_dims("kb_collide_boussinesq_vt_modified_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_collide_boussinesq_vt_modified_2d", dtype,
        (boussinesq_k<T, 2><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)f, (const T *)Temp, is_solid, grid2<T>(Nx, Ny), T(0), (T)nu_ref, (T)T0_visc,
            (T)alpha_visc, (T)beta_g, (T)T_ref_buoy)));
}

}  // extern "C"

extern "C" {

int kb_collide_guo_2d(void *f, const uint8_t *is_solid, int Nx, int Ny, double omega, double Fx,
                      double Fy, int dtype, void *stream) {
    KB_REQUIRE(f, "kb_collide_guo_2d: null population pointer");
    if (int e = check_dims("kb_collide_guo_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_collide_guo_2d", dtype,
        (launch_forced_2d<T, 1>((T *)f, nullptr, is_solid, nullptr, nullptr, Nx, Ny, (T)omega, T(0), T(0),
                                (T)Fx, (T)Fy, kb::as_stream(stream))));
}

int kb_collide_guo_field_2d(void *f, const uint8_t *is_solid, const void *Fx_field,
                            const void *Fy_field, int Nx, int Ny, double omega, int dtype,
                            void *stream) {
    KB_REQUIRE(f && Fx_field && Fy_field, "kb_collide_guo_field_2d: null pointer");
    if (int e = check_dims("kb_collide_guo_field_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_collide_guo_field_2d", dtype,
        (launch_forced_2d<T, 2>((T *)f, nullptr, is_solid, (const T *)Fx_field, (const T *)Fy_field, Nx,
                                Ny, (T)omega, T(0), T(0), T(0), T(0), kb::as_stream(stream))));
}

}  // extern "C"

extern "C" {

int kb_compute_macroscopic_forced_2d(void *rho, void *ux, void *uy, const void *f, int Nx, int Ny,
                                     double Fx, double Fy, int dtype, void *stream) {
    KB_REQUIRE(rho && ux && uy && f, "kb_compute_macroscopic_forced_2d: null pointer");
    if (int e = check_dims("kb_compute_macroscopic_forced_2d", Nx, Ny)) return e;
    KB_DISPATCH_PLAIN("kb_compute_macroscopic_forced_2d", dtype,
        (macroscopic_forced_k<T><<<nodes_grid(Nx, Ny), BX, 0, kb::as_stream(stream)>>>(
            (T *)rho, (T *)ux, (T *)uy, (const T *)f, grid2<T>(Nx, Ny), (T)Fx, (T)Fy)));
}

}  // extern "C"
