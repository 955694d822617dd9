// kb_d3q19.cuh -- D3Q19 geometry helpers shared by the exact and the
// deviation-storage translation units.
#pragma once

#include "kb_common.cuh"

namespace kb {
namespace d3 {

#ifndef KB_D3_BLOCK_X
#define KB_D3_BLOCK_X 128
#endif
constexpr int BX = KB_D3_BLOCK_X;  // threads per block along x

struct Grid3 {
    int Nx, Ny, Nz;
    size_t plane;  // population stride in nodes: Nx*Ny*Nz, or more for a z-range
    int per;       // bit 0 x, bit 1 y, bit 2 z periodic; bit 3 z halo (below)
    int zoff = 0;  // z-range: plane of the allocation that k = 0 is (staged copies)
};
// z halo (per bit 3): the grid is a range of z-planes inside a larger
// allocation whose planes k = -1 and k = Nz exist; z-pulls read them as they
// are (no wrap, no bounce-back).  The pointers passed start at plane zoff.
constexpr int KB_ZHALO = 8;

// Signed node offsets of the pull sources of one node, with the flags that
// say whether the source exists (inside the box, or wrapped on a periodic
// axis).  A missing source means half-way bounce-back: the node takes its
// own opposite population.  Follows PullHalfwayBB_3D
// (src/kernels/dsl/bricks_3d.jl:70-136) and stream_3d_kernel!
// (src/kernels/collide_stream_3d.jl:5-42).
// I is the element-offset type: int when every offset of the population
// buffer fits in 31 bits (all addresses are then a per-thread base pointer
// plus a 32-bit offset), long long otherwise.
template <typename I>
struct Pull3 {
    I dxm, dxp, dym, dyp, dzm, dzp;  // offset of the source for c=+1 (m) / c=-1 (p)
    bool xm, xp, ym, yp, zm, zp;
};

template <typename I = long long>
__device__ __forceinline__ Pull3<I> pull_geometry(const Grid3 &g, int i, int j, int k) {
    Pull3<I> s;
    const bool px = g.per & 1, py = (g.per >> 1) & 1, pz = (g.per >> 2) & 1;
    const bool zh = (g.per & KB_ZHALO) != 0;
    const I sx = 1, sy = (I)g.Nx, sz = (I)g.Nx * (I)g.Ny;
    s.xm = px || i > 0;
    s.xp = px || i < g.Nx - 1;
    s.ym = py || j > 0;
    s.yp = py || j < g.Ny - 1;
    s.zm = pz || zh || k > 0;
    s.zp = pz || zh || k < g.Nz - 1;
    s.dxm = (i > 0 ? (I)-1 : (I)(g.Nx - 1)) * sx;
    s.dxp = (i < g.Nx - 1 ? (I)1 : -(I)(g.Nx - 1)) * sx;
    s.dym = (j > 0 ? (I)-1 : (I)(g.Ny - 1)) * sy;
    s.dyp = (j < g.Ny - 1 ? (I)1 : -(I)(g.Ny - 1)) * sy;
    s.dzm = (k > 0 || zh ? (I)-1 : (I)(g.Nz - 1)) * sz;
    s.dzp = (k < g.Nz - 1 || zh ? (I)1 : -(I)(g.Nz - 1)) * sz;
    return s;
}

// Pull all 19 populations of the node at f0 (= f + node index) into p[]
// (any element type; Load(x) maps a stored value to the working value).
// P is the plane size in elements.
template <typename R, typename V, typename Load, typename I>
__device__ __forceinline__ void pull19_at(const R *__restrict__ f0, I P, const Pull3<I> &s, V *p,
                                          Load ld) {
    p[0] = ld(f0[0]);
    p[1] = ld(f0[s.xm ? s.dxm + 1 * P : 2 * P]);
    p[2] = ld(f0[s.xp ? s.dxp + 2 * P : 1 * P]);
    p[3] = ld(f0[s.ym ? s.dym + 3 * P : 4 * P]);
    p[4] = ld(f0[s.yp ? s.dyp + 4 * P : 3 * P]);
    p[5] = ld(f0[s.zm ? s.dzm + 5 * P : 6 * P]);
    p[6] = ld(f0[s.zp ? s.dzp + 6 * P : 5 * P]);
    p[7] = ld(f0[(s.xm && s.ym) ? s.dxm + s.dym + 7 * P : 10 * P]);
    p[8] = ld(f0[(s.xp && s.ym) ? s.dxp + s.dym + 8 * P : 9 * P]);
    p[9] = ld(f0[(s.xm && s.yp) ? s.dxm + s.dyp + 9 * P : 8 * P]);
    p[10] = ld(f0[(s.xp && s.yp) ? s.dxp + s.dyp + 10 * P : 7 * P]);
    p[11] = ld(f0[(s.xm && s.zm) ? s.dxm + s.dzm + 11 * P : 14 * P]);
    p[12] = ld(f0[(s.xp && s.zm) ? s.dxp + s.dzm + 12 * P : 13 * P]);
    p[13] = ld(f0[(s.xm && s.zp) ? s.dxm + s.dzp + 13 * P : 12 * P]);
    p[14] = ld(f0[(s.xp && s.zp) ? s.dxp + s.dzp + 14 * P : 11 * P]);
    p[15] = ld(f0[(s.ym && s.zm) ? s.dym + s.dzm + 15 * P : 18 * P]);
    p[16] = ld(f0[(s.yp && s.zm) ? s.dyp + s.dzm + 16 * P : 17 * P]);
    p[17] = ld(f0[(s.ym && s.zp) ? s.dym + s.dzp + 17 * P : 16 * P]);
    p[18] = ld(f0[(s.yp && s.zp) ? s.dyp + s.dzp + 18 * P : 15 * P]);
}

// Pull with 64-bit offsets from the buffer base f and node index c.
template <typename R, typename V, typename Load>
__device__ __forceinline__ void pull19(const R *__restrict__ f, size_t P, size_t c,
                                       const Pull3<long long> &s, V *p, Load ld) {
    pull19_at(f + c, (long long)P, s, p, ld);
}

// True when every element offset of a Q-population buffer on grid g fits
// in a signed 32-bit int.
inline bool offsets_fit_int(const Grid3 &g, int Q) {
    return (double)g.plane * (double)(Q + 1) < 2147483647.0;
}

inline dim3 nodes_grid(int Nx, int Ny, int Nz) { return dim3((Nx + BX - 1) / BX, Ny, Nz); }

inline int check_dims(const char *what, int Nx, int Ny, int Nz) {
    if (Nx < 1 || Ny < 1 || Nz < 1 || Ny > 65535 || Nz > 65535)
        return set_error(KB_ERR_ARG,
                         "%s: bad grid %d x %d x %d (need Nx >= 1, 1 <= Ny, Nz <= 65535)", what,
                         Nx, Ny, Nz);
    return KB_OK;
}

// _libb_branch (src/kernels/li_bb_2d.jl:70-83), shared by D3Q19.
template <typename T>
__device__ __forceinline__ T libb_branch(T q_w, T f_here, T f_back, T f_bar_here, T d) {
    if (q_w <= T(0.5)) return T(2) * q_w * f_here + (T(1) - T(2) * q_w) * f_back + d;
    const T inv = T(1) / (T(2) * q_w);
    return inv * f_here + (T(1) - inv) * f_bar_here + d * inv;
}

// ApplyLiBBPrePhase_3D (src/kernels/dsl/bricks_3d.jl:367-475): each cut
// link q (q_wall[q] > 0) replaces the pulled population of the opposite
// direction with the Bouzidi estimate; the wall-velocity term of each link
// is written as the reference writes it.  f0 points at the node (planes of
// stride P); the link data come through `lk` (LinkDense: the reference's
// dense per-link arrays; LinkRecord: one record of the compact table).
struct LoadSame {
    template <typename V> __device__ __forceinline__ V operator()(V v) const { return v; }
};

template <typename T, typename I, typename Links, typename F = T, typename Load = LoadSame>
__device__ __forceinline__ void libb_prephase_3d(const F *__restrict__ f0, I P, const Links &lk,
                                                 T *p, Load ld = Load()) {
    const T c3 = T(1.0 / 3.0), c6 = T(1.0 / 6.0);
    T q;
#define KB_LIBB(QA, QB, DELTA) \
    if ((q = lk.q(QA)) > T(0)) \
        p[QB] = libb_branch(q, (T)ld(f0[(QA) * P]), p[QA], (T)ld(f0[(QB) * P]), DELTA)
    KB_LIBB(1, 2, -c3 * lk.x(1));
    KB_LIBB(2, 1, c3 * lk.x(2));
    KB_LIBB(3, 4, -c3 * lk.y(3));
    KB_LIBB(4, 3, c3 * lk.y(4));
    KB_LIBB(5, 6, -c3 * lk.z(5));
    KB_LIBB(6, 5, c3 * lk.z(6));
    KB_LIBB(7, 10, -c6 * (lk.x(7) + lk.y(7)));
    KB_LIBB(10, 7, c6 * (lk.x(10) + lk.y(10)));
    KB_LIBB(8, 9, -c6 * (-lk.x(8) + lk.y(8)));
    KB_LIBB(9, 8, -c6 * (lk.x(9) - lk.y(9)));
    KB_LIBB(11, 14, -c6 * (lk.x(11) + lk.z(11)));
    KB_LIBB(14, 11, c6 * (lk.x(14) + lk.z(14)));
    KB_LIBB(12, 13, -c6 * (-lk.x(12) + lk.z(12)));
    KB_LIBB(13, 12, -c6 * (lk.x(13) - lk.z(13)));
    KB_LIBB(15, 18, -c6 * (lk.y(15) + lk.z(15)));
    KB_LIBB(18, 15, c6 * (lk.y(18) + lk.z(18)));
    KB_LIBB(16, 17, -c6 * (-lk.y(16) + lk.z(16)));
    KB_LIBB(17, 16, -c6 * (lk.y(17) - lk.z(17)));
#undef KB_LIBB
}

// The reference's dense per-link arrays (19 planes laid out like f).
template <typename T, typename I>
struct LinkDense {
    const T *qw, *wx, *wy, *wz;  // at the node
    I P;
    __device__ __forceinline__ T q(int a) const { return qw[a * P]; }
    __device__ __forceinline__ T x(int a) const { return wx[a * P]; }
    __device__ __forceinline__ T y(int a) const { return wy[a * P]; }
    __device__ __forceinline__ T z(int a) const { return wz[a * P]; }
};

// Compact cut-link table (kb_libb_links): the cut links of a grid gathered
// from the dense per-link arrays.  cls holds one byte per node (0 fluid,
// 1 solid, 2 fluid with cut links), so a step reads one byte per node, as it
// would read the solid mask, and touches link data only at wall nodes.
struct LinkTable3 {
    const uint8_t *cls;
    const int *rec;                  // record of each cls == 2 node
    const void *qw, *wx, *wy, *wz;   // link q = 1..18 of record r at [(q - 1) * n_rec + r]
    long long n_rec;
    const int *node;                 // node of each record
};

// One side stream and a fork / join event pair per device, created on first
// use and kept for the life of the process: the cut-node kernel of a
// cut-link step runs there, beside the kernel that updates the other nodes.
// Null when the current device has none (the caller then uses its stream).
struct SideStream {
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    bool ok = false;
};
SideStream *side_stream();

// One record of the table, read like LinkDense.
template <typename T>
struct LinkRecord {
    const T *qw, *wx, *wy, *wz;  // at the record
    long long n;                 // n_rec
    __device__ __forceinline__ T q(int a) const { return qw[(a - 1) * n]; }
    __device__ __forceinline__ T x(int a) const { return wx[(a - 1) * n]; }
    __device__ __forceinline__ T y(int a) const { return wy[(a - 1) * n]; }
    __device__ __forceinline__ T z(int a) const { return wz[(a - 1) * n]; }
};

template <typename T>
__device__ __forceinline__ LinkRecord<T> link_record(const LinkTable3 &L, int r) {
    return LinkRecord<T>{(const T *)L.qw + r, (const T *)L.wx + r, (const T *)L.wy + r,
                         (const T *)L.wz + r, L.n_rec};
}

// The link data of one record held in registers (read with constant link
// indices once libb_prephase_3d is inlined).
template <typename T>
struct LinkRegs {
    T qv[19], xv[19], yv[19], zv[19];
    __device__ __forceinline__ T q(int a) const { return qv[a]; }
    __device__ __forceinline__ T x(int a) const { return xv[a]; }
    __device__ __forceinline__ T y(int a) const { return yv[a]; }
    __device__ __forceinline__ T z(int a) const { return zv[a]; }
};

// libb_prephase_3d on record r of the compact table with every load issued
// up front: the node's own populations and the 18 link fractions, then the
// wall velocities of the cut links.  Read link by link, each cut link is a
// branch on a load that must return first, so a node waits for up to 18
// dependent rounds of memory latency; here it waits for two.  The
// interpolation then runs on registers with the same expressions, so the
// result equals the link-by-link form.  It pays in a kernel of cut nodes
// only (trt_dev_cut_k); inside a kernel over every node its ~90 extra live
// values cut the residency of all nodes (the one-node FP64 table step went
// from 0.80 to 1.29 ms at 256^3 with it), so those keep the direct form.
template <typename T, typename I, typename F, typename Load = LoadSame>
__device__ __forceinline__ void libb_prephase_3d_record(const F *__restrict__ f0, I P,
                                                        const LinkTable3 &L, int r, T *p,
                                                        Load ld = Load()) {
    const LinkRecord<T> rec = link_record<T>(L, r);
    T own[19];
    LinkRegs<T> lk;
    own[0] = lk.qv[0] = lk.xv[0] = lk.yv[0] = lk.zv[0] = T(0);
#pragma unroll
    for (int a = 1; a < 19; ++a) {
        own[a] = (T)ld(f0[(I)a * P]);
        lk.qv[a] = rec.q(a);
    }
#pragma unroll
    for (int a = 1; a < 19; ++a) {
        const bool cut = lk.qv[a] > T(0);
        lk.xv[a] = cut ? rec.x(a) : T(0);
        lk.yv[a] = cut ? rec.y(a) : T(0);
        lk.zv[a] = cut ? rec.z(a) : T(0);
    }
    libb_prephase_3d(own, (I)1, lk, p, LoadSame());
}

// Deviation-storage step with the compact cut-link table (kb_d3q19_dev.cu);
// `variant` follows kernel 1 of kb_set_kernel_variant (0 automatic, 5 the
// staged row tiles for 16-bit storages, anything else one node per thread).
int launch_trt3d_dev_links(int dtype, void *f_out, const void *f_in, float *rho, float *ux,
                           float *uy, float *uz, const LinkTable3 &L, const Grid3 &g, float sp,
                           float sm, cudaStream_t s, int variant);

// Launchers of the fused TRT step for the deviation storages
// (kb_d3q19_dev.cu); `per` = periodic bit mask.
// Fused thermal DDF natural-convection step on deviation storage (f - w_q,
// g - w_q T_ref; KB_F32_DEV / KB_F16_DEV / KB_BF16_DEV and the stochastic-
// rounding 16-bit storages); Temp is float.  vt: temperature-dependent
// viscosity.
int launch_natconv_dev(int dtype, bool vt, void *f_out, const void *f_in, void *g_out,
                       const void *g_in, float *Temp, int Nx, int Ny, double w_f, double w_T,
                       double beta_g, double T_ref, double T_hot, double T_cold, double nu_ref,
                       double T0_visc, double a_visc, cudaStream_t s);
int launch_trt3d_dev(int dtype, void *f_out, const void *f_in, float *rho, float *ux, float *uy,
                     float *uz, const uint8_t *solid, const Grid3 &g, float sp, float sm,
                     cudaStream_t s, int variant);

}  // namespace d3
}  // namespace kb
