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
    size_t plane;  // Nx*Ny*Nz nodes in one population plane
    int per;       // bit 0 x, bit 1 y, bit 2 z periodic
};

// Signed node offsets of the pull sources of one node, with the flags that
// say whether the source exists (inside the box, or wrapped on a periodic
// axis).  A missing source means half-way bounce-back: the node takes its
// own opposite population.  Follows PullHalfwayBB_3D
// (src/kernels/dsl/bricks_3d.jl:70-136) and stream_3d_kernel!
// (src/kernels/collide_stream_3d.jl:5-42).
struct Pull3 {
    long long dxm, dxp, dym, dyp, dzm, dzp;  // offset of source for c=+1 (m) / c=-1 (p)
    bool xm, xp, ym, yp, zm, zp;
};

__device__ __forceinline__ Pull3 pull_geometry(const Grid3 &g, int i, int j, int k) {
    Pull3 s;
    const bool px = g.per & 1, py = (g.per >> 1) & 1, pz = (g.per >> 2) & 1;
    const long long sx = 1, sy = g.Nx, sz = (long long)g.Nx * g.Ny;
    s.xm = px || i > 0;
    s.xp = px || i < g.Nx - 1;
    s.ym = py || j > 0;
    s.yp = py || j < g.Ny - 1;
    s.zm = pz || k > 0;
    s.zp = pz || k < g.Nz - 1;
    s.dxm = (i > 0 ? -1 : (long long)(g.Nx - 1)) * sx;
    s.dxp = (i < g.Nx - 1 ? 1 : -(long long)(g.Nx - 1)) * sx;
    s.dym = (j > 0 ? -1 : (long long)(g.Ny - 1)) * sy;
    s.dyp = (j < g.Ny - 1 ? 1 : -(long long)(g.Ny - 1)) * sy;
    s.dzm = (k > 0 ? -1 : (long long)(g.Nz - 1)) * sz;
    s.dzp = (k < g.Nz - 1 ? 1 : -(long long)(g.Nz - 1)) * sz;
    return s;
}

// Pull all 19 populations of node c into p[] (any element type; the
// conversion Load(x) maps a stored value to the working value).
template <typename R, typename V, typename Load>
__device__ __forceinline__ void pull19(const R *__restrict__ f, size_t P, size_t c, const Pull3 &s,
                                       V *p, Load ld) {
    const R *f0 = f + c;
    p[0] = ld(f0[0]);
    p[1] = s.xm ? ld(f0[s.dxm + 1 * P]) : ld(f0[2 * P]);
    p[2] = s.xp ? ld(f0[s.dxp + 2 * P]) : ld(f0[1 * P]);
    p[3] = s.ym ? ld(f0[s.dym + 3 * P]) : ld(f0[4 * P]);
    p[4] = s.yp ? ld(f0[s.dyp + 4 * P]) : ld(f0[3 * P]);
    p[5] = s.zm ? ld(f0[s.dzm + 5 * P]) : ld(f0[6 * P]);
    p[6] = s.zp ? ld(f0[s.dzp + 6 * P]) : ld(f0[5 * P]);
    p[7] = (s.xm && s.ym) ? ld(f0[s.dxm + s.dym + 7 * P]) : ld(f0[10 * P]);
    p[8] = (s.xp && s.ym) ? ld(f0[s.dxp + s.dym + 8 * P]) : ld(f0[9 * P]);
    p[9] = (s.xm && s.yp) ? ld(f0[s.dxm + s.dyp + 9 * P]) : ld(f0[8 * P]);
    p[10] = (s.xp && s.yp) ? ld(f0[s.dxp + s.dyp + 10 * P]) : ld(f0[7 * P]);
    p[11] = (s.xm && s.zm) ? ld(f0[s.dxm + s.dzm + 11 * P]) : ld(f0[14 * P]);
    p[12] = (s.xp && s.zm) ? ld(f0[s.dxp + s.dzm + 12 * P]) : ld(f0[13 * P]);
    p[13] = (s.xm && s.zp) ? ld(f0[s.dxm + s.dzp + 13 * P]) : ld(f0[12 * P]);
    p[14] = (s.xp && s.zp) ? ld(f0[s.dxp + s.dzp + 14 * P]) : ld(f0[11 * P]);
    p[15] = (s.ym && s.zm) ? ld(f0[s.dym + s.dzm + 15 * P]) : ld(f0[18 * P]);
    p[16] = (s.yp && s.zm) ? ld(f0[s.dyp + s.dzm + 16 * P]) : ld(f0[17 * P]);
    p[17] = (s.ym && s.zp) ? ld(f0[s.dym + s.dzp + 17 * P]) : ld(f0[16 * P]);
    p[18] = (s.yp && s.zp) ? ld(f0[s.dyp + s.dzp + 18 * P]) : ld(f0[15 * P]);
}

inline dim3 nodes_grid(int Nx, int Ny, int Nz) { return dim3((Nx + BX - 1) / BX, Ny, Nz); }

inline int check_dims(const char *what, int Nx, int Ny, int Nz) {
    if (Nx < 1 || Ny < 1 || Nz < 1 || Ny > 65535 || Nz > 65535)
        return set_error(KB_ERR_ARG,
                         "%s: bad grid %d x %d x %d (need Nx >= 1, 1 <= Ny, Nz <= 65535)", what,
                         Nx, Ny, Nz);
    return KB_OK;
}

// Launchers of the fused TRT step for the deviation storages
// (kb_d3q19_dev.cu); `per` = periodic bit mask.
int launch_trt3d_dev(int dtype, void *f_out, const void *f_in, float *rho, float *ux, float *uy,
                     float *uz, const uint8_t *solid, const Grid3 &g, float sp, float sm,
                     cudaStream_t s, int variant);

}  // namespace d3
}  // namespace kb
