// kb_batch.cu -- many lid-driven MRT cavities of different sizes advanced by
// ONE persistent kernel.
//
// Physics of one case: the MRT cavity loop of test/test_mrt.jl:19-25
// (stream_2d! with half-way bounce-back, apply_zou_he_north_2d! lid,
// collide_mrt_2d! with s_e = s_eps = 1.4, s_q = 1.2, s_nu = 1/(3 nu + 1/2)),
// run to the steady residual r_u = ||u^k - u^(k-1)|| / ||u^k|| of
// src/drivers/gnf_periodic_steady.jl:186-194 or to max_steps.
//
// Storage: deviations d = f - w_q in FP16 / BF16 / FP32, collision in FP32 on
// the deviations (moments of d; no O(w) background is rounded).
//
// Schedule: the nodes of all active cases are cut into tiles of `tile_nodes`
// consecutive nodes of one case.  The kernel is launched cooperatively with
// blocks_per_sm x SMs blocks; each step the blocks stride over the active
// tile list, then meet at a grid barrier (spin bounded by an iteration
// limit; a timeout sets an error flag that every block sees and returns on).
// Every `check_every` steps the residual of each case is reduced on the device
// (FP64 atomics per tile), block 0 retires converged / finished / non-finite
// cases and compacts the tile list, and the next step runs only live tiles.
#include <vector>

#include "kb_common.cuh"

namespace kb {
namespace batch {

#ifndef KB_BATCH_THREADS
#define KB_BATCH_THREADS 256
#endif
constexpr int BT = KB_BATCH_THREADS;  // threads per block
// Blocks per SM the register allocation is sized for (__launch_bounds__).
// The pair loop keeps two pairs of pulls in flight per thread; 4 blocks give
// it the registers for that with a small spill (5 or 6 spill far more).
#ifndef KB_BATCH_MIN_BLOCKS
#define KB_BATCH_MIN_BLOCKS 4
#endif

struct CaseDesc {
    int N;
    float s_nu, u_lid;
    int pad;
    long long f_off;  // element offset of the case's 9 planes in a pool
    long long m_off;  // offset of the case's N*N moment fields
};

struct Tile {
    int c;      // case
    int start;  // first node (linear index j*N + i)
};

struct BatchState {
    void *pool_a, *pool_b;
    float *ux, *uy, *uxp, *uyp;
    const CaseDesc *cases;
    const Tile *tiles_all;
    Tile *tiles;
    int *n_tiles;       // live tile count
    double *acc;        // per case: du2, u2
    int *state;         // per case: 0 live, 1 converged, 2 max steps, 3 non-finite
    int *steps;         // per case: steps run
    float *res;         // per case: last residual
    unsigned *bar;      // [0] arrivals, [1] generation
    int *err;           // barrier timeout flag
    long long *updates; // node updates performed
};

// Bounded grid barrier for a cooperative launch.  Returns false if any block
// gave up waiting (the error flag is then set and stays set).
__device__ bool grid_barrier(const BatchState &D, unsigned nblocks, long long limit) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = D.bar + 1;
        const unsigned g = *gen;
        __threadfence();
        const unsigned arrived = atomicAdd(D.bar, 1u);
        if (arrived == nblocks - 1) {
            D.bar[0] = 0;
            __threadfence();
            atomicAdd(D.bar + 1, 1u);
        } else {
            long long it = 0;
            while (*gen == g) {
                if (++it > limit || *(volatile int *)D.err) {
                    atomicExch(D.err, 1);
                    break;
                }
                __nanosleep(128);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int *)D.err == 0;
}

template <typename R>
__device__ __forceinline__ float ldv(const R *p, int m) { return Dev<R>::ld(p[m]); }

__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < BT / 32; ++w) t += sh[w];
    return t;
}

// One node of one case: pull (half-way bounce-back), Zou-He lid on the top
// row, MRT on deviations; returns the pre-collision velocity.
template <typename R, bool SR>
__device__ __forceinline__ void node_update(const R *__restrict__ src, R *__restrict__ dst, int N,
                                            int i, int j, float s_nu, float u_lid, float &ux,
                                            float &uy, uint32_t key) {
    const int P = N * N;  // 9 N^2 < 2^31 (kb_batch_create)
    const int c = j * N + i;
    const bool w = i > 0, e = i < N - 1, s = j > 0, n = j < N - 1;
    float d[9];
    d[0] = ldv(src, c);
    d[1] = w ? ldv(src, c - 1 + P) : ldv(src, c + 3 * P);
    d[2] = s ? ldv(src, c - N + 2 * P) : ldv(src, c + 4 * P);
    d[3] = e ? ldv(src, c + 1 + 3 * P) : ldv(src, c + P);
    d[4] = n ? ldv(src, c + N + 4 * P) : ldv(src, c + 2 * P);
    d[5] = (w && s) ? ldv(src, c - 1 - N + 5 * P) : ldv(src, c + 7 * P);
    d[6] = (e && s) ? ldv(src, c + 1 - N + 6 * P) : ldv(src, c + 8 * P);
    d[7] = (e && n) ? ldv(src, c + 1 + N + 7 * P) : ldv(src, c + 5 * P);
    d[8] = (w && n) ? ldv(src, c - 1 + N + 8 * P) : ldv(src, c + 6 * P);
    if (!n) {
        // Zou-He velocity lid (boundary_2d.jl:13-42) on deviations: the
        // weights of f1+f2+f4+2(f3+f6+f7) sum to 1.
        const float rw = 1.0f + (d[0] + d[1] + d[3] + 2.0f * (d[2] + d[5] + d[6]));
        const float h = 0.5f * (d[1] - d[3]), m = 0.5f * rw * u_lid;
        d[4] = d[2];
        d[8] = d[6] - h + m;
        d[7] = d[5] + h - m;
    }
    // moments of the deviations (rows of M, collide_mrt_2d.jl:17-28)
    const float drho = d[0] + d[1] + d[2] + d[3] + d[4] + d[5] + d[6] + d[7] + d[8];
    const float dg = d[5] + d[6] + d[7] + d[8];
    const float da = d[1] + d[2] + d[3] + d[4];
    const float e_d = -4.0f * d[0] - da + 2.0f * dg;
    const float eps_d = 4.0f * d[0] - 2.0f * da + dg;
    const float jx = d[1] - d[3] + d[5] - d[6] - d[7] + d[8];
    const float qx = -2.0f * (d[1] - d[3]) + d[5] - d[6] - d[7] + d[8];
    const float jy = d[2] - d[4] + d[5] + d[6] - d[7] - d[8];
    const float qy = -2.0f * (d[2] - d[4]) + d[5] + d[6] - d[7] - d[8];
    const float pxx = d[1] - d[2] + d[3] - d[4];
    const float pxy = d[5] - d[6] + d[7] - d[8];
    const float rho = 1.0f + drho;
    const float inv = 1.0f / rho;
    ux = jx * inv;
    uy = jy * inv;
    const float r3u = 3.0f * rho * (ux * ux + uy * uy);
    const float s_e = 1.4f, s_eps = 1.4f, s_q = 1.2f;
    // post-collision deviation moments: m*_d = m_d - S (m - m_eq)
    const float es = e_d - s_e * (e_d + 2.0f * drho - r3u);
    const float ep = eps_d - s_eps * (eps_d - drho + r3u);
    const float qxs = qx - s_q * (qx + jx);
    const float qys = qy - s_q * (qy + jy);
    const float ps = pxx - s_nu * (pxx - rho * (ux * ux - uy * uy));
    const float pxys = pxy - s_nu * (pxy - rho * ux * uy);
    const float r = drho;
    const float c9 = 1.0f / 9.0f, c36 = 1.0f / 36.0f, c18 = 1.0f / 18.0f, c6 = 1.0f / 6.0f,
                c4 = 0.25f, c12 = 1.0f / 12.0f;
    const float base_a = c9 * r - c36 * es - c18 * ep;
    const float base_d = c9 * r + c18 * es + c36 * ep;
    float o[9];
    o[0] = c9 * r - c9 * es + c9 * ep;
    o[1] = base_a + c6 * jx - c6 * qxs + c4 * ps;
    o[2] = base_a + c6 * jy - c6 * qys - c4 * ps;
    o[3] = base_a - c6 * jx + c6 * qxs + c4 * ps;
    o[4] = base_a - c6 * jy + c6 * qys - c4 * ps;
    o[5] = base_d + c6 * jx + c12 * qxs + c6 * jy + c12 * qys + c4 * pxys;
    o[6] = base_d - c6 * jx - c12 * qxs + c6 * jy + c12 * qys - c4 * pxys;
    o[7] = base_d - c6 * jx - c12 * qxs - c6 * jy - c12 * qys + c4 * pxys;
    o[8] = base_d + c6 * jx + c12 * qxs - c6 * jy - c12 * qys - c4 * pxys;
    if (SR) {
        // stochastic rounding: populations (0,1), (2,3), (4,5), (6,7), (8,-)
        // share one cvt.rs and one 32-bit random word
        unsigned short *d16 = reinterpret_cast<unsigned short *>(dst);
#pragma unroll
        for (int q = 0; q < 9; q += 2) {
            const uint32_t w = SRPack<R>::pack(o[q], q + 1 < 9 ? o[q + 1] : 0.f,
                                               key * 0x7FEB352Du + (uint32_t)q * 0x2C1B3C6Du);
            d16[c + q * P] = (unsigned short)(w & 0xFFFFu);
            if (q + 1 < 9) d16[c + (q + 1) * P] = (unsigned short)(w >> 16);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 9; ++q) dst[c + q * P] = Dev<R>::st(o[q]);
    }
}

// Two x-adjacent nodes (i even, i+1) of one case per thread: N is even, so a
// pair never straddles a row, and each population of the pair is one aligned
// 2-element access except the x-shifted pulls.  The MRT collision runs on the
// pair in packed FP32x2 arithmetic.
template <typename R> struct Pair2;
template <> struct Pair2<float> {
    static __device__ __forceinline__ float2 ld(const float *p) { return *reinterpret_cast<const float2 *>(p); }
    static __device__ __forceinline__ void st(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }
};
template <> struct Pair2<__half> {
    static __device__ __forceinline__ float2 ld(const __half *p) {
        return __half22float2(*reinterpret_cast<const __half2 *>(p));
    }
    static __device__ __forceinline__ void st(__half *p, float2 v) {
        *reinterpret_cast<__half2 *>(p) = __floats2half2_rn(v.x, v.y);
    }
};
template <> struct Pair2<__nv_bfloat16> {
    static __device__ __forceinline__ float2 ld(const __nv_bfloat16 *p) {
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(p));
    }
    static __device__ __forceinline__ void st(__nv_bfloat16 *p, float2 v) {
        *reinterpret_cast<__nv_bfloat162 *>(p) = __floats2bfloat162_rn(v.x, v.y);
    }
};

// The pulls of the pair (i, j), (i + 1, j) as raw stored values v[2q] (node
// A) and v[2q + 1] (node B), not yet converted: a loop can issue the next
// pair's loads and convert them only when it collides that pair.
template <typename R> struct Raw2;
template <> struct Raw2<float> {
    static __device__ __forceinline__ void ld(const float *p, float *v) {
        const float2 t = *reinterpret_cast<const float2 *>(p);
        v[0] = t.x; v[1] = t.y;
    }
};
template <> struct Raw2<__half> {
    static __device__ __forceinline__ void ld(const __half *p, __half *v) {
        const __half2 t = *reinterpret_cast<const __half2 *>(p);
        v[0] = __low2half(t); v[1] = __high2half(t);
    }
};
template <> struct Raw2<__nv_bfloat16> {
    static __device__ __forceinline__ void ld(const __nv_bfloat16 *p, __nv_bfloat16 *v) {
        const __nv_bfloat162 t = *reinterpret_cast<const __nv_bfloat162 *>(p);
        v[0] = __low2bfloat16(t); v[1] = __high2bfloat16(t);
    }
};

template <typename R>
__device__ __forceinline__ void pair_loads_raw(const R *__restrict__ src, int N, int i, int j, R *v) {
    const int P = N * N;  // 9 N^2 < 2^31 (kb_batch_create)
    const int c = j * N + i;  // node A = (i, j), node B = (i + 1, j)
    const bool w = i > 0, e = i + 1 < N - 1, s = j > 0, n = j < N - 1;
    Raw2<R>::ld(src + c, v + 0);
    Raw2<R>::ld(s ? src + c - N + 2 * P : src + c + 4 * P, v + 4);
    Raw2<R>::ld(n ? src + c + N + 4 * P : src + c + 2 * P, v + 8);
    v[2] = w ? src[c - 1 + P] : src[c + 3 * P];
    v[3] = src[c + P];
    v[6] = src[c + 1 + 3 * P];
    v[7] = e ? src[c + 2 + 3 * P] : src[c + 1 + P];
    v[10] = (w && s) ? src[c - 1 - N + 5 * P] : src[c + 7 * P];
    v[11] = s ? src[c - N + 5 * P] : src[c + 1 + 7 * P];
    v[12] = s ? src[c + 1 - N + 6 * P] : src[c + 8 * P];
    v[13] = (e && s) ? src[c + 2 - N + 6 * P] : src[c + 1 + 8 * P];
    v[14] = n ? src[c + 1 + N + 7 * P] : src[c + 5 * P];
    v[15] = (e && n) ? src[c + 2 + N + 7 * P] : src[c + 1 + 5 * P];
    v[16] = (w && n) ? src[c - 1 + N + 8 * P] : src[c + 6 * P];
    v[17] = n ? src[c + N + 8 * P] : src[c + 1 + 6 * P];
}

// Zou-He lid (top row), MRT collision and stores of the pair whose pulled
// deviations are d[]; returns the pre-collision velocity.
template <typename R, bool SR>
__device__ __forceinline__ void pair_finish(float2 *d, R *__restrict__ dst, int N, int i, int j,
                                            float s_nu, float u_lid, float2 &ux, float2 &uy,
                                            uint32_t key) {
    const int P = N * N;  // 9 N^2 < 2^31 (kb_batch_create)
    const int c = j * N + i;
    const bool n = j < N - 1;
    const float2 z = make_float2(0.f, 0.f);
    if (!n) {
        // Zou-He velocity lid on deviations, as node_update
        const float2 rw = vadd(vsplat(1.0f, z),
                               vadd(vadd(d[0], vadd(d[1], d[3])),
                                    vmul(vsplat(2.0f, z), vadd(d[2], vadd(d[5], d[6])))));
        const float2 h = vmul(vsplat(0.5f, z), vsub(d[1], d[3]));
        const float2 m = vmul(vsplat(0.5f * u_lid, z), rw);
        d[4] = d[2];
        d[8] = vadd(vsub(d[6], h), m);
        d[7] = vsub(vadd(d[5], h), m);
    }
    const float2 drho = vadd(vadd(vadd(d[0], d[1]), vadd(d[2], d[3])),
                             vadd(vadd(d[4], d[5]), vadd(vadd(d[6], d[7]), d[8])));
    const float2 dg = vadd(vadd(d[5], d[6]), vadd(d[7], d[8]));
    const float2 da = vadd(vadd(d[1], d[2]), vadd(d[3], d[4]));
    const float2 e_d = vadd(vsub(vmul(vsplat(-4.0f, z), d[0]), da), vmul(vsplat(2.0f, z), dg));
    const float2 eps_d = vadd(vsub(vmul(vsplat(4.0f, z), d[0]), vmul(vsplat(2.0f, z), da)), dg);
    const float2 t13 = vsub(d[1], d[3]), t24 = vsub(d[2], d[4]);
    const float2 jx = vadd(t13, vsub(vsub(vadd(d[5], d[8]), d[6]), d[7]));
    const float2 qx = vadd(vmul(vsplat(-2.0f, z), t13), vsub(vsub(vadd(d[5], d[8]), d[6]), d[7]));
    const float2 jy = vadd(t24, vsub(vsub(vadd(d[5], d[6]), d[7]), d[8]));
    const float2 qy = vadd(vmul(vsplat(-2.0f, z), t24), vsub(vsub(vadd(d[5], d[6]), d[7]), d[8]));
    const float2 pxx = vsub(vadd(d[1], d[3]), vadd(d[2], d[4]));
    const float2 pxy = vsub(vadd(d[5], d[7]), vadd(d[6], d[8]));
    const float2 rho = vadd(vsplat(1.0f, z), drho);
    const float2 inv = vrcp_fast(rho);
    ux = vmul(jx, inv);
    uy = vmul(jy, inv);
    const float2 r3u = vmul(vmul(vsplat(3.0f, z), rho), vfma(ux, ux, vmul(uy, uy)));
    const float s_e = 1.4f, s_eps = 1.4f, s_q = 1.2f;
    const float2 es = vsub(e_d, vmul(vsplat(s_e, z), vsub(vadd(e_d, vmul(vsplat(2.0f, z), drho)), r3u)));
    const float2 ep = vsub(eps_d, vmul(vsplat(s_eps, z), vadd(vsub(eps_d, drho), r3u)));
    const float2 qxs = vsub(qx, vmul(vsplat(s_q, z), vadd(qx, jx)));
    const float2 qys = vsub(qy, vmul(vsplat(s_q, z), vadd(qy, jy)));
    const float2 ps = vsub(pxx, vmul(vsplat(s_nu, z), vsub(pxx, vmul(rho, vsub(vmul(ux, ux), vmul(uy, uy))))));
    const float2 pxys = vsub(pxy, vmul(vsplat(s_nu, z), vsub(pxy, vmul(rho, vmul(ux, uy)))));
    const float c9 = 1.0f / 9.0f, c36 = 1.0f / 36.0f, c18 = 1.0f / 18.0f, c6 = 1.0f / 6.0f,
                c4 = 0.25f, c12 = 1.0f / 12.0f;
    const float2 base_a = vsub(vsub(vmul(vsplat(c9, z), drho), vmul(vsplat(c36, z), es)), vmul(vsplat(c18, z), ep));
    const float2 base_d = vadd(vadd(vmul(vsplat(c9, z), drho), vmul(vsplat(c18, z), es)), vmul(vsplat(c36, z), ep));
    const float2 ax = vsub(vmul(vsplat(c6, z), jx), vmul(vsplat(c6, z), qxs));   // c6 jx - c6 qx*
    const float2 ay = vsub(vmul(vsplat(c6, z), jy), vmul(vsplat(c6, z), qys));
    const float2 bx = vadd(vmul(vsplat(c6, z), jx), vmul(vsplat(c12, z), qxs));  // c6 jx + c12 qx*
    const float2 by = vadd(vmul(vsplat(c6, z), jy), vmul(vsplat(c12, z), qys));
    const float2 p4 = vmul(vsplat(c4, z), ps), x4 = vmul(vsplat(c4, z), pxys);
    float2 o[9];
    o[0] = vmul(vsplat(c9, z), vadd(vsub(drho, es), ep));
    o[1] = vadd(vadd(base_a, ax), p4);
    o[2] = vsub(vadd(base_a, ay), p4);
    o[3] = vadd(vsub(base_a, ax), p4);
    o[4] = vsub(vsub(base_a, ay), p4);
    o[5] = vadd(vadd(vadd(base_d, bx), by), x4);
    o[6] = vsub(vadd(vsub(base_d, bx), by), x4);
    o[7] = vadd(vsub(vsub(base_d, bx), by), x4);
    o[8] = vsub(vsub(vadd(base_d, bx), by), x4);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        if (SR) {
            *reinterpret_cast<uint32_t *>(dst + c + q * P) =
                SRPack<R>::pack(o[q].x, o[q].y, key * 0x7FEB352Du + (uint32_t)q * 0x2C1B3C6Du);
        } else {
            Pair2<R>::st(dst + c + q * P, o[q]);
        }
    }
}

template <typename R, bool SR>
__global__ void __launch_bounds__(BT, KB_BATCH_MIN_BLOCKS) batch_k(BatchState D, int n_cases, int n_tiles_all, int tile_nodes,
                                               int max_steps, int check_every, float tol,
                                               long long spin_limit, uint32_t seed) {
    __shared__ double sh[BT / 32];
    const unsigned nblocks = gridDim.x;
    for (int s = 0;; ++s) {
        const int nt = *(volatile int *)D.n_tiles;
        if (nt == 0) break;
        const R *src = (const R *)((s & 1) ? D.pool_b : D.pool_a);
        R *dst = (R *)((s & 1) ? D.pool_a : D.pool_b);
        const bool check = (s + 1) % check_every == 0;
        const bool save = (s + 2) % check_every == 0;
        for (int t = blockIdx.x; t < nt; t += nblocks) {
            const Tile T = D.tiles[t];
            const CaseDesc C = D.cases[T.c];
            const int NN = C.N * C.N;
            const int end = min(T.start + tile_nodes, NN);
            double du2 = 0.0, u2 = 0.0;
            if (C.N & 1) {
                // odd N: rows start at odd offsets, so one node per thread
                for (int m = T.start + threadIdx.x; m < end; m += BT) {
                    const int j = m / C.N, i = m - j * C.N;
                    float ux, uy;
                    const uint32_t key =
                        SR ? hash32((uint32_t)(C.f_off + m) ^ hash32((uint32_t)s * 0x632BE5ABu + seed)) : 0u;
                    node_update<R, SR>(src + C.f_off, dst + C.f_off, C.N, i, j, C.s_nu, C.u_lid, ux, uy,
                                       key);
                    const long long mo = C.m_off + m;
                    if (save) { D.uxp[mo] = ux; D.uyp[mo] = uy; }
                    if (check) {
                        D.ux[mo] = ux;
                        D.uy[mo] = uy;
                        const double a = (double)ux - (double)D.uxp[mo];
                        const double b = (double)uy - (double)D.uyp[mo];
                        du2 += a * a + b * b;
                        u2 += (double)ux * ux + (double)uy * uy;
                    }
                }
            } else {
            // node pairs (m, m + 1): tiles start at multiples of 32, N is even
            // and case offsets are multiples of 64, so every pair is aligned;
            // software-pipelined: the next pair's pulls are in flight (as raw
            // stored values) while this pair collides
            // (i, j) of node m advance by the stride 2 BT with one division
            // per tile, not per pair: 2 BT = dj rows + di columns (di even)
            R vn[18];
            int m = T.start + 2 * threadIdx.x;
            int j = m / C.N, i = m - j * C.N;
            const int dj = (2 * BT) / C.N, di = 2 * BT - dj * C.N;
            if (m < end) pair_loads_raw<R>(src + C.f_off, C.N, i, j, vn);
            for (; m < end; m += 2 * BT) {
                float2 d[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) d[q] = make_float2(Dev<R>::ld(vn[2 * q]), Dev<R>::ld(vn[2 * q + 1]));
                int in = i + di, jn = j + dj;
                if (in >= C.N) { in -= C.N; ++jn; }
                const int mn = m + 2 * BT;
                if (mn < end) pair_loads_raw<R>(src + C.f_off, C.N, in, jn, vn);
                float2 ux, uy;
                const uint32_t key =
                    SR ? hash32((uint32_t)(C.f_off + m) ^ hash32((uint32_t)s * 0x632BE5ABu + seed)) : 0u;
                pair_finish<R, SR>(d, dst + C.f_off, C.N, i, j, C.s_nu, C.u_lid, ux, uy, key);
                const long long mo = C.m_off + m;
                if (save) {
                    *reinterpret_cast<float2 *>(D.uxp + mo) = ux;
                    *reinterpret_cast<float2 *>(D.uyp + mo) = uy;
                }
                if (check) {
                    *reinterpret_cast<float2 *>(D.ux + mo) = ux;
                    *reinterpret_cast<float2 *>(D.uy + mo) = uy;
                    const float2 px = *reinterpret_cast<const float2 *>(D.uxp + mo);
                    const float2 py = *reinterpret_cast<const float2 *>(D.uyp + mo);
                    const double a0 = (double)ux.x - px.x, b0 = (double)uy.x - py.x;
                    const double a1 = (double)ux.y - px.y, b1 = (double)uy.y - py.y;
                    du2 += a0 * a0 + b0 * b0 + a1 * a1 + b1 * b1;
                    u2 += (double)ux.x * ux.x + (double)uy.x * uy.x + (double)ux.y * ux.y +
                          (double)uy.y * uy.y;
                }
                i = in;
                j = jn;
            }
            }
            if (check) {
                const double a = block_sum(du2, sh);
                const double b = block_sum(u2, sh);
                if (threadIdx.x == 0) {
                    atomicAdd(&D.acc[2 * T.c], a);
                    atomicAdd(&D.acc[2 * T.c + 1], b);
                }
            }
            if (threadIdx.x == 0) atomicAdd((unsigned long long *)D.updates,
                                            (unsigned long long)(end - T.start));
        }
        if (!grid_barrier(D, nblocks, spin_limit)) return;
        if (!check) continue;
        if (blockIdx.x == 0) {
            // retire cases, then compact the tile list in order
            for (int c = threadIdx.x; c < n_cases; c += BT) {
                if (D.state[c] != 0) continue;
                const double du2 = D.acc[2 * c], u2 = D.acc[2 * c + 1];
                const double r = sqrt(du2 / u2);
                D.steps[c] = s + 1;
                D.res[c] = (float)r;
                if (!isfinite(r)) D.state[c] = 3;
                else if (r < tol) D.state[c] = 1;
                else if (s + 1 >= max_steps) D.state[c] = 2;
                D.acc[2 * c] = 0.0;
                D.acc[2 * c + 1] = 0.0;
            }
            __syncthreads();
            __shared__ int base;
            __shared__ int wsum[BT / 32];
            if (threadIdx.x == 0) base = 0;
            __syncthreads();
            for (int t0 = 0; t0 < n_tiles_all; t0 += BT) {
                const int t = t0 + threadIdx.x;
                Tile T = {0, 0};
                bool live = false;
                if (t < n_tiles_all) {
                    T = D.tiles_all[t];
                    live = D.state[T.c] == 0;
                }
                const unsigned bal = __ballot_sync(0xffffffffu, live);
                const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
                if (lane == 0) wsum[warp] = __popc(bal);
                __syncthreads();
                int off = base;
                for (int w2 = 0; w2 < warp; ++w2) off += wsum[w2];
                off += __popc(bal & ((1u << lane) - 1u));
                if (live) D.tiles[off] = T;
                __syncthreads();
                if (threadIdx.x == 0)
                    for (int w2 = 0; w2 < BT / 32; ++w2) base += wsum[w2];
                __syncthreads();
            }
            if (threadIdx.x == 0) *D.n_tiles = base;
        }
        if (!grid_barrier(D, nblocks, spin_limit)) return;
    }
}

}  // namespace batch
}  // namespace kb

// ------------------------------------------------------------------- host --
struct kb_batch {
    int n_cases = 0, dtype = KB_F16_DEV, n_tiles_all = 0, tile_nodes = 0;
    int device = 0;
    std::vector<int> N;
    std::vector<double> nu, u_lid;
    std::vector<kb::batch::CaseDesc> cases_h;
    long long pool_elems = 0, moment_elems = 0;
    void *pool_a = nullptr, *pool_b = nullptr;
    float *mom = nullptr;  // ux, uy, uxp, uyp
    kb::batch::CaseDesc *cases = nullptr;
    kb::batch::Tile *tiles_all = nullptr, *tiles = nullptr;
    char *scal = nullptr;  // n_tiles, bar[2], err, updates, acc, state, steps, res
    int tuned_tile = 0, tuned_bpsm = 0;
    unsigned runs = 0;  // launches so far; seeds the stochastic-rounding bits
};

namespace {

using namespace kb::batch;

int cuda_err(const char *what, cudaError_t e) {
    return kb::set_error(KB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

struct ScalLayout {
    size_t n_tiles, bar, err, updates, acc, state, steps, res, total;
};

ScalLayout scal_layout(int n_cases) {
    ScalLayout L;
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t r = o; o += (bytes + 255) & ~size_t(255); return r; };
    L.n_tiles = take(sizeof(int));
    L.bar = take(2 * sizeof(unsigned));
    L.err = take(sizeof(int));
    L.updates = take(sizeof(long long));
    L.acc = take(2 * sizeof(double) * n_cases);
    L.state = take(sizeof(int) * n_cases);
    L.steps = take(sizeof(int) * n_cases);
    L.res = take(sizeof(float) * n_cases);
    L.total = o;
    return L;
}

size_t elem_bytes(int dtype) { return kb::dtype_bytes(dtype); }

int build_tiles(kb_batch *b, int tile_nodes) {
    std::vector<Tile> t;
    for (int c = 0; c < b->n_cases; ++c) {
        const int NN = b->N[c] * b->N[c];
        for (int s = 0; s < NN; s += tile_nodes) t.push_back(Tile{c, s});
    }
    if (b->tiles_all) { cudaFree(b->tiles_all); b->tiles_all = nullptr; }
    if (b->tiles) { cudaFree(b->tiles); b->tiles = nullptr; }
    cudaError_t e = cudaMalloc(&b->tiles_all, sizeof(Tile) * t.size());
    if (e == cudaSuccess) e = cudaMalloc(&b->tiles, sizeof(Tile) * t.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(b->tiles_all, t.data(), sizeof(Tile) * t.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_err("kb_batch: tile list", e);
    b->n_tiles_all = (int)t.size();
    b->tile_nodes = tile_nodes;
    return KB_OK;
}

// Reset populations to rest (d = 0), states to live and the live list to all
// tiles; all on `s`.
int reset(kb_batch *b, cudaStream_t s) {
    const size_t eb = elem_bytes(b->dtype);
    const ScalLayout L = scal_layout(b->n_cases);
    cudaError_t e = cudaMemsetAsync(b->pool_a, 0, eb * b->pool_elems, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->pool_b, 0, eb * b->pool_elems, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->mom, 0, sizeof(float) * 4 * b->moment_elems, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->scal, 0, L.total, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->tiles, b->tiles_all, sizeof(Tile) * b->n_tiles_all,
                            cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->scal + L.n_tiles, &b->n_tiles_all, sizeof(int),
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_err("kb_batch_reset", e);
    return KB_OK;
}

template <typename R, bool SR = false>
int launch(kb_batch *b, int max_steps, int check_every, double tol, int blocks_per_sm,
           cudaStream_t s) {
    const ScalLayout L = scal_layout(b->n_cases);
    BatchState D;
    D.pool_a = b->pool_a; D.pool_b = b->pool_b;
    D.ux = b->mom; D.uy = b->mom + b->moment_elems;
    D.uxp = b->mom + 2 * b->moment_elems; D.uyp = b->mom + 3 * b->moment_elems;
    D.cases = b->cases; D.tiles_all = b->tiles_all; D.tiles = b->tiles;
    D.n_tiles = (int *)(b->scal + L.n_tiles);
    D.bar = (unsigned *)(b->scal + L.bar);
    D.err = (int *)(b->scal + L.err);
    D.updates = (long long *)(b->scal + L.updates);
    D.acc = (double *)(b->scal + L.acc);
    D.state = (int *)(b->scal + L.state);
    D.steps = (int *)(b->scal + L.steps);
    D.res = (float *)(b->scal + L.res);
    int occ = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_k<R, SR>, BT, 0);
    if (e != cudaSuccess) return cuda_err("kb_batch_run: occupancy", e);
    const int bpsm = blocks_per_sm < 1 ? occ : (blocks_per_sm < occ ? blocks_per_sm : occ);
    if (bpsm < 1) return kb::set_error(KB_ERR_UNSUPPORTED, "kb_batch_run: kernel does not fit an SM");
    int n_cases = b->n_cases, n_all = b->n_tiles_all, tn = b->tile_nodes;
    float tolf = (float)tol;
    // ~ 2^24 waits of >= 128 ns: a barrier that has not opened after a few
    // seconds is declared timed out
    long long spin = 1ll << 24;
    uint32_t seed = b->runs++;  // fresh random bits for every run of the batch
    void *args[] = {&D, &n_cases, &n_all, &tn, &max_steps, &check_every, &tolf, &spin, &seed};
    dim3 grid(bpsm * kb::sm_count()), block(BT);
    e = cudaLaunchCooperativeKernel((void *)batch_k<R, SR>, grid, block, args, 0, s);
    if (e != cudaSuccess) return cuda_err("kb_batch_run: cooperative launch", e);
    return KB_OK;
}

// Resident blocks per SM of the batched kernel for a storage.
int batch_occupancy(int dtype) {
    int occ = 0;
    cudaError_t e;
    switch (dtype) {
        case KB_F16_DEV: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_k<__half, false>, BT, 0); break;
        case KB_BF16_DEV: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_k<__nv_bfloat16, false>, BT, 0); break;
        case KB_F16_DEV_SR: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_k<__half, true>, BT, 0); break;
        case KB_BF16_DEV_SR: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_k<__nv_bfloat16, true>, BT, 0); break;
        default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_k<float, false>, BT, 0); break;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return occ;
}

}  // namespace

extern "C" {

int kb_batch_create(kb_batch **out, int n_cases, const int *N, const double *nu,
                    const double *u_lid, int dtype, void *stream) {
    KB_REQUIRE(out && N && nu && u_lid, "kb_batch_create: null pointer");
    KB_REQUIRE(n_cases > 0, "kb_batch_create: n_cases must be positive");
    KB_REQUIRE(dtype == KB_F16_DEV || dtype == KB_BF16_DEV || dtype == KB_F32_DEV ||
                   dtype == KB_F16_DEV_SR || dtype == KB_BF16_DEV_SR,
               "kb_batch_create: storage must be KB_F16_DEV, KB_BF16_DEV, KB_F32_DEV or a "
               "stochastic-rounding 16-bit storage");
    int coop = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) return kb::set_error(KB_ERR_UNSUPPORTED, "kb_batch_create: device lacks cooperative launch");
    kb_batch *b = new kb_batch();
    b->n_cases = n_cases; b->dtype = dtype; b->device = dev;
    long long fo = 0, mo = 0;
    for (int c = 0; c < n_cases; ++c) {
        // a case's 9 N^2 population elements are addressed with 32-bit offsets
        if (N[c] < 2 || N[c] > 15000 || !(nu[c] > 0.0)) {
            delete b;
            return kb::set_error(KB_ERR_ARG, "kb_batch_create: case %d has N=%d nu=%g", c, N[c], nu[c]);
        }
        b->N.push_back(N[c]); b->nu.push_back(nu[c]); b->u_lid.push_back(u_lid[c]);
        CaseDesc d;
        d.N = N[c];
        d.s_nu = (float)(1.0 / (3.0 * nu[c] + 0.5));
        d.u_lid = (float)u_lid[c];
        d.pad = 0;
        d.f_off = fo;
        d.m_off = mo;
        b->cases_h.push_back(d);
        const long long NN = (long long)N[c] * N[c];
        fo += (9 * NN + 63) / 64 * 64;
        mo += (NN + 63) / 64 * 64;
    }
    b->pool_elems = fo; b->moment_elems = mo;
    const size_t eb = elem_bytes(dtype);
    const ScalLayout L = scal_layout(n_cases);
    cudaError_t e = cudaMalloc(&b->pool_a, eb * fo);
    if (e == cudaSuccess) e = cudaMalloc(&b->pool_b, eb * fo);
    if (e == cudaSuccess) e = cudaMalloc(&b->mom, sizeof(float) * 4 * mo);
    if (e == cudaSuccess) e = cudaMalloc(&b->cases, sizeof(CaseDesc) * n_cases);
    if (e == cudaSuccess) e = cudaMalloc(&b->scal, L.total);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->cases, b->cases_h.data(), sizeof(CaseDesc) * n_cases, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaGetLastError();
        kb_batch_destroy(b);
        return kb::set_error(KB_ERR_NOMEM, "kb_batch_create: device allocation failed: %s",
                             cudaGetErrorString(e));
    }
    if (int r = build_tiles(b, 256)) { kb_batch_destroy(b); return r; }
    if (int r = reset(b, kb::as_stream(stream))) { kb_batch_destroy(b); return r; }
    *out = b;
    return KB_OK;
}

int kb_batch_destroy(kb_batch *b) {
    if (!b) return KB_OK;
    cudaFree(b->pool_a); cudaFree(b->pool_b); cudaFree(b->mom); cudaFree(b->cases);
    cudaFree(b->scal); cudaFree(b->tiles_all); cudaFree(b->tiles);
    delete b;
    return KB_OK;
}

int kb_batch_reset(kb_batch *b, void *stream) {
    KB_REQUIRE(b, "kb_batch_reset: null handle");
    return reset(b, kb::as_stream(stream));
}

int kb_batch_run(kb_batch *b, int max_steps, int check_every, double tol, int tile_nodes,
                 int blocks_per_sm, void *stream) {
    KB_REQUIRE(b, "kb_batch_run: null handle");
    KB_REQUIRE(check_every >= 2, "kb_batch_run: check_every must be >= 2");
    KB_REQUIRE(max_steps >= check_every && max_steps % check_every == 0,
               "kb_batch_run: max_steps must be a positive multiple of check_every");
    if (tile_nodes <= 0) tile_nodes = b->tuned_tile > 0 ? b->tuned_tile : 256;
    if (blocks_per_sm <= 0) blocks_per_sm = b->tuned_bpsm > 0 ? b->tuned_bpsm : 0;
    KB_REQUIRE(tile_nodes % 32 == 0 && tile_nodes <= (1 << 20),
               "kb_batch_run: tile_nodes must be a multiple of 32");
    cudaStream_t s = kb::as_stream(stream);
    if (tile_nodes != b->tile_nodes) {
        if (int r = build_tiles(b, tile_nodes)) return r;
        if (int r = reset(b, s)) return r;
    }
    switch (b->dtype) {
        case KB_F16_DEV: return launch<__half>(b, max_steps, check_every, tol, blocks_per_sm, s);
        case KB_BF16_DEV: return launch<__nv_bfloat16>(b, max_steps, check_every, tol, blocks_per_sm, s);
        case KB_F16_DEV_SR: return launch<__half, true>(b, max_steps, check_every, tol, blocks_per_sm, s);
        case KB_BF16_DEV_SR:
            return launch<__nv_bfloat16, true>(b, max_steps, check_every, tol, blocks_per_sm, s);
        default: return launch<float>(b, max_steps, check_every, tol, blocks_per_sm, s);
    }
}

int kb_batch_status(kb_batch *b, long long *updates, int *n_live, int *timed_out, void *stream) {
    KB_REQUIRE(b, "kb_batch_status: null handle");
    const ScalLayout L = scal_layout(b->n_cases);
    cudaStream_t s = kb::as_stream(stream);
    int nt = 0, err = 0;
    long long up = 0;
    cudaError_t e = cudaMemcpyAsync(&nt, b->scal + L.n_tiles, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, b->scal + L.err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&up, b->scal + L.updates, sizeof(long long), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_err("kb_batch_status", e);
    if (updates) *updates = up;
    if (n_live) *n_live = nt;
    if (timed_out) *timed_out = err;
    if (err) return kb::set_error(KB_ERR_TIMEOUT, "kb_batch: a grid barrier timed out");
    return KB_OK;
}

int kb_batch_case(kb_batch *b, int c, int *N, int *steps, double *residual, int *state,
                  float *ux_host, float *uy_host, void *stream) {
    KB_REQUIRE(b, "kb_batch_case: null handle");
    KB_REQUIRE(c >= 0 && c < b->n_cases, "kb_batch_case: case %d out of range", c);
    const ScalLayout L = scal_layout(b->n_cases);
    cudaStream_t s = kb::as_stream(stream);
    int st = 0, sp = 0;
    float r = 0.f;
    cudaError_t e = cudaMemcpyAsync(&st, b->scal + L.state + sizeof(int) * c, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&sp, b->scal + L.steps + sizeof(int) * c, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&r, b->scal + L.res + sizeof(float) * c, sizeof(float), cudaMemcpyDeviceToHost, s);
    const long long NN = (long long)b->N[c] * b->N[c];
    const long long mo = b->cases_h[c].m_off;
    if (e == cudaSuccess && ux_host)
        e = cudaMemcpyAsync(ux_host, b->mom + mo, sizeof(float) * NN, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && uy_host)
        e = cudaMemcpyAsync(uy_host, b->mom + b->moment_elems + mo, sizeof(float) * NN, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_err("kb_batch_case", e);
    if (N) *N = b->N[c];
    if (steps) *steps = sp;
    if (residual) *residual = r;
    if (state) *state = st;
    return KB_OK;
}

int kb_batch_autotune(kb_batch *b, int trial_steps, int *best_tile, int *best_bpsm,
                      double *best_mlups, double *fixed_mlups, void *stream) {
    KB_REQUIRE(b, "kb_batch_autotune: null handle");
    KB_REQUIRE(trial_steps >= 2 && trial_steps % 2 == 0, "kb_batch_autotune: trial_steps must be even and >= 2");
    cudaStream_t s = kb::as_stream(stream);
    // the candidates: tile sizes x every residency up to the occupancy limit;
    // the fixed schedule is what kb_batch_run takes untuned (256-node tiles,
    // as many blocks per SM as fit)
    const int occ = batch_occupancy(b->dtype);
    if (occ < 1) return kb::set_error(KB_ERR_UNSUPPORTED, "kb_batch_autotune: kernel does not fit an SM");
    const int tiles[] = {256, 512, 1024, 2048, 4096};
    double best = -1.0, fixed = -1.0;
    int bt = 256, bb = occ;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int tn : tiles)
        for (int bp = 1; bp <= occ; ++bp) {
            if (int r = build_tiles(b, tn)) return r;
            if (int r = reset(b, s)) return r;
            cudaEventRecord(e0, s);
            if (int r = kb_batch_run(b, trial_steps, trial_steps, 0.0, tn, bp, stream)) return r;
            cudaEventRecord(e1, s);
            cudaError_t e = cudaEventSynchronize(e1);
            if (e != cudaSuccess) return cuda_err("kb_batch_autotune", e);
            long long up = 0;
            int live = 0, tout = 0;
            if (int r = kb_batch_status(b, &up, &live, &tout, stream)) return r;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            const double mlups = (double)up / (ms * 1e-3) / 1e6;
            if (tn == 256 && bp == occ) fixed = mlups;
            if (mlups > best) { best = mlups; bt = tn; bb = bp; }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->tuned_tile = bt;
    b->tuned_bpsm = bb;
    if (int r = build_tiles(b, bt)) return r;
    if (int r = reset(b, s)) return r;
    if (best_tile) *best_tile = bt;
    if (best_bpsm) *best_bpsm = bb;
    if (best_mlups) *best_mlups = best;
    if (fixed_mlups) *fixed_mlups = fixed;
    return KB_OK;
}

// Device pointer of case c's populations after its last step (the buffer
// its final step wrote), for conversions and error checks.
int kb_batch_populations(kb_batch *b, int c, void **f, int *dtype, void *stream) {
    KB_REQUIRE(b && f, "kb_batch_populations: null pointer");
    KB_REQUIRE(c >= 0 && c < b->n_cases, "kb_batch_populations: case %d out of range", c);
    int steps = 0;
    if (int r = kb_batch_case(b, c, nullptr, &steps, nullptr, nullptr, nullptr, nullptr, stream)) return r;
    void *pool = (steps % 2 == 1) ? b->pool_b : b->pool_a;
    *f = (char *)pool + elem_bytes(b->dtype) * b->cases_h[c].f_off;
    if (dtype) *dtype = b->dtype;
    return KB_OK;
}

}  // extern "C"
