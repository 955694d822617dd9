// kb_umma.cuh -- tcgen05 (UMMA) BF16 tensor-core mainloop for sm_100a, and the
// operand loaders of the warm-start network's convolutions.
//
// One CTA = 128 threads (4 warps) computes one 128 x BN tile of D (FP32, in
// TMEM) over a range of 64-wide K steps:
//   * all 128 threads stage the A tile (128 x 64 BF16) and the B tile
//     (BN x 64) of a K step into shared memory with 16-byte cp.async copies
//     (zero-fill for padding), in the canonical no-swizzle UMMA layout
//     (16-byte rows, 8-row core matrices);
//   * one thread issues four tcgen05.mma.cta_group::1.kind::f16 (M=128, N=BN,
//     K=16) and commits them to the stage's mbarrier;
//   * STAGES shared-memory stages rotate: while the tensor core works on step
//     k, the copies of steps k+1 .. k+STAGES-1 are in flight;
//   * the epilogue reads the accumulator with tcgen05.ld.32x32b (warp w owns
//     TMEM lanes 32w..32w+31 = tile rows) and hands 8 columns at a time to the
//     operation's store().
//
// Shared-memory layouts (both with SBO = 128 B between 8-row groups along
// M/N and LBO = rows*16 B between 8-element groups along K):
//   K-major : element (r, k) at (k/8)*rows*16 + r*16 + (k%8)*2
//   MN-major: element (r, k) at (k/8)*rows*16 + (r/8)*128 + (k%8)*16 + (r%8)*2
// A K-major 16-byte chunk is 8 consecutive k of one row; an MN-major chunk is
// 8 consecutive rows of one k.  The instruction descriptor's a_major/b_major
// bits select the layout per operand.
//
// Every wait is bounded.  A CTA that gives up records the failure in *err,
// waits (bounded) for the MMAs it issued, frees its TMEM and returns.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace kb {
namespace umma {

constexpr int BM = 128, BK = 64, NT = 128, THREADS = 128;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, no swizzle, sm_100 version field = 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor, kind::f16: D F32, A = B = BF16, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(int N, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) |
           ((b_mn ? 1u : 0u) << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit) {
    const uint32_t a = smem_u32(bar);
    for (long long it = 0; it < limit; ++it) {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (it > 64) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v) {
    uint32_t r[8];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// 16-byte asynchronous global->shared copy; valid = false writes zeros (the
// source pointer must still be a valid address; callers pass a tensor base).
__device__ __forceinline__ void cp16(uint32_t saddr, const void *g, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr), "l"(g),
                 "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

constexpr int STAGES = 3;
struct Smem {
    alignas(128) unsigned char a[STAGES][BM * BK * 2];  // 16 KB per stage
    alignas(128) unsigned char b[STAGES][NT * BK * 2];  // 16 KB per stage
    uint64_t bar[STAGES + 1];
    uint32_t tmem;
};

__host__ __device__ constexpr uint32_t tmem_cols(int bn) { return bn <= 32 ? 32u : (bn <= 64 ? 64u : 128u); }

// Op interface:
//   static constexpr bool A_MN, B_MN;
//   int bn;                                     N tile width (16..128, multiple of 16)
//   __device__ void k_range(const uint3 &t, int &k0, int &k1)  K steps of tile t
//   __device__ void load_a(uint32_t s, int kt, const uint3 &t)  cp.async the 128 x 64 A tile
//   __device__ void load_b(uint32_t s, int kt, const uint3 &t)  cp.async the bn x 64 B tile
//   __device__ void store(int row, int col, const float *v, const uint3 &t)  8 columns of row
// (t = the tile's (m, n, split) coordinates; loads are issued by threads 0..127)
template <class Op>
__global__ void __launch_bounds__(THREADS) umma_k(const Op op, int *__restrict__ err, long long spin) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    Smem &S = *reinterpret_cast<Smem *>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bn = op.bn;
    const uint32_t cols = tmem_cols(bn);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&S.tmem)), "r"(cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i <= STAGES; ++i) mbar_init(&S.bar[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = S.tmem;
    const uint32_t idesc = idesc_bf16(bn, Op::A_MN, Op::B_MN);
    int k0, k1;
    const uint3 tile = blockIdx;
    op.k_range(tile, k0, k1);
    const int n = k1 - k0;
    const uint32_t lbo_a = BM * 16, lbo_b = (uint32_t)bn * 16;
    const uint32_t sa0 = smem_u32(S.a[0]), sb0 = smem_u32(S.b[0]);
    constexpr uint32_t SA = BM * BK * 2, SB = NT * BK * 2;

#pragma unroll
    for (int i = 0; i < STAGES - 1; ++i) {
        if (i < n) {
            op.load_a(sa0 + i * SA, k0 + i, tile);
            op.load_b(sb0 + i * SB, k0 + i, tile);
        }
        cp_commit();
    }
    uint32_t phase_bits = 0;
    bool ok = true;
    for (int i = 0; i < n; ++i) {
        const int s = i % STAGES;
        cp_wait<STAGES - 2>();  // this thread's copies of step i have landed
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        // one barrier per step; it also makes a timeout a block-uniform exit
        if (!__syncthreads_and(ok ? 1 : 0)) {
            ok = false;
            break;
        }
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = sa0 + s * SA, sb = sb0 + s * SB;
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
                const uint64_t da = sdesc(sa + kk * 2 * lbo_a, lbo_a, 128);
                const uint64_t db = sdesc(sb + kk * 2 * lbo_b, lbo_b, 128);
                mma_bf16(tmem, da, db, idesc, (i > 0 || kk > 0) ? 1u : 0u);
            }
            mma_commit(&S.bar[s]);
        }
        // refill the stage that step i-1 used, once its MMAs are done
        const int nx = i + STAGES - 1;
        if (nx < n) {
            const int sp = nx % STAGES;
            if (i >= 1) {
                ok = mbar_wait(&S.bar[sp], (phase_bits >> sp) & 1u, spin);
                phase_bits ^= 1u << sp;
            }
            if (ok) {
                op.load_a(sa0 + sp * SA, k0 + nx, tile);
                op.load_b(sb0 + sp * SB, k0 + nx, tile);
            }
        }
        cp_commit();
    }
    cp_wait<0>();
    // One more commit tracks every MMA this thread issued; wait for it on all
    // paths (also after a timeout) before reading or freeing TMEM.
    const bool issued = n > 0;
    if (threadIdx.x == 0 && issued) mma_commit(&S.bar[STAGES]);
    const bool drained = !issued || mbar_wait(&S.bar[STAGES], 0u, spin);
    ok = ok && drained;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool all_ok = __syncthreads_and(ok ? 1 : 0);
    const int row = warp * 32 + lane;
    if (!all_ok) {
        if (threadIdx.x == 0) atomicExch(err, 1);
    } else if (issued) {
        for (int c0 = 0; c0 < bn; c0 += 8) {
            float v[8];
            tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            op.store(row, c0, v, tile);
        }
    } else {
        const float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int c0 = 0; c0 < bn; c0 += 8) op.store(row, c0, z, tile);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols));
}

inline size_t smem_bytes() { return sizeof(Smem) + 1024; }

// ---------------------------------------------------------------------------
// Warp-specialised persistent form of the mainloop.  One CTA per SM loops
// over the tiles t = blockIdx.x, blockIdx.x + gridDim.x, ... of the grid
// `tiles` (x fastest):
//   warps 0-3  producers: cp.async every K step of every tile into a ring of
//              WS_STAGES shared-memory stages; after a step's copies land
//              (one step of lag), each producer thread fences them to the
//              async proxy and arrives on the stage's `full` barrier
//   warp 8     MMA: lane 0 waits `full`, issues the four tcgen05.mma of the
//              step into one of two TMEM accumulators, commits to the stage's
//              `empty` barrier, and after a tile's last step to `acc_full`
//   warps 4-7  epilogue: warp w reads TMEM lanes 32(w%4)..+31 of the finished
//              accumulator, calls op.store, and arrives on `acc_empty`
// so the loads of the next steps and the epilogue of tile j overlap the MMAs
// of tile j+1.  Every wait is bounded; a role that gives up stops, sets *err,
// and the others run out of their own bounded waits.
constexpr int WS_STAGES = 4, WS_THREADS = 288;

struct SmemWS {
    alignas(128) unsigned char a[WS_STAGES][BM * BK * 2];
    alignas(128) unsigned char b[WS_STAGES][NT * BK * 2];
    uint64_t full[WS_STAGES], empty[WS_STAGES], acc_full[2], acc_empty[2], drain;
    uint32_t tmem;
};

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ uint3 tile_of(long long T, const uint3 &n) {
    uint3 t;
    t.x = (unsigned)(T % n.x);
    const long long r = T / n.x;
    t.y = (unsigned)(r % n.y);
    t.z = (unsigned)(r / n.y);
    return t;
}

template <class Op>
__global__ void __launch_bounds__(WS_THREADS, 1) umma_ws_k(const Op op, const uint3 tiles,
                                                           int *__restrict__ err, long long spin) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    SmemWS &S = *reinterpret_cast<SmemWS *>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bn = op.bn;
    const uint32_t cols = tmem_cols(bn);  // per accumulator; two of them
    const long long ntiles = (long long)tiles.x * tiles.y * tiles.z;
    constexpr uint32_t SA = BM * BK * 2, SB = NT * BK * 2;

    if (warp == 8) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&S.tmem)), "r"(2 * cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < WS_STAGES; ++i) {
            mbar_init(&S.full[i], 128);
            mbar_init(&S.empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&S.acc_full[i], 1);
            mbar_init(&S.acc_empty[i], 128);
        }
        mbar_init(&S.drain, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = S.tmem;
    bool ok = true;

    if (warp < 4) {
        // ------------------------------------------------------ producers
        const uint32_t sa0 = smem_u32(S.a[0]), sb0 = smem_u32(S.b[0]);
        long long g = 0;
        for (long long T = blockIdx.x; T < ntiles && ok; T += gridDim.x) {
            const uint3 t = tile_of(T, tiles);
            int k0, k1;
            op.k_range(t, k0, k1);
            for (int kt = k0; kt < k1; ++kt, ++g) {
                const int s = (int)(g % WS_STAGES);
                const long long use = g / WS_STAGES;
                if (use >= 1) {
                    ok = mbar_wait(&S.empty[s], (uint32_t)((use - 1) & 1), spin);
                    if (!ok) break;
                }
                op.load_a(sa0 + s * SA, kt, t);
                op.load_b(sb0 + s * SB, kt, t);
                cp_commit();
                if (g >= 1) {
                    cp_wait<1>();
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    mbar_arrive(&S.full[(g - 1) % WS_STAGES]);
                }
            }
        }
        cp_wait<0>();
        if (ok && g >= 1) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(&S.full[(g - 1) % WS_STAGES]);
        }
    } else if (warp == 8) {
        // ------------------------------------------------------ MMA issue
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16(bn, Op::A_MN, Op::B_MN);
            const uint32_t lbo_a = BM * 16, lbo_b = (uint32_t)bn * 16;
            const uint32_t sa0 = smem_u32(S.a[0]), sb0 = smem_u32(S.b[0]);
            long long g = 0;
            int j = 0;
            bool issued = false;
            for (long long T = blockIdx.x; T < ntiles && ok; T += gridDim.x, ++j) {
                const int buf = j & 1;
                if (j >= 2) {
                    ok = mbar_wait(&S.acc_empty[buf], (uint32_t)(((j >> 1) - 1) & 1), spin);
                    if (!ok) break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint3 t = tile_of(T, tiles);
                int k0, k1;
                op.k_range(t, k0, k1);
                const uint32_t acc = tmem + (uint32_t)buf * cols;
                for (int kt = k0; kt < k1; ++kt, ++g) {
                    const int s = (int)(g % WS_STAGES);
                    ok = mbar_wait(&S.full[s], (uint32_t)((g / WS_STAGES) & 1), spin);
                    if (!ok) break;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sa = sa0 + s * SA, sb = sb0 + s * SB;
#pragma unroll
                    for (int kk = 0; kk < BK / 16; ++kk) {
                        const uint64_t da = sdesc(sa + kk * 2 * lbo_a, lbo_a, 128);
                        const uint64_t db = sdesc(sb + kk * 2 * lbo_b, lbo_b, 128);
                        mma_bf16(acc, da, db, idesc, (kt > k0 || kk > 0) ? 1u : 0u);
                    }
                    mma_commit(&S.empty[s]);
                    issued = true;
                }
                if (!ok) break;
                mma_commit(&S.acc_full[buf]);
            }
            // every MMA issued above is complete once this commit arrives
            mma_commit(&S.drain);
            if (!mbar_wait(&S.drain, 0u, spin)) ok = false;
            (void)issued;
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------ epilogue
        const int q = warp & 3;
        const int row = q * 32 + lane;
        int j = 0;
        for (long long T = blockIdx.x; T < ntiles && ok; T += gridDim.x, ++j) {
            const int buf = j & 1;
            ok = mbar_wait(&S.acc_full[buf], (uint32_t)((j >> 1) & 1), spin);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint3 t = tile_of(T, tiles);
            int k0, k1;
            op.k_range(t, k0, k1);
            if (k1 > k0) {
                for (int c0 = 0; c0 < bn; c0 += 8) {
                    float v[8];
                    tmem_ld8(tmem + (uint32_t)buf * cols + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, v);
                    op.store(row, c0, v, t);
                }
            } else {
                const float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                for (int c0 = 0; c0 < bn; c0 += 8) op.store(row, c0, z, t);
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            mbar_arrive(&S.acc_empty[buf]);
        }
    }
    if (!ok) atomicExch(err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 8)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * cols));
}

inline size_t smem_bytes_ws() { return sizeof(SmemWS) + 1024; }

// ---------------------------------------------------------------------------
// Activation view: the input of a 3x3 convolution at resolution H x W, NHWC
// BF16.  Channels [0, c1) come from s1, stored at (H >> up1) x (W >> up1)
// (nearest-neighbour upsampling when up1 = 1); channels [c1, c1 + c2) come from
// s2 at H x W.  This is the decoder's "upsample, then concatenate the skip"
// without materialising either.
struct ActView {
    const __nv_bfloat16 *s1;
    const __nv_bfloat16 *s2;
    int c1, c2, up1;
    int B, H, W;
    __device__ __forceinline__ int C() const { return c1 + c2; }
    // Address of channels [c, c+8) of pixel (b, h, w); valid = false (and a
    // harmless address) outside the image.
    __device__ __forceinline__ const __nv_bfloat16 *chunk_ptr(int b, int h, int w, int c,
                                                              bool &valid) const {
        valid = h >= 0 && h < H && w >= 0 && w < W;
        if (!valid) return s1;
        if (c < c1) {
            const int Hs = H >> up1, Ws = W >> up1;
            const size_t p = ((size_t)b * Hs + (h >> up1)) * Ws + (w >> up1);
            return s1 + p * c1 + c;
        }
        const size_t p = ((size_t)b * H + h) * W + w;
        return s2 + p * c2 + (c - c1);
    }
    // 8 channels [c, c+8) of pixel (b, h, w); zero outside the image.
    __device__ __forceinline__ uint4 chunk(int b, int h, int w, int c) const {
        if (h < 0 || h >= H || w < 0 || w >= W) return make_uint4(0, 0, 0, 0);
        if (c < c1) {
            const int Hs = H >> up1, Ws = W >> up1;
            const size_t p = ((size_t)b * Hs + (h >> up1)) * Ws + (w >> up1);
            return __ldg(reinterpret_cast<const uint4 *>(s1 + p * c1 + c));
        }
        const size_t p = ((size_t)b * H + h) * W + w;
        return __ldg(reinterpret_cast<const uint4 *>(s2 + p * c2 + (c - c1)));
    }
};

// Source of the weight gradient's bias row: BF16 1.0 followed by seven zeros.
static __device__ __align__(16) const unsigned short kOneChunk[8] = {0x3F80u, 0, 0, 0, 0, 0, 0, 0};

__device__ __forceinline__ void pixel_of(int m, int H, int W, int &b, int &h, int &w) {
    const int hw = H * W;
    b = m / hw;
    const int r = m - b * hw;
    h = r / W;
    w = r - h * W;
}

// Epilogue of a convolution tile: + bias, ReLU, multiply by (mask view > 0),
// store BF16 or FP32 rows of [M][Nout].
struct ConvStore {
    const float *bias;  // [Nout] or null
    ActView mask;       // mask.s1 == null: no mask
    void *out;          // [M][Nout] BF16 or FP32
    int M, Nout, bn, relu, out_f32;
    int store_cols;     // store_row(): output columns written (0: all); the rest nobody reads

    __device__ void store(int row, int col, const float *v, const uint3 &t) const {
        const int m = t.x * BM + row;
        if (m >= M) return;
        const int n = t.y * bn + col;
        float o[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            float t = v[i] + (bias ? bias[n + i] : 0.f);
            o[i] = relu ? fmaxf(t, 0.f) : t;
        }
        if (mask.s1) {
            int b, h, w;
            pixel_of(m, mask.H, mask.W, b, h, w);
            const uint4 mv = mask.chunk(b, h, w, n);
            const __nv_bfloat16 *mb = reinterpret_cast<const __nv_bfloat16 *>(&mv);
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (!(__bfloat162float(mb[i]) > 0.f)) o[i] = 0.f;
        }
        if (out_f32) {
            float4 *d = reinterpret_cast<float4 *>((float *)out + (size_t)m * Nout + n);
            d[0] = make_float4(o[0], o[1], o[2], o[3]);
            d[1] = make_float4(o[4], o[5], o[6], o[7]);
        } else {
            __align__(16) __nv_bfloat162 p[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) p[i] = __floats2bfloat162_rn(o[2 * i], o[2 * i + 1]);
            *reinterpret_cast<uint4 *>((__nv_bfloat16 *)out + (size_t)m * Nout + n) =
                *reinterpret_cast<const uint4 *>(p);
        }
    }

    // The same epilogue with the row's pixel and mask addresses derived once
    // per tile row (row()) rather than once per 8 columns (store_row()).
    struct Row {
        const __nv_bfloat16 *m1, *m2;  // mask channels [0, c1) and [c1, c1 + c2) of the row's pixel
        size_t o;                      // output offset of the row
        bool live;
    };
    __device__ Row row(int r, const uint3 &t) const {
        Row R;
        const int m = t.x * BM + r;
        R.live = m < M;
        R.o = (size_t)m * Nout;
        R.m1 = R.m2 = nullptr;
        if (mask.s1 && R.live) {
            int b, h, w;
            pixel_of(m, mask.H, mask.W, b, h, w);
            const int Hs = mask.H >> mask.up1, Ws = mask.W >> mask.up1;
            R.m1 = mask.s1 + (((size_t)b * Hs + (h >> mask.up1)) * Ws + (w >> mask.up1)) * mask.c1;
            if (mask.s2) R.m2 = mask.s2 + (((size_t)b * mask.H + h) * mask.W + w) * mask.c2;
        }
        return R;
    }
    __device__ void store_row(const Row &R, int col, const float *v, const uint3 &t) const {
        const int n = t.y * bn + col;
        if (!R.live || (store_cols && n >= store_cols)) return;
        float o[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            float t = v[i] + (bias ? bias[n + i] : 0.f);
            o[i] = relu ? fmaxf(t, 0.f) : t;
        }
        if (mask.s1) {
            const uint4 mv =
                __ldg(reinterpret_cast<const uint4 *>(n < mask.c1 ? R.m1 + n : R.m2 + (n - mask.c1)));
            const __nv_bfloat16 *mb = reinterpret_cast<const __nv_bfloat16 *>(&mv);
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (!(__bfloat162float(mb[i]) > 0.f)) o[i] = 0.f;
        }
        if (out_f32) {
            float4 *d = reinterpret_cast<float4 *>((float *)out + R.o + n);
            d[0] = make_float4(o[0], o[1], o[2], o[3]);
            d[1] = make_float4(o[4], o[5], o[6], o[7]);
        } else {
            __align__(16) __nv_bfloat162 p[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) p[i] = __floats2bfloat162_rn(o[2 * i], o[2 * i + 1]);
            *reinterpret_cast<uint4 *>((__nv_bfloat16 *)out + R.o + n) = *reinterpret_cast<const uint4 *>(p);
        }
    }
};

// Convolution forward (and data gradient): D[m, n] = sum_k X9[m, k] Wt[n, k],
// k = tap * C + c, tap = (dy + 1) * 3 + (dx + 1), X9[m, k] = X[pixel m shifted
// by (dy, dx), channel c].  Wt is [Nout][Kp] BF16 with Kp = roundup(9 C, 64).
struct ConvOp : ConvStore {
    static constexpr bool A_MN = false, B_MN = false;
    ActView x;
    const __nv_bfloat16 *wt;  // [Nout][Kp]
    int Kp, nsteps;

    __device__ void k_range(const uint3 &t, int &k0, int &k1) const { k0 = 0; k1 = nsteps; }

    __device__ void load_a(uint32_t s, int kt, const uint3 &t) const {
        const int r = threadIdx.x;  // one tile row (pixel) per thread
        const int m = t.x * BM + r;
        const int C = x.C(), K9 = 9 * C;
        int b = 0, h = 0, w = 0;
        const bool live = m < M;
        if (live) pixel_of(m, x.H, x.W, b, h, w);
        // (tap, c) of the step's first chunk by one division; the next chunks
        // step c by 8 and carry into tap (C is a multiple of 8)
        int tap = (kt * BK) / C, c = kt * BK - tap * C;
#pragma unroll
        for (int kc = 0; kc < 8; ++kc) {
            const int k = kt * BK + kc * 8;
            bool v = false;
            const __nv_bfloat16 *p = x.s1;
            if (live && k < K9) p = x.chunk_ptr(b, h + tap / 3 - 1, w + tap % 3 - 1, c, v);
            cp16(s + (uint32_t)(kc * BM * 16 + r * 16), p, v);
            c += 8;
            if (c >= C) { c -= C; ++tap; }
        }
    }

    __device__ void load_b(uint32_t s, int kt, const uint3 &t) const {
        const int n0 = t.y * bn;
        // chunk c = kc * bn + r; stepping c by THREADS steps (kc, r) with a carry
        int kc = threadIdx.x / bn, r = threadIdx.x - kc * bn;
        const int dk = THREADS / bn, dr = THREADS - dk * bn;
        for (int c = threadIdx.x; c < bn * 8; c += THREADS) {
            cp16(s + (uint32_t)(kc * bn * 16 + r * 16), wt + (size_t)(n0 + r) * Kp + kt * BK + kc * 8,
                 true);
            kc += dk;
            r += dr;
            if (r >= bn) { r -= bn; ++kc; }
        }
    }
};

// Weight gradient, split over pixels:
//   P[z][r, n] = sum_{m in split z} X9[m, r] dY[m, n],  r = tap * C + c,
// plus one extra row r = 9C whose A operand is 1, giving the bias gradient
// sum_m dY[m, n].  Both operands are staged MN-major: a 16-byte chunk is 8
// consecutive channels of one pixel, which is contiguous in NHWC.
struct WgradOp {
    static constexpr bool A_MN = true, B_MN = true;
    ActView x;
    const __nv_bfloat16 *dy;  // [M][Nout]
    float *part;              // [splits][9C + 1][Nout]
    int M, Nout, bn, steps_per_split, nsteps;

    __device__ void k_range(const uint3 &t, int &k0, int &k1) const {
        k0 = t.z * steps_per_split;
        k1 = min(nsteps, k0 + steps_per_split);
    }

    __device__ void load_a(uint32_t s, int kt, const uint3 &t) const {
        const int C = x.C(), R = 9 * C;
        const int k_lo = threadIdx.x & 7, g = (threadIdx.x >> 3) & 15;
        const int r = t.x * BM + g * 8;
        const int tap = r / C, c = r - tap * C;
        const int dy = tap / 3 - 1, dx = tap % 3 - 1;
        // pixel of the step's first chunk by one pixel_of; the next chunks
        // are 8 pixels on (one row carry when the image is at least 8 wide;
        // the deepest levels of a small image may be narrower)
        int b, h, w;
        pixel_of(kt * BK + k_lo, x.H, x.W, b, h, w);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int m = kt * BK + i * 8 + k_lo;
            bool v = false;
            const void *p = x.s1;
            if (m < M) {
                if (r < R) {
                    p = x.chunk_ptr(b, h + dy, w + dx, c, v);
                } else if (r == R) {
                    p = kOneChunk;  // bf16 1.0 in element 0: the bias row
                    v = true;
                }
            }
            cp16(s + (uint32_t)(i * BM * 16 + g * 128 + k_lo * 16), p, v);
            w += 8;
            while (w >= x.W) {
                w -= x.W;
                if (++h == x.H) { h = 0; ++b; }
            }
        }
    }

    __device__ void load_b(uint32_t s, int kt, const uint3 &t) const {
        const int groups = bn >> 3, n0 = t.y * bn;
        // chunk c: k_lo = c % 8 and (c / 8) = k_hi * groups + g; stepping c by
        // THREADS steps (k_hi, g) with a carry
        const int k_lo = threadIdx.x & 7;
        int k_hi = (threadIdx.x >> 3) / groups, g = (threadIdx.x >> 3) - k_hi * groups;
        const int dq = THREADS >> 3, dk = dq / groups, dg = dq - dk * groups;
        for (int c = threadIdx.x; c < bn * 8; c += THREADS) {
            const int m = kt * BK + k_hi * 8 + k_lo;
            const bool v = m < M;
            cp16(s + (uint32_t)(k_hi * bn * 16 + g * 128 + k_lo * 16),
                 v ? (const void *)(dy + (size_t)m * Nout + n0 + g * 8) : (const void *)dy, v);
            k_hi += dk;
            g += dg;
            if (g >= groups) { g -= groups; ++k_hi; }
        }
    }

    __device__ void store(int row, int col, const float *v, const uint3 &t) const {
        const int R = 9 * x.C();
        const int r = t.x * BM + row;
        if (r > R) return;
        const int n = t.y * bn + col;
        float4 *d = reinterpret_cast<float4 *>(part + ((size_t)t.z * (R + 1) + r) * Nout + n);
        d[0] = make_float4(v[0], v[1], v[2], v[3]);
        d[1] = make_float4(v[4], v[5], v[6], v[7]);
    }
};

// Plain GEMM for testing both operand majors: C[M][N] = A B^T in FP32, with A
// stored [M][K] (K-major) or [K][M] (MN-major), B stored [N][K] or [K][N].
template <bool AMN, bool BMN>
struct GemmOp {
    static constexpr bool A_MN = AMN, B_MN = BMN;
    const __nv_bfloat16 *a, *b;
    float *c;
    int M, N, K, bn;

    __device__ void k_range(const uint3 &t, int &k0, int &k1) const { k0 = 0; k1 = K / BK; }

    __device__ static void load(uint32_t s, const __nv_bfloat16 *src, int rows, int r0, int ld_rows,
                                int K, int kt, bool mn) {
        for (int c = threadIdx.x; c < rows * 8; c += THREADS) {
            uint32_t off;
            const __nv_bfloat16 *p;
            if (!mn) {  // chunk = row r, k chunk kc
                const int r = c % rows, kc = c / rows;
                p = src + (size_t)(r0 + r) * K + kt * BK + kc * 8;
                off = (uint32_t)(kc * rows * 16 + r * 16);
            } else {    // chunk = 8 rows of one k
                const int groups = rows >> 3;
                const int k_lo = c & 7, g = (c >> 3) % groups, k_hi = (c >> 3) / groups;
                p = src + (size_t)(kt * BK + k_hi * 8 + k_lo) * ld_rows + r0 + g * 8;
                off = (uint32_t)(k_hi * rows * 16 + g * 128 + k_lo * 16);
            }
            cp16(s + off, p, true);
        }
    }
    __device__ void load_a(uint32_t s, int kt, const uint3 &t) const { load(s, a, BM, t.x * BM, M, K, kt, AMN); }
    __device__ void load_b(uint32_t s, int kt, const uint3 &t) const { load(s, b, bn, t.y * bn, N, K, kt, BMN); }
    __device__ void store(int row, int col, const float *v, const uint3 &t) const {
        const int m = t.x * BM + row, n = t.y * bn + col;
        float4 *d = reinterpret_cast<float4 *>(c + (size_t)m * N + n);
        d[0] = make_float4(v[0], v[1], v[2], v[3]);
        d[1] = make_float4(v[4], v[5], v[6], v[7]);
    }
};

}  // namespace umma
}  // namespace kb

namespace kb {
namespace umma {

// Largest multiple of 16 that is <= 128 and divides n (0 if none).
int pick_bn(int n);

// Launch umma_k<Op> with the dynamic shared memory it needs.  The attribute
// is set once per device and instantiation.
// Engine choice for the convolutions and the plain GEMM: 0 the warp-
// specialised persistent kernel with cp.async staging, 1 one CTA per tile
// with cp.async staging, 2 (default) the TMA-staged persistent kernel of
// kb_umma_tma.cuh.  Under engine 2 an operation whose shapes the TMA boxes
// cannot tile runs on engine 1 (launch() below).
int engine();

template <class Op>
int launch_ws(const Op &op, dim3 grid, int *err, cudaStream_t stream, long long spin = 1ll << 22) {
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(umma_ws_k<Op>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem_bytes_ws());
        if (e != cudaSuccess) return kb::check_launch("umma_ws_k: shared-memory attribute");
        configured[dev] = true;
    }
    const long long ntiles = (long long)grid.x * grid.y * grid.z;
    const long long ctas = ntiles < kb::sm_count() ? ntiles : kb::sm_count();
    umma_ws_k<Op><<<(unsigned)ctas, WS_THREADS, smem_bytes_ws(), stream>>>(
        op, make_uint3(grid.x, grid.y, grid.z), err, spin);
    return 0;
}

template <class Op>
int launch(const Op &op, dim3 grid, int *err, cudaStream_t stream, long long spin = 1ll << 22) {
    if (engine() == 0) return launch_ws(op, grid, err, stream, spin);  // 1 and 2: one CTA per tile
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(umma_k<Op>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem_bytes());
        if (e != cudaSuccess) return kb::check_launch("umma_k: shared-memory attribute");
        configured[dev] = true;
    }
    umma_k<Op><<<grid, THREADS, smem_bytes(), stream>>>(op, err, spin);
    return 0;
}

}  // namespace umma
}  // namespace kb
