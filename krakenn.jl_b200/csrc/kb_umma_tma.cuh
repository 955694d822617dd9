// kb_umma_tma.cuh -- TMA-staged, warp-specialised tcgen05 engine (engine 2)
// of the warm-start network's convolutions and of the plain BF16 GEMM.
//
// cps persistent CTAs per SM (64 + 128 TM_EPI threads each) loop over the
// tiles t = blockIdx.x, blockIdx.x + gridDim.x, ... of the grid `tiles` (x
// fastest).  One warp issues at most one tcgen05.mma about every 180 cycles
// whatever N is, so an N = 32 tile reaches 1/8 of the tensor rate from one
// issuer; several CTAs per SM, each with its own ring, MMA lane and share of
// TMEM, multiply the issue rate.  In each CTA:
//   warp 0    producer: lane 0 waits for a free ring stage (`empty`), posts
//             the stage's byte count on its `full` barrier and issues the
//             step's cp.async.bulk.tensor copies, one per operand box;
//   warp 1    MMA: allocates TMEM (two accumulators of the tile width);
//             lane 0 waits `full`, issues the step's tcgen05.mma, commits to
//             the stage's `empty` barrier, and to `acc_full` after a tile's
//             last step;
//   warps 2.. epilogue, TM_EPI warps per TMEM lane quarter: warp w reads
//             TMEM lanes 32(w%4)..+31 (tile rows) of the finished
//             accumulator, every TM_EPI-th group of 8 columns, calls op.store
//             and arrives on `acc_empty`, so the epilogue of tile j overlaps
//             the MMAs of tile j+1.  Several warps per quarter keep several
//             TMEM-load / store chains of a tile in flight.
// The copies carry no address arithmetic per element: a 3x3 tap of a
// convolution is one 4D box (channels, x, y, image) of the NHWC activation
// shifted by (dx, dy), and the zero padding of the image border is the
// copy's out-of-bounds fill.  No copy uses cluster multicast; every source
// is this GPU's own memory.
//
// Operand tiles are the canonical swizzled UMMA layouts that a TMA box with
// the same swizzle writes (S = 32, 64 or 128 bytes, E = S / 2 elements):
//   K-major : tile row r (a pixel, or a weight row) holds E consecutive K
//             elements in S bytes; 8-row groups are SBO = 8 S apart.  A stage
//             holds K = E: E / 16 MMAs at start offsets 0, 32, 64, 96 bytes.
//   MN-major: K row k (a pixel) holds E consecutive M (or N) elements in S
//             bytes; a block of 64 K rows is 64 S bytes, blocks along M are
//             LBO = 64 S apart, 8-row groups SBO = 8 S.  A stage holds K =
//             64: four MMAs at start offsets 0, 16 S, 32 S, 48 S.
// Every stage and block starts on a 1024-byte boundary (or a multiple of
// the swizzle period), so each tile's swizzle phase is zero and the
// descriptors' base offset is 0.
//
// Every wait is bounded.  A role that gives up records the failure in *err;
// the producer then waits (bounded) for the copies it issued, the MMA lane
// for the MMAs it issued, and TMEM is freed before the CTA exits.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include "kb_umma.cuh"

namespace kb {
namespace umma {

constexpr int TM_EPI = 2;                       // epilogue warps per TMEM lane quarter
constexpr int TM_THREADS = 64 + 128 * TM_EPI, TM_MAX_STAGES = 24, TM_MAX_CPS = 4;
constexpr uint32_t TM_RING = 200u * 1024u;  // bytes of ring + resident operand, one CTA per SM
// ... and with cps CTAs per SM (each CTA also takes barriers, alignment slack
// and the 1 KB the runtime reserves)
__host__ __device__ constexpr uint32_t tm_ring(int cps) {
    return cps <= 1 ? TM_RING : (cps == 2 ? 108u * 1024u : (cps == 3 ? 72u * 1024u : 52u * 1024u));
}

// Shared-memory matrix descriptor of a swizzled layout (sm_100 version 1).
__device__ __forceinline__ uint64_t sdesc_sw(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t swz) {
    const uint64_t layout = swz == 128u ? 2u : (swz == 64u ? 4u : 6u);
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (layout << 61);
}

// Descriptor of MMA kk (16 K elements) of a stage's operand tile.
__device__ __forceinline__ uint64_t op_desc(uint32_t base, bool mn, uint32_t swz, int kk) {
    return mn ? sdesc_sw(base + (uint32_t)kk * 16u * swz, 64u * swz, 8u * swz, swz)
              : sdesc_sw(base + (uint32_t)kk * 32u, 16u, 8u * swz, swz);
}

__device__ __forceinline__ void expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void tma2(uint32_t dst, const CUtensorMap *m, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(m)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tma4(uint32_t dst, const CUtensorMap *m, int c, int x, int y, int b,
                                     uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(m)), "r"(c), "r"(x), "r"(y), "r"(b), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void prefetch_map(const CUtensorMap *m) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(m)) : "memory");
}

// Tile coordinates (x fastest) of the tiles T = T0, T0 + G, ... one CTA
// visits: the first by division, the next ones by stepping the previous
// coordinates by G (decomposed once).
struct TileCursor {
    uint3 n, d, cur;
    int last = -1;
    __device__ explicit TileCursor(const uint3 &tiles) : n(tiles), d(), cur() {}
    __device__ uint3 at(int T) {
        if (last < 0) {
            cur.x = (unsigned)T % n.x;
            const unsigned r = (unsigned)T / n.x;
            cur.y = r % n.y;
            cur.z = r / n.y;
            const unsigned G = gridDim.x;
            d.x = G % n.x;
            d.y = (G / n.x) % n.y;
            d.z = G / (n.x * n.y);
        } else {
            cur.x += d.x;
            unsigned c = cur.x >= n.x;
            cur.x -= c ? n.x : 0u;
            cur.y += d.y + c;
            c = cur.y >= n.y;
            cur.y -= c ? n.y : 0u;
            cur.z += d.z + c;
        }
        last = T;
        return cur;
    }
};

// Fields every operation carries (set on the host).
struct TmaBase {
    uint32_t a_bytes, b_bytes;  // operand bytes of one ring stage (multiples of 1024)
    uint32_t res_bytes;         // operand bytes copied once per CTA and kept (0: none)
    uint32_t acc_cols;          // TMEM columns of one accumulator (32..512, a power of two)
    int nbuf;                   // accumulators: 2 (epilogue of tile j overlaps tile j+1) or 1
    int ncols;                  // accumulator columns the epilogue stores (multiple of 8)
    int cps;                    // CTAs per SM (tma_fit)
};

// Op interface (TmaBase plus bn, k_range and store as in the other engines):
//   static constexpr bool A_MN, B_MN;
//   __device__ uint32_t step_tx(const uint3 &t)    bytes the copies of one step of tile t bring
//   __device__ void prefetch()                     prefetch the tensor maps
//   __device__ void issue_res(uint32_t res, uint32_t bar)   copies of the resident operand
//   struct Cursor; __device__ Cursor begin(const uint3 &t, int k0)   state of step k0 of tile t
//   __device__ void issue(Cursor &c, const uint3 &t, uint32_t sa, uint32_t sb, uint32_t bar)
//                                                  copies of the cursor's step; advance it
//   __device__ void mma(uint32_t acc, uint32_t sa, uint32_t sb, uint32_t res, int kt, int k0,
//                       const uint3 &t, uint32_t idesc)   the MMAs of step kt of tile t
template <class Op>
__global__ void __launch_bounds__(TM_THREADS, TM_MAX_CPS)
    umma_tma_k(const __grid_constant__ Op op, const uint3 tiles, const int nstages,
               int *__restrict__ err, const long long spin) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    const uint32_t stage_bytes = op.a_bytes + op.b_bytes;
    const uint32_t res = base + (uint32_t)nstages * stage_bytes;  // resident operand
    uint64_t *full = reinterpret_cast<uint64_t *>(smem_raw + (base - raw) + (size_t)nstages * stage_bytes +
                                                  op.res_bytes);
    uint64_t *empty = full + nstages;
    uint64_t *acc_full = empty + nstages, *acc_empty = acc_full + 2, *drain = acc_empty + 2;
    uint64_t *resbar = drain + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(resbar + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t cols = op.acc_cols;
    const int nbuf = op.nbuf;
    const int ntiles = (int)(tiles.x * tiles.y * tiles.z);  // < 2^31 (checked by launch_tma)

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_slot)), "r"((uint32_t)nbuf * cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < nstages; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&acc_full[i], 1);
            mbar_init(&acc_empty[i], 128 * TM_EPI);
        }
        mbar_init(drain, 1);
        mbar_init(resbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    bool ok = true;

    // Ring position (slot s, parity `par` of its current use) and tile
    // coordinates advance incrementally: the producer and MMA lanes are
    // single threads, and a division per step would be their critical path.
    if (warp == 0) {
        // ---------------------------------------------------------- producer
        if (lane == 0) {
            op.prefetch();
            if (op.res_bytes) {
                expect_tx(smem_u32(resbar), op.res_bytes);
                op.issue_res(res, smem_u32(resbar));
            }
            long long g = 0;
            int s = 0;
            uint32_t par = 0;
            TileCursor tc(tiles);
            for (int T = blockIdx.x; T < ntiles && ok; T += gridDim.x) {
                const uint3 t = tc.at(T);
                int k0, k1;
                op.k_range(t, k0, k1);
                const uint32_t tx = op.step_tx(t);
                typename Op::Cursor cur = op.begin(t, k0);
                for (int kt = k0; kt < k1; ++kt, ++g) {
                    if (g >= nstages && !(ok = mbar_wait(&empty[s], par ^ 1u, spin))) break;
                    const uint32_t sa = base + (uint32_t)s * stage_bytes;
                    const uint32_t bar = smem_u32(&full[s]);
                    expect_tx(bar, tx);
                    op.issue(cur, t, sa, sa + op.a_bytes, bar);
                    if (++s == nstages) {
                        s = 0;
                        par ^= 1u;
                    }
                }
            }
            // the copies this thread issued have all landed before it leaves
            // (on the normal path they have: the MMAs consumed them)
            for (long long i = 0; i < g && i < nstages; ++i) {
                if (s == 0) {
                    s = nstages;
                    par ^= 1u;
                }
                --s;
                if (!mbar_wait(&full[s], par, spin)) ok = false;
            }
            if (op.res_bytes && !mbar_wait(resbar, 0u, spin)) ok = false;
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------------------------------------------------- MMA issue
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16(op.bn, Op::A_MN, Op::B_MN);
            int s = 0, j = 0;
            uint32_t par = 0;
            if (op.res_bytes) ok = mbar_wait(resbar, 0u, spin);
            TileCursor tc(tiles);
            for (int T = blockIdx.x; T < ntiles && ok; T += gridDim.x, ++j) {
                const int buf = nbuf == 2 ? (j & 1) : 0, use = nbuf == 2 ? (j >> 1) : j;
                if (use >= 1 && !(ok = mbar_wait(&acc_empty[buf], (uint32_t)((use - 1) & 1), spin))) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint3 t = tc.at(T);
                int k0, k1;
                op.k_range(t, k0, k1);
                const uint32_t acc = tmem + (uint32_t)buf * cols;
                for (int kt = k0; kt < k1; ++kt) {
                    if (!(ok = mbar_wait(&full[s], par, spin))) break;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sa = base + (uint32_t)s * stage_bytes;
                    op.mma(acc, sa, sa + op.a_bytes, res, kt, k0, t, idesc);
                    mma_commit(&empty[s]);
                    if (++s == nstages) {
                        s = 0;
                        par ^= 1u;
                    }
                }
                if (!ok) break;
                mma_commit(&acc_full[buf]);
            }
            // every MMA issued above is complete once this commit arrives
            mma_commit(drain);
            if (!mbar_wait(drain, 0u, spin)) ok = false;
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------- epilogue
        const int q = warp & 3, grp = (warp - 2) >> 2;
        const int row = q * 32 + lane;
        int j = 0;
        TileCursor tc(tiles);
        for (int T = blockIdx.x; T < ntiles && ok; T += gridDim.x, ++j) {
            const int buf = nbuf == 2 ? (j & 1) : 0, use = nbuf == 2 ? (j >> 1) : j;
            if (!(ok = mbar_wait(&acc_full[buf], (uint32_t)(use & 1), spin))) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint3 t = tc.at(T);
            int k0, k1;
            op.k_range(t, k0, k1);
            const auto R = op.row(row, t);  // per-row state, once per tile
            if (k1 > k0) {
                for (int c0 = grp * 8; c0 < op.ncols; c0 += 8 * TM_EPI) {
                    float v[8];
                    tmem_ld8(tmem + (uint32_t)buf * cols + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, v);
                    op.store_row(R, c0, v, t);
                }
            } else {
                const float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                for (int c0 = grp * 8; c0 < op.ncols; c0 += 8 * TM_EPI) op.store_row(R, c0, z, t);
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            mbar_arrive(&acc_empty[buf]);
        }
    }
    if (!ok) atomicExch(err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"((uint32_t)nbuf * cols));
}

// Ring stages that fit beside a resident operand of `res_bytes` with cps
// CTAs per SM, and the dynamic shared memory of a launch with that many stages.
inline int tma_stages(uint32_t stage_bytes, uint32_t res_bytes, int cps = 1) {
    const uint32_t ring = tm_ring(cps);
    if (res_bytes >= ring) return 0;
    const int n = (int)((ring - res_bytes) / stage_bytes);
    return n > TM_MAX_STAGES ? TM_MAX_STAGES : n;
}
inline size_t tma_smem_bytes(int nstages, uint32_t stage_bytes, uint32_t res_bytes) {
    return 1024 + (size_t)nstages * stage_bytes + res_bytes + (size_t)(2 * nstages + 6) * 8 + 16;
}
// Most CTAs per SM (<= TM_MAX_CPS) whose rings hold >= 2 stages and whose
// accumulators fit TMEM together; 0 if not even one CTA fits.
inline int tma_fit(const TmaBase &b) {
    for (int c = TM_MAX_CPS; c >= 1; --c)
        if (tma_stages(b.a_bytes + b.b_bytes, b.res_bytes, c) >= 2 &&
            (uint32_t)c * (uint32_t)b.nbuf * b.acc_cols <= 512u && c * TM_THREADS <= 2048)
            return c;
    return 0;
}
constexpr size_t TM_SMEM_MAX = 1024 + TM_RING + (2 * TM_MAX_STAGES + 6) * 8 + 16;

// ---------------------------------------------------------------------------
// Operations.

__device__ __forceinline__ void split_pixel(int p, int H, int W, int &b, int &y, int &x) {
    const int hw = H * W;
    b = p / hw;
    const int r = p - b * hw;
    y = r / W;
    x = r - y * W;
}

// Convolution forward (and data gradient) with TMA-staged operands:
// D[m, n] = sum over taps and channel chunks of X[pixel m + (dy, dx), c] W[n, tap C + c].
// X is channels [0, c1) of x1 and [c1, C) of x2 (both NHWC at H x W); a step
// is one tap and one chunk of e channels (box e x 128 pixels), K-major with
// swizzle 2e; the weights [Nout][Kp] are boxes of e K elements x bn rows.
struct ConvTma : ConvStore, TmaBase {
    static constexpr bool A_MN = false, B_MN = false;
    CUtensorMap x1, x2, w;
    int e, c1, C, H, W, nck;
    uint32_t tx;

    __device__ void k_range(const uint3 &, int &k0, int &k1) const { k0 = 0; k1 = 9 * nck; }
    __device__ uint32_t step_tx(const uint3 &) const { return tx; }
    __device__ void prefetch() const {
        prefetch_map(&x1);
        if (c1 < C) prefetch_map(&x2);
        prefetch_map(&w);
    }
    // step cursor: channel c of the chunk, tap offsets (dx, dy), weight column
    // wk = tap C + c, and the tile's first pixel (b, y, x)
    struct Cursor { int c, dx, dy, wk, b, y, x; };
    __device__ Cursor begin(const uint3 &t, int) const {
        Cursor u;
        split_pixel((int)t.x * BM, H, W, u.b, u.y, u.x);
        u.c = 0;
        u.dx = -1;
        u.dy = -1;
        u.wk = 0;
        return u;
    }
    __device__ void issue(Cursor &u, const uint3 &t, uint32_t sa, uint32_t sb, uint32_t bar) const {
        if (u.c < c1) tma4(sa, &x1, u.c, u.x + u.dx, u.y + u.dy, u.b, bar);
        else tma4(sa, &x2, u.c - c1, u.x + u.dx, u.y + u.dy, u.b, bar);
        tma2(sb, &w, u.wk, (int)t.y * bn, bar);
        u.wk += e;
        u.c += e;
        if (u.c == C) {
            u.c = 0;
            if (++u.dx == 2) {
                u.dx = -1;
                ++u.dy;
            }
        }
    }
    __device__ void issue_res(uint32_t, uint32_t) const {}
    __device__ void mma(uint32_t acc, uint32_t sa, uint32_t sb, uint32_t, int kt, int k0, const uint3 &,
                        uint32_t idesc) const {
        const bool first = kt == k0;
        const uint32_t s = 2u * (uint32_t)e;
        for (int kk = 0; kk < e / 16; ++kk)
            mma_bf16(acc, op_desc(sa, false, s, kk), op_desc(sb, false, s, kk), idesc,
                     (first && kk == 0) ? 0u : 1u);
    }
};

// Convolution (forward or data gradient) of rows that are a multiple of 128
// pixels wide, by row strips: a tile is 128 pixels of one row, a step is one
// kernel row dy.  The step's copies are one strip per channel chunk, pixels
// x0-1 .. x0+128 of row y+dy (box e x 130, K-major, swizzle 2e), so an
// activation row crosses to shared memory three times instead of nine.  The
// MMAs of tap dx read the strip from row dx+1 on: the tensor core applies the
// swizzle to the absolute shared-memory address, so a start 2e bytes further
// reads the rows shifted by one pixel.  The layer's weights (9 nck blocks of
// bn x e, one output-channel tile) are the resident operand, in tap, chunk,
// 16-wide K group order (the other engines' order); or, where that lets more
// CTAs share an SM, they are streamed: a stage is then one kernel row and one
// chunk, its strip and the three taps' weight blocks (order row, chunk, tap).
struct ConvStrip : ConvStore, TmaBase {
    static constexpr bool A_MN = false, B_MN = false;
    CUtensorMap x1, x2, w;
    int e, c1, C, H, W, nck;
    int streamed;  // 1: weights copied per stage (kernel row dy, chunk) instead of resident
    uint32_t strip_bytes, tx;

    __device__ void k_range(const uint3 &, int &k0, int &k1) const {
        k0 = 0;
        k1 = streamed ? 3 * nck : 3;
    }
    __device__ uint32_t step_tx(const uint3 &) const { return tx; }
    __device__ void prefetch() const {
        prefetch_map(&x1);
        if (c1 < C) prefetch_map(&x2);
        prefetch_map(&w);
    }
    __device__ void issue_res(uint32_t res, uint32_t bar) const {
        if (streamed) return;
        const uint32_t blk = (uint32_t)(bn * 2 * e);
        for (int j = 0, wk = 0; j < 9 * nck; ++j, wk += e) tma2(res + (uint32_t)j * blk, &w, wk, 0, bar);
    }
    struct Cursor { int dy, ci, b, y, x; };
    __device__ Cursor begin(const uint3 &t, int) const {
        Cursor u;
        split_pixel((int)t.x * BM, H, W, u.b, u.y, u.x);
        u.dy = -1;
        u.ci = 0;
        return u;
    }
    __device__ void issue(Cursor &u, const uint3 &, uint32_t sa, uint32_t sb, uint32_t bar) const {
        if (streamed) {
            // one strip (row y + dy, chunk ci) and the three taps' weight blocks
            const int c = u.ci * e;
            if (c < c1) tma4(sa, &x1, c, u.x - 1, u.y + u.dy, u.b, bar);
            else tma4(sa, &x2, c - c1, u.x - 1, u.y + u.dy, u.b, bar);
            const uint32_t blk = (uint32_t)(bn * 2 * e);
            const int wk0 = (u.dy + 1) * 3 * C + c;  // tap (dy + 1) * 3 + (dx + 1)
            for (int dx = 0; dx < 3; ++dx) tma2(sb + (uint32_t)dx * blk, &w, wk0 + dx * C, 0, bar);
            if (++u.ci == nck) {
                u.ci = 0;
                ++u.dy;
            }
            return;
        }
        uint32_t dst = sa;
        for (int ci = 0, c = 0; ci < nck; ++ci, c += e, dst += strip_bytes) {
            if (c < c1) tma4(dst, &x1, c, u.x - 1, u.y + u.dy, u.b, bar);
            else tma4(dst, &x2, c - c1, u.x - 1, u.y + u.dy, u.b, bar);
        }
        ++u.dy;
    }
    __device__ void mma(uint32_t acc, uint32_t sa, uint32_t sb, uint32_t res, int kt, int, const uint3 &,
                        uint32_t idesc) const {
        const uint32_t S = 2u * (uint32_t)e, blk = (uint32_t)bn * S;
        if (streamed) {
            for (int dx = 0; dx < 3; ++dx)
                for (int kk = 0; kk < e / 16; ++kk)
                    mma_bf16(acc, op_desc(sa + (uint32_t)dx * S, false, S, kk),
                             op_desc(sb + (uint32_t)dx * blk, false, S, kk), idesc,
                             (kt == 0 && dx == 0 && kk == 0) ? 0u : 1u);
            return;
        }
        uint32_t wb = res + (uint32_t)(kt * 3 * nck) * blk;  // tap kt*3 + dx
        for (int dx = 0; dx < 3; ++dx)
            for (int ci = 0; ci < nck; ++ci, wb += blk) {
                const uint32_t a = sa + (uint32_t)ci * strip_bytes + (uint32_t)dx * S;
                for (int kk = 0; kk < e / 16; ++kk)
                    mma_bf16(acc, op_desc(a, false, S, kk), op_desc(wb, false, S, kk), idesc,
                             (kt == 0 && dx == 0 && ci == 0 && kk == 0) ? 0u : 1u);
            }
    }
};

// Weight gradient of rows that are a multiple of 64 pixels wide, one whole
// gradient per tile: the tiles are the pixel splits, and a tile accumulates
// every row r = tap C + c (and the bias row) in TMEM.  A step is 64 pixels
// of one row.  Its copies are, per kernel row dy and channel chunk, one strip
// of pixels x-1 .. x+sr-2 (box ea x sr, MN-major, swizzle 2ea), and the
// step's output gradient (nb blocks of eb channels x 64 pixels), so each
// input row crosses three times and each output-gradient row once.  M-tile m
// = (dy, chunk, h) reads its strip with the blocks one row apart (LBO = 2ea
// bytes): block j is the strip shifted by j pixels, i.e. tap dx = 2h - 1 + j
// (blocks of taps beyond +1 are computed and not stored).  The bias M-tile
// reads the resident `ones` rows (1 in channel 0).  Accumulator m holds
// columns m bn .. m bn + bn - 1; the epilogue maps (m, row) to r.
struct WgradStrip : TmaBase {
    static constexpr bool A_MN = true, B_MN = true;
    CUtensorMap x1, x2, ones, dy;
    float *part;  // [splits][9C + 1][Nout]
    int bn, ea, eb, c1, C, H, W, Nout, steps_per_split, nsteps;
    int cpt, mtp, nb, nmt, ea_shift, bn_shift;  // chunks per tile, M-tiles per strip (1, 2), dY blocks, strip M-tiles
    uint32_t strip_bytes, tx;

    __device__ void k_range(const uint3 &t, int &k0, int &k1) const {
        k0 = (int)t.z * steps_per_split;
        k1 = min(nsteps, k0 + steps_per_split);
    }
    __device__ uint32_t step_tx(const uint3 &) const { return tx; }
    __device__ void prefetch() const {
        prefetch_map(&x1);
        if (c1 < C) prefetch_map(&x2);
        prefetch_map(&ones);
        prefetch_map(&dy);
    }
    __device__ void issue_res(uint32_t res, uint32_t bar) const { tma2(res, &ones, 0, 0, bar); }
    struct Cursor { int b, y, x; };
    __device__ Cursor begin(const uint3 &, int k0) const {
        Cursor u;
        split_pixel(k0 * BK, H, W, u.b, u.y, u.x);
        return u;
    }
    __device__ void issue(Cursor &u, const uint3 &t, uint32_t sa, uint32_t sb, uint32_t bar) const {
        uint32_t dst = sa;
        const int cg = (int)t.x * cpt * ea;  // first channel of this tile's chunk group
        for (int dyi = -1; dyi <= 1; ++dyi)
            for (int ci = 0, c = cg; ci < cpt; ++ci, c += ea, dst += strip_bytes) {
                if (c < c1) tma4(dst, &x1, c, u.x - 1, u.y + dyi, u.b, bar);
                else tma4(dst, &x2, c - c1, u.x - 1, u.y + dyi, u.b, bar);
            }
        for (int j = 0; j < nb; ++j) tma4(sb + (uint32_t)(j * 128 * eb), &dy, j * eb, u.x, u.y, u.b, bar);
        u.x += BK;
        if (u.x == W) {
            u.x = 0;
            if (++u.y == H) {
                u.y = 0;
                ++u.b;
            }
        }
    }
    __device__ void mma(uint32_t acc, uint32_t sa, uint32_t sb, uint32_t res, int kt, int k0, const uint3 &t,
                        uint32_t idesc) const {
        const bool first = kt == k0;
        const uint32_t sA = 2u * (uint32_t)ea, sB = 2u * (uint32_t)eb;
        uint32_t a0 = sa, accm = acc;
        for (int st = 0; st < 3 * cpt; ++st, a0 += strip_bytes)
            for (int h = 0; h < mtp; ++h, accm += (uint32_t)bn) {
                const uint32_t start = a0 + (uint32_t)(2 * h) * sA;
#pragma unroll
                for (int kk = 0; kk < BK / 16; ++kk)
                    mma_bf16(accm, sdesc_sw(start + (uint32_t)kk * 16u * sA, sA, 8u * sA, sA),
                             op_desc(sb, true, sB, kk), idesc, (first && kk == 0) ? 0u : 1u);
            }
        if (t.x != 0) return;  // the bias row belongs to chunk group 0
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk)
            mma_bf16(accm, sdesc_sw(res + (uint32_t)kk * 16u * sA, sA, 8u * sA, sA), op_desc(sb, true, sB, kk),
                     idesc, (first && kk == 0) ? 0u : 1u);
    }
    __device__ void store(int row, int col, const float *v, const uint3 &t) const {
        const int m = col >> bn_shift, n = col & (bn - 1);
        const int R = 9 * C;
        int r;
        if (m == nmt) {
            if (row != 0 || t.x != 0) return;
            r = R;
        } else {
            const int st = mtp == 2 ? (m >> 1) : m, h = m - st * mtp;
            const int dyi = st / cpt, ci = (int)t.x * cpt + st - dyi * cpt;
            const int j = row >> ea_shift, c = row & (ea - 1);
            const int dx = 2 * h - 1 + j;
            if (dx > 1) return;
            r = (dyi * 3 + dx + 1) * C + ci * ea + c;
        }
        float4 *d = reinterpret_cast<float4 *>(part + ((size_t)t.z * (R + 1) + r) * Nout + n);
        d[0] = make_float4(v[0], v[1], v[2], v[3]);
        d[1] = make_float4(v[4], v[5], v[6], v[7]);
    }
    struct Row { int r; };
    __device__ Row row(int r, const uint3 &) const { return Row{r}; }
    __device__ void store_row(const Row &R, int col, const float *v, const uint3 &t) const {
        store(R.r, col, v, t);
    }
};

// Weight gradient with TMA-staged operands, split over pixels:
//   P[z][r, n] = sum_{pixels m of split z} X[m + shift(tap), c] dY[m, n],
// r = tap C + c, plus the bias row r = 9C whose A operand is 1 (a constant
// block copied from `ones`).  Both operands are MN-major: a block is e
// channels x 64 pixels (swizzle 2e), the A tile is 128 / ea blocks of rows,
// the B tile bn / eb blocks of output channels.  Blocks past the bias row
// are not copied (their rows are not stored).
struct WgradTma : TmaBase {
    static constexpr bool A_MN = true, B_MN = true;
    CUtensorMap x1, x2, ones, dy;
    float *part;  // [splits][9C + 1][Nout]
    int bn, ea, eb, c1, C, H, W, Nout, steps_per_split, nsteps;
    int py, pb;  // rows (W < 64) or images (H W < 64) per 64-pixel step, else 0
    int na, nb;  // blocks of the A tile (BM / ea) and of the B tile (bn / eb)

    __device__ void k_range(const uint3 &t, int &k0, int &k1) const {
        k0 = (int)t.z * steps_per_split;
        k1 = min(nsteps, k0 + steps_per_split);
    }
    __device__ uint32_t step_tx(const uint3 &t) const {
        const int R = 9 * C, r0 = (int)t.x * BM;
        int xr = R - r0;
        xr = xr < 0 ? 0 : (xr > BM ? BM : xr);
        const int blocks = xr / ea + ((R >= r0 && R < r0 + BM) ? 1 : 0);
        return (uint32_t)(blocks * 128 * ea + bn * 128);
    }
    __device__ void prefetch() const {
        prefetch_map(&x1);
        if (c1 < C) prefetch_map(&x2);
        prefetch_map(&ones);
        prefetch_map(&dy);
    }
    // step cursor: the step's first pixel (b, y, x) and the (tap, c) of the
    // tile's first row
    struct Cursor { int b, y, x, tap0, c0; };
    __device__ Cursor begin(const uint3 &t, int k0) const {
        Cursor u;
        split_pixel(k0 * BK, H, W, u.b, u.y, u.x);
        const int r0 = (int)t.x * BM;
        u.tap0 = r0 / C;
        u.c0 = r0 - u.tap0 * C;
        return u;
    }
    __device__ void issue(Cursor &u, const uint3 &t, uint32_t sa, uint32_t sb, uint32_t bar) const {
        const int R = 9 * C;
        int r = (int)t.x * BM, tap = u.tap0, c = u.c0;
        for (int j = 0; j < na; ++j, r += ea) {
            const uint32_t dst = sa + (uint32_t)(j * 128 * ea);
            if (r < R) {
                const int dyy = tap / 3 - 1, dxx = tap % 3 - 1;
                if (c < c1) tma4(dst, &x1, c, u.x + dxx, u.y + dyy, u.b, bar);
                else tma4(dst, &x2, c - c1, u.x + dxx, u.y + dyy, u.b, bar);
            } else if (r == R) {
                tma2(dst, &ones, 0, 0, bar);
            }
            c += ea;
            if (c == C) {
                c = 0;
                ++tap;
            }
        }
        for (int j = 0; j < nb; ++j)
            tma4(sb + (uint32_t)(j * 128 * eb), &dy, (int)t.y * bn + j * eb, u.x, u.y, u.b, bar);
        // next 64 pixels: along the row (W >= 64), whole rows (py = 64 / W)
        // or whole images (pb = 64 / (H W))
        if (pb) {
            u.b += pb;
        } else if (py) {
            u.y += py;
            if (u.y == H) {
                u.y = 0;
                ++u.b;
            }
        } else {
            u.x += BK;
            if (u.x == W) {
                u.x = 0;
                if (++u.y == H) {
                    u.y = 0;
                    ++u.b;
                }
            }
        }
    }
    __device__ void issue_res(uint32_t, uint32_t) const {}
    __device__ void mma(uint32_t acc, uint32_t sa, uint32_t sb, uint32_t, int kt, int k0, const uint3 &,
                        uint32_t idesc) const {
        const bool first = kt == k0;
        const uint32_t s_a = 2u * (uint32_t)ea, s_b = 2u * (uint32_t)eb;
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk)
            mma_bf16(acc, op_desc(sa, true, s_a, kk), op_desc(sb, true, s_b, kk), idesc,
                     (first && kk == 0) ? 0u : 1u);
    }
    __device__ void store(int row, int col, const float *v, const uint3 &t) const {
        const int R = 9 * C;
        const int r = (int)t.x * BM + row;
        if (r > R) return;
        const int n = (int)t.y * bn + col;
        float4 *d = reinterpret_cast<float4 *>(part + ((size_t)t.z * (R + 1) + r) * Nout + n);
        d[0] = make_float4(v[0], v[1], v[2], v[3]);
        d[1] = make_float4(v[4], v[5], v[6], v[7]);
    }
    struct Row { int r; };
    __device__ Row row(int r, const uint3 &) const { return Row{r}; }
    __device__ void store_row(const Row &R, int col, const float *v, const uint3 &t) const {
        store(R.r, col, v, t);
    }
};

// Plain GEMM (test of the swizzled layouts): C[M][N] = A B^T in FP32, A
// stored [M][K] (K-major: boxes 64 K x 128 rows) or [K][M] (MN-major: two
// boxes of 64 M x 64 K), B stored [N][K] (box 64 K x bn) or [K][N] (boxes of
// eb N x 64 K).  A stage holds K = 64.
template <bool AMN, bool BMN>
struct GemmTma : TmaBase {
    static constexpr bool A_MN = AMN, B_MN = BMN;
    CUtensorMap ma, mb;
    float *c;
    int M, N, K, bn, eb, nb;  // nb = bn / eb

    __device__ void k_range(const uint3 &, int &k0, int &k1) const { k0 = 0; k1 = K / BK; }
    __device__ uint32_t step_tx(const uint3 &) const { return (uint32_t)(BM * BK * 2 + bn * BK * 2); }
    __device__ void prefetch() const {
        prefetch_map(&ma);
        prefetch_map(&mb);
    }
    struct Cursor { int k; };
    __device__ Cursor begin(const uint3 &, int k0) const { return Cursor{k0 * BK}; }
    __device__ void issue(Cursor &u, const uint3 &t, uint32_t sa, uint32_t sb, uint32_t bar) const {
        if (!AMN) {
            tma2(sa, &ma, u.k, (int)t.x * BM, bar);
        } else {
            tma2(sa, &ma, (int)t.x * BM, u.k, bar);
            tma2(sa + 8192u, &ma, (int)t.x * BM + 64, u.k, bar);
        }
        if (!BMN) {
            tma2(sb, &mb, u.k, (int)t.y * bn, bar);
        } else {
            for (int j = 0; j < nb; ++j)
                tma2(sb + (uint32_t)(j * 128 * eb), &mb, (int)t.y * bn + j * eb, u.k, bar);
        }
        u.k += BK;
    }
    __device__ void issue_res(uint32_t, uint32_t) const {}
    __device__ void mma(uint32_t acc, uint32_t sa, uint32_t sb, uint32_t, int kt, int k0, const uint3 &,
                        uint32_t idesc) const {
        const bool first = kt == k0;
        const uint32_t s_b = BMN ? 2u * (uint32_t)eb : 128u;
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk)
            mma_bf16(acc, op_desc(sa, AMN, 128u, kk), op_desc(sb, BMN, s_b, kk), idesc,
                     (first && kk == 0) ? 0u : 1u);
    }
    __device__ void store(int row, int col, const float *v, const uint3 &t) const {
        const int m = (int)t.x * BM + row, n = (int)t.y * bn + col;
        float4 *d = reinterpret_cast<float4 *>(c + (size_t)m * N + n);
        d[0] = make_float4(v[0], v[1], v[2], v[3]);
        d[1] = make_float4(v[4], v[5], v[6], v[7]);
    }
    struct Row { int r; };
    __device__ Row row(int r, const uint3 &) const { return Row{r}; }
    __device__ void store_row(const Row &R, int col, const float *v, const uint3 &t) const {
        store(R.r, col, v, t);
    }
};

}  // namespace umma
}  // namespace kb

// ---------------------------------------------------------------- host side
namespace kb {
namespace umma {

// Largest run of 16-bit elements (64, 32 or 16) that divides a and b, 0 if none.
inline int chunk_of(int a, int b = 0) {
    for (int e = 64; e >= 16; e >>= 1)
        if (a % e == 0 && b % e == 0) return e;
    return 0;
}

// A run of `px` consecutive pixels of an NHWC tensor [B][H][W] as a box
// (bx pixels of a row, by rows, bb images) that starts at a multiple of px:
// a part of one row, whole rows of one image, or whole images.
struct PixBox { int bx, by, bb; };
inline bool pix_box(int px, int H, int W, PixBox &p) {
    if (W % px == 0) { p = {px, 1, 1}; return true; }
    if (px % W) return false;
    const int r = px / W;
    if (H % r == 0) { p = {W, r, 1}; return true; }
    if (r % H) return false;
    p = {W, H, r / H};
    return true;
}

// BF16 tensor map (cuTensorMapEncodeTiled) with out-of-bounds zero fill and
// swizzle `swz` bytes (32, 64 or 128); 0 or a KB error code.
int bf16_map(CUtensorMap *m, const void *base, int rank, const cuuint64_t *dims,
             const cuuint64_t *strides, const cuuint32_t *box, int swz, const char *what);

// 4D map of an NHWC tensor [B][H][W][C] with boxes of e channels x a pixel box.
inline int nhwc_map(CUtensorMap *m, const void *base, int C, int W, int H, int B, int e,
                    const PixBox &p, const char *what) {
    const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
    const cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
    const cuuint32_t box[4] = {(cuuint32_t)e, (cuuint32_t)p.bx, (cuuint32_t)p.by, (cuuint32_t)p.bb};
    return bf16_map(m, base, 4, dims, strides, box, 2 * e, what);
}

inline uint32_t round1k(uint32_t b) { return (b + 1023u) & ~1023u; }

template <class Op>
int launch_tma(const Op &op, dim3 grid, int *err, cudaStream_t stream, long long spin = 1ll << 22) {
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(umma_tma_k<Op>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)TM_SMEM_MAX);
        if (e != cudaSuccess) return kb::check_launch("umma_tma_k: shared-memory attribute");
        configured[dev] = true;
    }
    const uint32_t stage = op.a_bytes + op.b_bytes;
    const int cps = op.cps < 1 ? 1 : (op.cps > TM_MAX_CPS ? TM_MAX_CPS : op.cps);
    const int ns = tma_stages(stage, op.res_bytes, cps);
    if (ns < 2)
        return kb::set_error(KB_ERR_ARG, "umma_tma_k: stage of %u bytes with %u resident bytes too large",
                             stage, op.res_bytes);
    if (op.nbuf < 1 || op.nbuf > 2 || (uint32_t)cps * op.nbuf * op.acc_cols > 512u || op.acc_cols < 32u ||
        (op.acc_cols & (op.acc_cols - 1u)) || op.ncols > (int)op.acc_cols || op.ncols % 8)
        return kb::set_error(KB_ERR_ARG, "umma_tma_k: accumulator shape %u x %d (store %d) invalid",
                             op.acc_cols, op.nbuf, op.ncols);
    const long long ntiles = (long long)grid.x * grid.y * grid.z;
    if (ntiles >= (1ll << 31) - (1ll << 16))
        return kb::set_error(KB_ERR_ARG, "umma_tma_k: %lld tiles exceed the tile index range", ntiles);
    const long long slots = (long long)kb::sm_count() * cps;
    const long long ctas = ntiles < slots ? ntiles : slots;
    umma_tma_k<Op><<<(unsigned)ctas, TM_THREADS, tma_smem_bytes(ns, stage, op.res_bytes), stream>>>(
        op, make_uint3(grid.x, grid.y, grid.z), ns, err, spin);
    return 0;
}

}  // namespace umma
}  // namespace kb
